"""Loader of the C/OpenMP restatement (oracle/letkf_ref.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference leg.  Builds the two shared objects with
oracle/Makefile when they are missing or stale and hands them OpenBLAS's
dgemm / sgemm / dsyev through scipy's cython_blas / cython_lapack capsules.
"""
from __future__ import annotations

import os

# The restatement calls BLAS from its own OpenMP threads; OpenBLAS must not
# start threads of its own (it reads this when scipy first loads it).
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

import ctypes  # noqa: E402
import subprocess  # noqa: E402

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict = {}


def build(force: bool = False) -> None:
    """Compile oracle/libletkf_ref{64,32}.so with gcc (make)."""
    args = ["make", "-s", "-C", HERE]
    if force:
        args.append("-B")
    subprocess.run(args, check=True)


def _capsule_ptr(cap) -> int:
    get_name = ctypes.pythonapi.PyCapsule_GetName
    get_name.restype = ctypes.c_char_p
    get_name.argtypes = [ctypes.py_object]
    get_ptr = ctypes.pythonapi.PyCapsule_GetPointer
    get_ptr.restype = ctypes.c_void_p
    get_ptr.argtypes = [ctypes.py_object, ctypes.c_char_p]
    return get_ptr(cap, get_name(cap))


def load(rsize: int = 8):
    """The restatement compiled with r_size = binary64 (8) or binary32 (4)."""
    if rsize in _LIBS:
        return _LIBS[rsize]
    path = os.path.join(HERE, f"libletkf_ref{64 if rsize == 8 else 32}.so")
    src = os.path.join(HERE, "letkf_ref.c")
    if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
        build()
    lib = ctypes.CDLL(path)
    from scipy.linalg import cython_blas, cython_lapack
    sfx = "64" if rsize == 8 else "32"
    setf = getattr(lib, f"ref_set_lapack{sfx}")
    setf.argtypes = [ctypes.c_void_p] * 3
    setf(_capsule_ptr(cython_lapack.__pyx_capi__["dsyev"]),
         _capsule_ptr(cython_blas.__pyx_capi__["dgemm"]),
         _capsule_ptr(cython_blas.__pyx_capi__["sgemm"]))
    fn = getattr(lib, f"ref_da_main{sfx}")
    fn.restype = ctypes.c_int
    _LIBS[rsize] = lib
    return lib


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else ctypes.c_void_p(0)


class SortedInputs:
    """Observations in cell order plus cellstart (the set_obs output)."""

    def __init__(self, params, obs: dict, rsize: int):
        rt = np.float64 if rsize == 8 else np.float32
        nlon, nlat = params.nlon, params.nlat
        idx = np.asarray(obs["idx"], np.int64)
        idy = np.asarray(obs["idy"], np.int64)
        key = (idy - 1) * nlon + (idx - 1)
        self.perm = np.argsort(key, kind="stable")
        cnt = np.bincount(key, minlength=nlon * nlat)
        self.cellstart = np.zeros(nlon * nlat + 1, np.int64)
        np.cumsum(cnt, out=self.cellstart[1:])
        pm = self.perm
        self.elm = np.ascontiguousarray(np.asarray(obs["elm"], np.int32)[pm])
        self.lon = np.ascontiguousarray(np.asarray(obs["lon"])[pm].astype(rt))
        self.lat = np.ascontiguousarray(np.asarray(obs["lat"])[pm].astype(rt))
        self.lev = np.ascontiguousarray(np.asarray(obs["lev"])[pm].astype(rt))
        self.err = np.ascontiguousarray(np.asarray(obs["err"])[pm].astype(rt))
        self.dep = np.ascontiguousarray(np.asarray(obs["dep"])[pm].astype(rt))
        self.hdxf = np.ascontiguousarray(np.asarray(obs["hdxf"])[:, pm].T.astype(rt))
        self.nobs = int(idx.size)


def da_main(params, grid: dict, obs: dict, fcst3d, fcst2d, uniforms=None, points=None,
            rsize: int = 8, nthreads: int = 0, sorted_inputs: SortedInputs | None = None,
            want_src: bool = False):
    """Run the restatement.  Returns dict(anal3d, anal2d, nobsl, status, src).

    points: optional int64 array of point ids p = k*nij1 + i to analyse (the
    other entries of anal* stay zero)."""
    lib = load(rsize)
    rt = np.float64 if rsize == 8 else np.float32
    g = {k: np.ascontiguousarray(np.asarray(v, np.float64)) for k, v in grid.items()}
    nij1 = g["lon1"].size
    si = sorted_inputs or SortedInputs(params, obs, rsize)
    f3 = np.ascontiguousarray(np.asarray(fcst3d).astype(rt))
    f2 = np.ascontiguousarray(np.asarray(fcst2d).astype(rt))
    a3 = np.zeros_like(f3)
    a2 = np.zeros_like(f2)
    P = params.nlev * nij1
    nobsl = np.full(P, -1, np.int32)
    uni = None if uniforms is None else np.ascontiguousarray(np.asarray(uniforms, np.float64))
    src = None
    if want_src and params.iswitch_da != 1:
        src = np.full((P, params.nmonte, params.nmem), -1, np.int32)
    pts = None if points is None else np.ascontiguousarray(np.asarray(points, np.int64))
    cp = params.to_c()
    sfx = "64" if rsize == 8 else "32"
    fn = getattr(lib, f"ref_da_main{sfx}")
    st = fn(ctypes.byref(cp), ctypes.c_int(nij1), _p(g["lon1"]), _p(g["lat1"]), _p(g["ri1"]), _p(g["rj1"]),
            _p(g["dlon1"]), _p(g["dlat1"]), _p(g["phi1"]), _p(g["depth1"]), ctypes.c_int(si.nobs),
            _p(si.cellstart), _p(si.elm), _p(si.lon), _p(si.lat), _p(si.lev), _p(si.err), _p(si.dep),
            _p(si.hdxf), _p(f3), _p(f2), _p(a3), _p(a2), _p(uni), _p(src), _p(nobsl),
            ctypes.c_int(-1 if pts is None else pts.size), _p(pts), ctypes.c_int(int(nthreads)))
    return dict(anal3d=a3, anal2d=a2, nobsl=nobsl.reshape(params.nlev, nij1), status=st,
                src=None if src is None else src)
