"""ctypes binding of libsbletkf.so (the C ABI declared in include/sbletkf.h).

The library is built in-tree by ``sbpom_letkf_v2_b200.build``.  There is no
fallback: if the shared object is missing or cannot be loaded every entry
point raises.
"""
from __future__ import annotations

import ctypes
import os

from .params import CParams

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsbletkf.so")

OK = 0
ERR_ARG, ERR_CUDA, ERR_WORKSPACE, ERR_OBS_CELL = 1, 2, 4, 8
ERR_EIG_NOCONV, ERR_NONFINITE, ERR_EIG_NEG, ERR_ROWS, ERR_UNSUPPORTED = 16, 32, 64, 128, 256
ERR_TIMEOUT = 512
_NAMES = {ERR_ARG: "bad argument", ERR_CUDA: "CUDA error", ERR_WORKSPACE: "workspace too small",
          ERR_OBS_CELL: "obs cell index out of range", ERR_EIG_NOCONV: "Jacobi sweep cap reached",
          ERR_NONFINITE: "non-finite value", ERR_EIG_NEG: "all eigenvalues negative",
          ERR_ROWS: "search box has too many rows", ERR_UNSUPPORTED: "unsupported option",
          ERR_TIMEOUT: "bounded device wait expired"}

#: every symbol include/sbletkf.h declares
EXPORTS = ("sbletkf_abi_version", "sbletkf_workspace_create", "sbletkf_workspace_destroy",
           "sbletkf_prepare_obs", "sbletkf_analysis", "sbletkf_count_nobsl", "sbletkf_get_status",
           "sbletkf_core_batched", "sbletkf_backward", "sbletkf_analysis_noalloc",
           "sbletkf_obs_operator", "sbletkf_ensemble_mean_spread", "sbletkf_workspace_set_schedule",
           "sbletkf_latch_status", "sbletkf_obs_monitor", "sbletkf_workspace_set_item_width")
NOALLOC_MAX_OBS, NOALLOC_MAX_CELLS = 8192, 65536


class SBLETKFError(RuntimeError):
    """A non-zero status of the library (the reference would STOP)."""

    def __init__(self, code: int, where: str = ""):
        self.code = code
        names = [n for b, n in _NAMES.items() if code & b]
        super().__init__(f"{where}: status {code} ({', '.join(names) or 'unknown'})")


class CGrid(ctypes.Structure):
    _fields_ = [("nij1", ctypes.c_int32), ("reserved", ctypes.c_int32)] + [
        (n, ctypes.c_void_p) for n in ("lon1", "lat1", "ri1", "rj1", "dlon1", "dlat1", "phi1", "depth1")]


class CObsIn(ctypes.Structure):
    _fields_ = [("nobs", ctypes.c_int32), ("reserved", ctypes.c_int32)] + [
        (n, ctypes.c_void_p) for n in ("elm", "lon", "lat", "lev", "dat", "err")]


class CObsOut(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("idx", "idy", "qc", "hxmean", "hxsprd", "dep", "err", "hdxf")]


class CObs(ctypes.Structure):
    _fields_ = [("nobs", ctypes.c_int32), ("hdxf_dtype", ctypes.c_int32)] + [
        (n, ctypes.c_void_p) for n in ("elm", "idx", "idy", "lon", "lat", "lev", "err", "dep", "hdxf")]


_lib = None


def load(path: str = LIB_PATH):
    """Load libsbletkf.so (once) and declare its signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -m sbpom_letkf_v2_b200.build`")
    lib = ctypes.CDLL(path)
    vp, i32, pp = ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(CParams)
    sig = {
        "sbletkf_abi_version": ([], i32),
        "sbletkf_workspace_create": ([pp, i32, i32, i32, ctypes.POINTER(vp)], ctypes.c_int),
        "sbletkf_workspace_destroy": ([vp], ctypes.c_int),
        "sbletkf_prepare_obs": ([vp, pp, ctypes.POINTER(CObs), vp], ctypes.c_int),
        "sbletkf_analysis": ([vp, pp, ctypes.POINTER(CGrid), vp, vp, vp, vp, i32, vp, vp, vp, vp], ctypes.c_int),
        "sbletkf_count_nobsl": ([vp, pp, ctypes.POINTER(CGrid), vp, vp], ctypes.c_int),
        "sbletkf_get_status": ([vp, vp, ctypes.POINTER(i32)], ctypes.c_int),
        "sbletkf_core_batched": ([pp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp], ctypes.c_int),
        "sbletkf_backward": ([vp, pp, ctypes.POINTER(CGrid), vp, vp, i32, vp, vp, vp, vp, vp, vp, vp],
                             ctypes.c_int),
        "sbletkf_analysis_noalloc": ([pp, ctypes.POINTER(CGrid), ctypes.POINTER(CObs), vp, vp, vp, vp, i32, vp,
                                      vp, vp], ctypes.c_int),
        "sbletkf_obs_operator": ([pp, vp, vp, vp, vp, vp, vp, i32, ctypes.POINTER(CObsIn), i32,
                                  ctypes.POINTER(CObsOut), vp, vp], ctypes.c_int),
        "sbletkf_ensemble_mean_spread": ([pp, i32, vp, vp, i32, vp, vp, vp, vp, vp], ctypes.c_int),
        "sbletkf_workspace_set_schedule": ([vp, i32], ctypes.c_int),
        "sbletkf_latch_status": ([vp, i32, vp], ctypes.c_int),
        "sbletkf_obs_monitor": ([pp, i32, vp, vp, vp, vp, i32, vp, vp], ctypes.c_int),
        "sbletkf_workspace_set_item_width": ([vp, i32], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def check(code: int, where: str) -> None:
    if code != OK:
        raise SBLETKFError(code, where)
