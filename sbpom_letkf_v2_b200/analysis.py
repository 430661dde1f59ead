"""Host API of the analysis step, mirroring the reference's call surface.

``Analysis.da_main(grid, fcst3d, fcst2d)`` is the counterpart of
``CALL da_main(fcst3d,fcst2d,anal3d,anal2d)`` (letkf/run/src/main.f90:92,
common_da.f90:22): the module-global observation and grid state of the
reference become ``prepare_obs(obs)`` (the sort of common_obs.f90:266-377)
and the ``grid`` mapping.  Arrays use the reference's layouts (see
include/sbletkf.h) as torch CUDA tensors; everything runs in libsbletkf.so.
Errors the reference reports with STOP raise ``SBLETKFError``.
"""
from __future__ import annotations

import ctypes

import torch

from . import _abi
from .params import F32, F64, LETKFParams

GRID_KEYS = ("lon1", "lat1", "ri1", "rj1", "dlon1", "dlat1", "phi1", "depth1")
OBS_KEYS = ("elm", "idx", "idy", "lon", "lat", "lev", "err", "dep", "hdxf")


def _stream_ptr(stream) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def _dev(t: torch.Tensor, dtype, device, name: str) -> torch.Tensor:
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"{name} must be a torch tensor")
    if t.device != device:
        raise ValueError(f"{name} is on {t.device}, expected {device}")
    if t.dtype != dtype or not t.is_contiguous():
        t = t.to(dtype).contiguous()
    return t


def _ptr(t) -> int:
    return 0 if t is None else t.data_ptr()


class Analysis:
    """One GPU's analysis step for a fixed grid and ensemble size."""

    def __init__(self, params: LETKFParams, nij1: int, max_nobs: int, device=None):
        params.validate()
        self.lib = _abi.load()
        self.params = params
        self.device = torch.device(device if device is not None else f"cuda:{torch.cuda.current_device()}")
        if self.device.type != "cuda":
            raise ValueError("the analysis runs on a CUDA device")
        self.nij1 = int(nij1)
        self.max_nobs = int(max_nobs)
        self._cp = params.to_c()
        self._ws = ctypes.c_void_p()
        idx = self.device.index if self.device.index is not None else torch.cuda.current_device()
        with torch.cuda.device(idx):
            torch.cuda.current_stream().synchronize()
            _abi.check(self.lib.sbletkf_workspace_create(ctypes.byref(self._cp), self.nij1, self.max_nobs,
                                                          idx, ctypes.byref(self._ws)), "workspace_create")
        self._keep = []
        self.nobs = None

    SCHED_AUTO, SCHED_POINT, SCHED_COLUMNS, SCHED_PIPELINE = -1, 0, 1, 2

    def set_schedule(self, schedule: int) -> None:
        """SCHED_AUTO (default): SCHED_PIPELINE for the mixed path with
        65 <= nmem <= 112, SCHED_COLUMNS for the other LETKF / LPFGM cases,
        SCHED_POINT for the LPF.  SCHED_PIPELINE (LETKF / LPFGM,
        nmem <= 112): the column walk with the next point's selection and Gram
        (producer warps) overlapped with the current point's eigensolve and
        update (consumer warps); SCHED_COLUMNS: persistent column queue with
        warm-started eigensolves; SCHED_POINT: one CTA per grid point."""
        _abi.check(self.lib.sbletkf_workspace_set_schedule(self._ws, int(schedule)), "set_schedule")

    def set_item_width(self, width: int) -> None:
        """Columns per column-queue item (0: automatic, 1..8)."""
        _abi.check(self.lib.sbletkf_workspace_set_item_width(self._ws, int(width)), "set_item_width")

    # -- lifetime ---------------------------------------------------------
    def close(self) -> None:
        if self._ws:
            self.lib.sbletkf_workspace_destroy(self._ws)
            self._ws = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _params(self, params):
        if params is None:
            return self._cp
        params.validate()
        return params.to_c()

    # -- set_obs ----------------------------------------------------------
    def prepare_obs(self, obs: dict, params: LETKFParams | None = None, stream=None) -> None:
        """Bucket the observations (common_obs.f90:266-377).  obs: elm idx idy
        (int32), lon lat lev err dep (float64) [nobs], hdxf [nmem][nobs]
        (float32 or float64)."""
        d = self.device
        nobs = int(obs["elm"].numel())
        o = {k: _dev(obs[k], torch.int32, d, k) for k in ("elm", "idx", "idy")}
        o.update({k: _dev(obs[k], torch.float64, d, k) for k in ("lon", "lat", "lev", "err", "dep")})
        h = obs["hdxf"]
        hd = torch.float64 if h.dtype == torch.float64 else torch.float32
        o["hdxf"] = _dev(h, hd, d, "hdxf")
        if nobs and tuple(o["hdxf"].shape) != (self.params.nmem, nobs):
            raise ValueError(f"hdxf must be [nmem={self.params.nmem}][nobs={nobs}], got {tuple(o['hdxf'].shape)}")
        co = _abi.CObs(nobs=nobs, hdxf_dtype=F64 if hd == torch.float64 else F32,
                       **{k: _ptr(o[k]) for k in OBS_KEYS})
        cp = self._params(params)
        _abi.check(self.lib.sbletkf_prepare_obs(self._ws, ctypes.byref(cp), ctypes.byref(co), _stream_ptr(stream)),
                   "prepare_obs")
        self._keep = [o]
        self.nobs = nobs

    def _grid(self, grid: dict):
        g = {k: _dev(grid[k], torch.float64, self.device, k) for k in GRID_KEYS}
        if g["lon1"].numel() != self.nij1 or g["depth1"].numel() != self.nij1 * self.params.nlev:
            raise ValueError("grid arrays do not match nij1 / nlev")
        return g, _abi.CGrid(nij1=self.nij1, reserved=0, **{k: _ptr(g[k]) for k in GRID_KEYS})

    # -- da_main ----------------------------------------------------------
    def da_main(self, grid: dict, fcst3d: torch.Tensor, fcst2d: torch.Tensor, uniforms=None,
                anal3d=None, anal2d=None, resample_src=None, point_status=None,
                params: LETKFParams | None = None, stream=None, check: bool = True):
        """Analysis ensemble of every grid point (common_da.f90:22-124).

        fcst3d [nv3d][nmem][nlev][nij1], fcst2d [nv2d][nmem][nij1] (float32 or
        float64; the analysis has the same dtype).  uniforms: LPF/LPFGM
        resampling uniforms [P][nmonte] (SR) or [P][nmonte][nmem] (MR).
        With check=True the stream is synchronised and a latched device error
        raises SBLETKFError."""
        if self.nobs is None:
            raise RuntimeError("prepare_obs() must be called first")
        p = params or self.params
        cp = self._params(params)
        st_dtype = fcst3d.dtype
        if st_dtype not in (torch.float32, torch.float64):
            raise TypeError("state must be float32 or float64")
        f3 = _dev(fcst3d, st_dtype, self.device, "fcst3d")
        f2 = _dev(fcst2d, st_dtype, self.device, "fcst2d")
        if tuple(f3.shape) != (p.nv3d, p.nmem, p.nlev, self.nij1):
            raise ValueError(f"fcst3d shape {tuple(f3.shape)} != {(p.nv3d, p.nmem, p.nlev, self.nij1)}")
        if tuple(f2.shape) != (p.nv2d, p.nmem, self.nij1):
            raise ValueError(f"fcst2d shape {tuple(f2.shape)} != {(p.nv2d, p.nmem, self.nij1)}")
        a3 = anal3d if anal3d is not None else torch.empty_like(f3)
        a2 = anal2d if anal2d is not None else torch.empty_like(f2)
        uni = None
        if p.iswitch_da != 1:
            if uniforms is None:
                raise ValueError("LPF / LPFGM need resampling uniforms")
            uni = _dev(uniforms, torch.float64, self.device, "uniforms")
            P = p.nlev * self.nij1
            want = P * p.nmonte * (1 if p.rm == 0 else p.nmem)
            if uni.numel() != want:
                raise ValueError(f"uniforms must have {want} values")
        g, cg = self._grid(grid)
        code = self.lib.sbletkf_analysis(self._ws, ctypes.byref(cp), ctypes.byref(cg), _ptr(f3), _ptr(f2), _ptr(a3),
                                         _ptr(a2), F64 if st_dtype == torch.float64 else F32, _ptr(uni),
                                         _ptr(resample_src), _ptr(point_status), _stream_ptr(stream))
        _abi.check(code, "analysis")
        if check:
            self.raise_status(stream)
        return a3, a2

    def backward(self, grid: dict, fcst3d: torch.Tensor, fcst2d: torch.Tensor, grad_anal3d: torch.Tensor,
                 grad_anal2d: torch.Tensor, params: LETKFParams | None = None, stream=None, check: bool = True):
        """Vector-Jacobian product of ``da_main`` (LETKF) for the observations
        of the last ``prepare_obs``: returns FP64 (dJ/d dep [nobs], dJ/d rdiag
        [nobs], dJ/d cov_infl_mul, dJ/d sigma_obs) in the caller's obs order,
        with dist_zero held at its value in ``params``."""
        if self.nobs is None:
            raise RuntimeError("prepare_obs() must be called first")
        p = params or self.params
        cp = self._params(params)
        st_dtype = fcst3d.dtype
        if st_dtype not in (torch.float32, torch.float64):
            raise TypeError("state must be float32 or float64")
        f3 = _dev(fcst3d, st_dtype, self.device, "fcst3d")
        f2 = _dev(fcst2d, st_dtype, self.device, "fcst2d")
        g3 = _dev(grad_anal3d, st_dtype, self.device, "grad_anal3d")
        g2 = _dev(grad_anal2d, st_dtype, self.device, "grad_anal2d")
        if tuple(f3.shape) != (p.nv3d, p.nmem, p.nlev, self.nij1) or g3.shape != f3.shape:
            raise ValueError("fcst3d / grad_anal3d must be [nv3d][nmem][nlev][nij1]")
        if tuple(f2.shape) != (p.nv2d, p.nmem, self.nij1) or g2.shape != f2.shape:
            raise ValueError("fcst2d / grad_anal2d must be [nv2d][nmem][nij1]")
        gdep = torch.zeros(max(self.nobs, 1), dtype=torch.float64, device=self.device)
        grd = torch.zeros_like(gdep)
        gsc = torch.zeros(2, dtype=torch.float64, device=self.device)
        g, cg = self._grid(grid)
        code = self.lib.sbletkf_backward(self._ws, ctypes.byref(cp), ctypes.byref(cg), _ptr(f3), _ptr(f2),
                                         F64 if st_dtype == torch.float64 else F32, _ptr(g3), _ptr(g2),
                                         _ptr(gdep), _ptr(grd), _ptr(gsc), gsc.data_ptr() + 8,
                                         _stream_ptr(stream))
        _abi.check(code, "backward")
        if check:
            self.raise_status(stream)
        return gdep[: self.nobs], grd[: self.nobs], gsc[0], gsc[1]

    def count_nobsl(self, grid: dict, params: LETKFParams | None = None, stream=None) -> torch.Tensor:
        """nobsl of every point as [nlev][nij1] int32 (common_da.f90:133-205)."""
        g, cg = self._grid(grid)
        out = torch.empty(self.params.nlev, self.nij1, dtype=torch.int32, device=self.device)
        cp = self._params(params)
        _abi.check(self.lib.sbletkf_count_nobsl(self._ws, ctypes.byref(cp), ctypes.byref(cg), _ptr(out),
                                                _stream_ptr(stream)), "count_nobsl")
        self.raise_status(stream)
        return out

    def status(self, stream=None) -> int:
        """Synchronise the stream; return and clear the latched device status."""
        st = ctypes.c_int32(0)
        _abi.check(self.lib.sbletkf_get_status(self._ws, _stream_ptr(stream), ctypes.byref(st)), "get_status")
        return int(st.value)

    def latch_status(self, bits: int, stream=None) -> None:
        """OR `bits` into the latched device status (failure injection on the
        host, for tests of the error paths)."""
        _abi.check(self.lib.sbletkf_latch_status(self._ws, int(bits), _stream_ptr(stream)), "latch_status")

    def raise_status(self, stream=None) -> None:
        st = self.status(stream)
        if st:
            raise _abi.SBLETKFError(st, "analysis (device)")


def core_batched(params: LETKFParams, nobsl, hdxf, rdiag, rloc, dep, uniforms=None, resample_src=None,
                 point_status=None, stream=None):
    """letkf_core / lpfgm_core over a ragged batch (common_letkf.f90:61-210,
    common_lpfgm.f90:444-494).  nobsl: int64 [npts] (CUDA); hdxf: concatenated
    Fortran hdxf(nobsl,nmem) blocks (float64); rdiag/rloc/dep [sum nobsl].
    Returns (wvec [npts][nmem], wmat [npts][nmem][nmem] with W(i,j) at [q][j][i])."""
    params.validate()
    lib = _abi.load()
    dev = nobsl.device
    npts = int(nobsl.numel())
    off = torch.zeros(npts + 1, dtype=torch.int64, device=dev)
    off[1:] = torch.cumsum(nobsl.to(torch.int64), 0)
    h = _dev(hdxf, torch.float64, dev, "hdxf")
    rd = _dev(rdiag, torch.float64, dev, "rdiag")
    rl = _dev(rloc, torch.float64, dev, "rloc")
    dp = _dev(dep, torch.float64, dev, "dep")
    k = params.nmem
    wvec = torch.empty(npts, k, dtype=torch.float64, device=dev)
    wmat = torch.empty(npts, k, k, dtype=torch.float64, device=dev)
    uni = None if uniforms is None else _dev(uniforms, torch.float64, dev, "uniforms")
    cp = params.to_c()
    _abi.check(lib.sbletkf_core_batched(ctypes.byref(cp), npts, _ptr(off), _ptr(h), _ptr(rd), _ptr(rl), _ptr(dp),
                                        _ptr(wvec), _ptr(wmat), _ptr(uni), _ptr(resample_src), _ptr(point_status),
                                        _stream_ptr(stream)), "core_batched")
    torch.cuda.current_stream().synchronize() if stream is None else stream.synchronize()
    return wvec, wmat


def ensemble_mean_spread(params: LETKFParams, state3d: torch.Tensor, state2d: torch.Tensor, stream=None):
    """Ensemble mean and spread of a state (ensemble_mesp, common.f90:505-596):
    [nv3d][nmem][nlev][nij1] -> mean, spread [nv3d][nlev][nij1] and
    [nv2d][nmem][nij1] -> [nv2d][nij1], in the state's dtype."""
    lib = _abi.load()
    s3, s2 = state3d.contiguous(), state2d.contiguous()
    if s3.dtype not in (torch.float32, torch.float64) or s2.dtype != s3.dtype:
        raise TypeError("state must be float32 or float64, both parts alike")
    nv3d, k, nlev, nij1 = s3.shape
    if (nv3d, k, nlev) != (params.nv3d, params.nmem, params.nlev) or tuple(s2.shape) != (params.nv2d, k, nij1):
        raise ValueError("state shapes do not match the parameters")
    m3 = torch.empty(nv3d, nlev, nij1, dtype=s3.dtype, device=s3.device)
    d3 = torch.empty_like(m3)
    m2 = torch.empty(params.nv2d, nij1, dtype=s2.dtype, device=s2.device)
    d2 = torch.empty_like(m2)
    cp = params.to_c()
    _abi.check(lib.sbletkf_ensemble_mean_spread(ctypes.byref(cp), nij1, _ptr(s3), _ptr(s2),
                                                F64 if s3.dtype == torch.float64 else F32, _ptr(m3), _ptr(d3),
                                                _ptr(m2), _ptr(d2), _stream_ptr(stream)), "ensemble_mean_spread")
    return m3, d3, m2, d2
