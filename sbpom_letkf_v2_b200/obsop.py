"""Observation-space preprocessing on the GPU (the step before the analysis).

``obs_operator`` is set_obs (letkf/run/src/common_obs.f90:24-265, 380-399):
H(x) of every member by Trans_XtoY (common.f90:391-500), the ensemble mean
and spread in observation space, dYf = H(x_m) - mean, the innovation, the
optional gross-error check and AOEI, through ``sbletkf_obs_operator``.
``analysis_obs`` keeps the qc = 1 observations in the form
``Analysis.prepare_obs`` takes (the "Remove undef" step,
common_obs.f90:238-258).  ``monit_dep`` turns the per-variable sums into the
bias / RMSD table of monit_dep (common.f90:602-675).
"""
from __future__ import annotations

import ctypes

import torch

from . import _abi
from .params import F32, F64, LETKFParams

GROSS_QC, AOEI = 1, 2


def _stream_ptr(stream) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def obs_operator(params: LETKFParams, grid: dict, fcst3d: torch.Tensor, fcst2d: torch.Tensor, obs: dict,
                 gross_qc: bool = False, aoei: bool = True, stats: bool = False, stream=None) -> dict:
    """grid: global lon, lat, fsm [nlat*nlon] and depth [nlev][nlat*nlon]
    (FP64, CUDA); fcst3d [nv3d][nmem][nlev][nlat*nlon], fcst2d
    [nv2d][nmem][nlat*nlon]; obs: elm (int32), lon, lat, lev, dat, err
    [nobs].  Returns device tensors idx, idy, qc, hxmean, hxsprd, dep, err,
    hdxf [nmem][nobs] (NaN where undef) and, with stats=True, the
    [(nv3d+nv2d)][3] sums (count, sum dep, sum dep^2)."""
    params.validate()
    lib = _abi.load()
    dev = fcst3d.device
    f64 = lambda t: t.to(dev, torch.float64).contiguous()
    g = {k: f64(grid[k]) for k in ("lon", "lat", "fsm", "depth")}
    o = {k: f64(obs[k]) for k in ("lon", "lat", "lev", "dat", "err")}
    o["elm"] = obs["elm"].to(dev, torch.int32).contiguous()
    nobs = int(o["elm"].numel())
    k = params.nmem
    out = dict(idx=torch.empty(nobs, dtype=torch.int32, device=dev),
               idy=torch.empty(nobs, dtype=torch.int32, device=dev),
               qc=torch.empty(nobs, dtype=torch.int32, device=dev),
               hxmean=torch.empty(nobs, dtype=torch.float64, device=dev),
               hxsprd=torch.empty(nobs, dtype=torch.float64, device=dev),
               dep=torch.empty(nobs, dtype=torch.float64, device=dev),
               err=torch.empty(nobs, dtype=torch.float64, device=dev),
               hdxf=torch.empty(k, nobs, dtype=torch.float64, device=dev))
    st = torch.zeros(params.nv3d + params.nv2d, 3, dtype=torch.float64, device=dev) if stats else None
    f3, f2 = fcst3d.contiguous(), fcst2d.contiguous()
    if f2.dtype != f3.dtype:
        raise TypeError("fcst3d and fcst2d must have the same dtype")
    cin = _abi.CObsIn(nobs=nobs, reserved=0, **{kk: o[kk].data_ptr() for kk in ("elm", "lon", "lat", "lev", "dat",
                                                                               "err")})
    cout = _abi.CObsOut(**{kk: v.data_ptr() for kk, v in out.items()})
    cp = params.to_c()
    flags = (GROSS_QC if gross_qc else 0) | (AOEI if aoei else 0)
    _abi.check(lib.sbletkf_obs_operator(ctypes.byref(cp), g["lon"].data_ptr(), g["lat"].data_ptr(),
                                        g["fsm"].data_ptr(), g["depth"].data_ptr(), f3.data_ptr(), f2.data_ptr(),
                                        F64 if f3.dtype == torch.float64 else F32, ctypes.byref(cin), flags,
                                        ctypes.byref(cout), 0 if st is None else st.data_ptr(),
                                        _stream_ptr(stream)), "obs_operator")
    if st is not None:
        out["stats"] = st
    out["_inputs"] = (o, g)
    return out


def analysis_obs(obs: dict, res: dict, hdxf_dtype=torch.float32) -> dict:
    """The qc = 1 observations as Analysis.prepare_obs inputs (elm idx idy lon
    lat lev err dep hdxf), in input order."""
    keep = res["qc"] == 1
    o = res["_inputs"][0]
    return dict(elm=o["elm"][keep], idx=res["idx"][keep], idy=res["idy"][keep], lon=o["lon"][keep],
                lat=o["lat"][keep], lev=o["lev"][keep], err=res["err"][keep], dep=res["dep"][keep],
                hdxf=res["hdxf"][:, keep].to(hdxf_dtype).contiguous())


def monit_dep(stats: torch.Tensor) -> dict:
    """bias, rmsd and count of the innovations per variable (NaN where none)."""
    s = stats.double().cpu()
    n = s[:, 0]
    bias = torch.where(n > 0, s[:, 1] / n.clamp_min(1), torch.full_like(n, float("nan")))
    rmsd = torch.where(n > 0, torch.sqrt(s[:, 2] / n.clamp_min(1)), torch.full_like(n, float("nan")))
    return dict(bias=bias, rmsd=rmsd, n=n.long())


MONIT_DEPARTURE, MONIT_VALUE = 0, 1
CATEGORIES = ("all", "surface", "interior")


def hx_of_field(params: LETKFParams, grid: dict, field3d: torch.Tensor, field2d: torch.Tensor, obs: dict,
                stream=None) -> torch.Tensor:
    """Trans_XtoY of one state field (common.f90:391-500): field3d
    [nv3d][nlev][nlat*nlon], field2d [nv2d][nlat*nlon] -> H(field) [nobs]
    (FP64, NaN where undef).  This is how write_ens_mpi takes the ensemble
    mean and spread fields to observation space (common_io.f90:967-985).  The
    field runs through sbletkf_obs_operator as a two-member ensemble of
    identical members, whose mean (h + h) / 2 is h exactly."""
    f3 = torch.stack([field3d, field3d], dim=1).contiguous()
    f2 = torch.stack([field2d, field2d], dim=1).contiguous()
    p = params.replace(nmem=2)
    res = obs_operator(p, grid, f3, f2, obs, gross_qc=False, aoei=False, stream=stream)
    return res["hxmean"]


def obs_monitor(params: LETKFParams, obs: dict, hx: torch.Tensor, mode: int, stream=None) -> torch.Tensor:
    """The sums of sbletkf_obs_monitor: [(nv3d+nv2d)][all, surface,
    interior][count, sum, sum of squares] (FP64, device) of dat - hx
    (MONIT_DEPARTURE) or hx (MONIT_VALUE) over the observations whose hx is
    defined."""
    lib = _abi.load()
    dev = hx.device
    elm = obs["elm"].to(dev, torch.int32).contiguous()
    lev = obs["lev"].to(dev, torch.float64).contiguous()
    dat = obs["dat"].to(dev, torch.float64).contiguous() if mode == MONIT_DEPARTURE else None
    h = hx.to(torch.float64).contiguous()
    nv = params.nv3d + params.nv2d
    st = torch.zeros(nv, 3, 3, dtype=torch.float64, device=dev)
    cp = params.to_c()
    _abi.check(lib.sbletkf_obs_monitor(ctypes.byref(cp), int(elm.numel()), elm.data_ptr(), lev.data_ptr(),
                                       0 if dat is None else dat.data_ptr(), h.data_ptr(), int(mode),
                                       st.data_ptr(), _stream_ptr(stream)), "obs_monitor")
    return st


def _finish(st: torch.Tensor, params: LETKFParams, rms: bool) -> dict:
    s = st.double().cpu()
    n = s[..., 0]
    nan = torch.full_like(n, float("nan"))
    mean = torch.where(n > 0, s[..., 1] / n.clamp_min(1), nan)
    out = dict(n=n.long(), mean=mean)   # the 2D variables count no surface / interior
    if rms:
        out["rms"] = torch.where(n > 0, torch.sqrt(s[..., 2] / n.clamp_min(1)), nan)
    return out


def monit_mean(params: LETKFParams, obs: dict, hx: torch.Tensor, stream=None) -> dict:
    """monit_mean (common.f90:681-840): bias and RMSD of dat - hx per variable
    and category (columns of CATEGORIES), NaN (the reference's undef) where
    no observation counted, and the counts."""
    r = _finish(obs_monitor(params, obs, hx, MONIT_DEPARTURE, stream), params, rms=True)
    return dict(bias=r["mean"], rmsd=r["rms"], n=r["n"])


def monit_sprd(params: LETKFParams, obs: dict, hx: torch.Tensor, stream=None) -> dict:
    """monit_sprd (common.f90:846-978): the mean of hx (an ensemble spread in
    observation space) per variable and category, and the counts."""
    r = _finish(obs_monitor(params, obs, hx, MONIT_VALUE, stream), params, rms=False)
    return dict(spread=r["mean"], n=r["n"])


def write_ens_monitors(params: LETKFParams, grid: dict, obs: dict, fcst3d: torch.Tensor, fcst2d: torch.Tensor,
                       anal3d: torch.Tensor, anal2d: torch.Tensor, stream=None) -> dict:
    """The observation-space monitors write_ens_mpi prints after the analysis
    (common_io.f90:917-1045): ensemble mean and spread of the forecast and of
    the analysis (ensemble_mesp), each taken to observation space by
    Trans_XtoY, then monit_mean on the means (O-B and O-A departures) and
    monit_sprd on the spreads.  grid and obs as for obs_operator; states
    [nv3d][nmem][nlev][nlat*nlon] / [nv2d][nmem][nlat*nlon]."""
    from .analysis import ensemble_mean_spread
    out = {}
    for name, s3, s2 in (("fcst", fcst3d, fcst2d), ("anal", anal3d, anal2d)):
        m3, d3, m2, d2 = ensemble_mean_spread(params, s3, s2, stream)
        hxm = hx_of_field(params, grid, m3, m2, obs, stream)
        hxs = hx_of_field(params, grid, d3, d2, obs, stream)
        out[name] = dict(hxmean=hxm, hxsprd=hxs, mean=monit_mean(params, obs, hxm, stream),
                         sprd=monit_sprd(params, obs, hxs, stream))
    return out
