"""sbletkf_analysis_noalloc, the allocation-free entry point, against the
workspace entry point sbletkf_analysis (both through the C ABI).

The entry point exists for callers that cannot allocate device memory where
they run the analysis (a host model whose memory pool owns the device, where
cudaMalloc would synchronise or fail); it keeps all scratch in a fixed array of
the library.  Two calls in a row with different inputs check that the reused
array carries nothing over from the previous call.  Errors that only the
device sees (an observation outside the grid, a NaN innovation) must reach the
caller through point_status.  Collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from sbpom_letkf_v2_b200 import _abi
from sbpom_letkf_v2_b200.analysis import GRID_KEYS, OBS_KEYS, Analysis
from sbpom_letkf_v2_b200.params import DA_LPF, F32, F64, RM_SR
from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case, pf_uniforms
from tests._util import field_relerr

pytestmark = pytest.mark.gpu
TOL64 = 1e-10
TOL32 = 2e-6     # float32 state: both entry points round the same FP64 analysis to float32


def _noalloc(case, dev, dtype=torch.float64, uniforms=None, obs=None, with_status=True):
    lib = _abi.load()
    p = case.params
    g = {k: case.grid[k].to(dev, torch.float64).contiguous() for k in GRID_KEYS}
    o = {k: v.to(dev).contiguous() for k, v in (obs or case.obs).items()}
    f3 = case.fcst3d.to(dev, dtype).contiguous()
    f2 = case.fcst2d.to(dev, dtype).contiguous()
    a3 = torch.full_like(f3, float("nan"))
    a2 = torch.full_like(f2, float("nan"))
    pst = torch.full((p.nlev * case.nij1,), -1, dtype=torch.int32, device=dev)
    uni = None if uniforms is None else uniforms.to(dev, torch.float64).contiguous()
    cg = _abi.CGrid(nij1=case.nij1, reserved=0, **{k: g[k].data_ptr() for k in GRID_KEYS})
    co = _abi.CObs(nobs=o["elm"].numel(), hdxf_dtype=F64 if o["hdxf"].dtype == torch.float64 else F32,
                   **{k: o[k].data_ptr() for k in OBS_KEYS})
    cp = p.to_c()
    code = lib.sbletkf_analysis_noalloc(ctypes.byref(cp), ctypes.byref(cg), ctypes.byref(co), f3.data_ptr(),
                                        f2.data_ptr(), a3.data_ptr(), a2.data_ptr(),
                                        F64 if dtype == torch.float64 else F32,
                                        None if uni is None else uni.data_ptr(),
                                        pst.data_ptr() if with_status else None,
                                        torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return code, a3.cpu().numpy(), a2.cpu().numpy(), pst.cpu().numpy()


def _workspace(case, dev, dtype=torch.float64, uniforms=None):
    an = Analysis(case.params, case.nij1, max(1, case.obs["elm"].numel()), device=dev)
    an.prepare_obs({k: v.to(dev) for k, v in case.obs.items()})
    g = {k: v.to(dev) for k, v in case.grid.items()}
    uni = None if uniforms is None else uniforms.to(dev)
    a3, a2 = an.da_main(g, case.fcst3d.to(dev, dtype), case.fcst2d.to(dev, dtype), uniforms=uni)
    out = a3.cpu().numpy(), a2.cpu().numpy()
    an.close()
    return out


def _small(seed, **kw):
    wl = WORKLOADS[0].scaled(nlon=16, nlat=12, nlev=3, nmem=16, n_sst=200, n_ssh=60, n_prof=2, seed=seed)
    return make_case(wl, **kw)


def test_noalloc_matches_workspace_entry_on_two_calls_in_a_row(cuda):
    cases = [
        make_case(WORKLOADS[0].scaled(nlon=24, nlat=18, nlev=5, nmem=20, n_sst=600, n_ssh=200, n_prof=6,
                                      seed=501), cov_infl_mul=1.1, alpha_rtpp=0.5),
        make_case(WORKLOADS[0].scaled(nlon=20, nlat=14, nlev=4, nmem=100, n_sst=250, n_ssh=60, n_prof=3,
                                      seed=502), cov_infl_mul=1.05),
    ]
    for case in cases:
        code, a3, a2, pst = _noalloc(case, cuda)
        assert code == _abi.OK
        assert (pst == 0).all()
        r3, r2 = _workspace(case, cuda)
        assert np.isfinite(a3).all() and np.isfinite(a2).all()
        assert field_relerr(a3, r3) <= TOL64
        assert field_relerr(a2, r2) <= TOL64


def test_noalloc_float32_state_and_lpf_with_uniforms(cuda):
    case = _small(504, cov_infl_mul=1.1)
    code, a3, a2, pst = _noalloc(case, cuda, dtype=torch.float32)
    assert code == _abi.OK and (pst == 0).all()
    r3, r2 = _workspace(case, cuda, dtype=torch.float32)
    assert field_relerr(a3, r3) <= TOL32 and field_relerr(a2, r2) <= TOL32

    case = _small(505, iswitch_da=DA_LPF, rm=RM_SR, nmonte=3)
    uni = pf_uniforms(case.params.nlev * case.nij1, 3, case.params.nmem, RM_SR, seed=9)
    code, a3, a2, pst = _noalloc(case, cuda, uniforms=uni)
    assert code == _abi.OK and (pst == 0).all()
    r3, r2 = _workspace(case, cuda, uniforms=uni)
    assert field_relerr(a3, r3) <= TOL64 and field_relerr(a2, r2) <= TOL64


def test_noalloc_without_observations_copies_the_forecast(cuda):
    case = _small(506)
    empty = {k: v[..., :0].contiguous() for k, v in case.obs.items()}
    code, a3, a2, pst = _noalloc(case, cuda, obs=empty)
    assert code == _abi.OK and (pst == 0).all()
    assert np.array_equal(a3, case.fcst3d.double().numpy())
    assert np.array_equal(a2, case.fcst2d.double().numpy())


@pytest.mark.parametrize("what", ["cell", "dep_nan"])
def test_noalloc_reports_observation_errors_in_point_status(what, cuda):
    case = _small(507)
    obs = {k: v.clone() for k, v in case.obs.items()}
    if what == "cell":
        obs["idx"][5] = case.params.nlon          # a cell outside [1, nlon-1]
        want = _abi.ERR_OBS_CELL
    else:
        obs["dep"][5] = float("nan")
        want = _abi.ERR_NONFINITE
    code, _, _, pst = _noalloc(case, cuda, obs=obs)
    assert code == _abi.OK                        # the call itself is asynchronous
    assert ((pst & want) != 0).all()
    code, a3, _, pst = _noalloc(case, cuda)       # the next call starts clean
    assert code == _abi.OK and (pst == 0).all() and np.isfinite(a3).all()


def test_noalloc_rejects_sizes_beyond_its_limits(cuda):
    case = _small(503)
    code, _, _, _ = _noalloc(case, cuda, with_status=False)
    assert code == _abi.ERR_ARG                   # point_status is required
    big = dict(case.obs)
    n = _abi.NOALLOC_MAX_OBS + 1
    reps = -(-n // big["elm"].numel())
    big = {k: (v.repeat(1, reps)[:, :n] if v.dim() == 2 else v.repeat(reps)[:n]) for k, v in big.items()}
    code, _, _, _ = _noalloc(case, cuda, obs=big)
    assert code == _abi.ERR_WORKSPACE
    wide = WORKLOADS[0].scaled(nlon=300, nlat=220, nlev=2, nmem=8, n_sst=50, n_ssh=0, n_prof=1, seed=508)
    assert wide.nlon * wide.nlat > _abi.NOALLOC_MAX_CELLS
    code, _, _, _ = _noalloc(make_case(wide), cuda)
    assert code == _abi.ERR_WORKSPACE
