"""sbletkf_analysis_noalloc, the allocation-free entry point, against the
workspace entry point sbletkf_analysis (both through the C ABI).

The entry point exists for callers that cannot allocate device memory where
they run the analysis (a host model whose memory pool owns the device, where
cudaMalloc would synchronise or fail); it keeps all scratch in a fixed array of
the library.  Two calls in a row with different inputs check that the reused
array carries nothing over from the previous call.  Collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from sbpom_letkf_v2_b200 import _abi
from sbpom_letkf_v2_b200.analysis import GRID_KEYS, OBS_KEYS, Analysis
from sbpom_letkf_v2_b200.params import F32, F64
from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case
from tests._util import field_relerr

pytestmark = pytest.mark.gpu
TOL64 = 1e-10


def _noalloc(case, dev, dtype=torch.float64):
    lib = _abi.load()
    p = case.params
    g = {k: case.grid[k].to(dev, torch.float64).contiguous() for k in GRID_KEYS}
    o = {k: case.obs[k].to(dev).contiguous() for k in OBS_KEYS}
    f3 = case.fcst3d.to(dev, dtype).contiguous()
    f2 = case.fcst2d.to(dev, dtype).contiguous()
    a3 = torch.full_like(f3, float("nan"))
    a2 = torch.full_like(f2, float("nan"))
    pst = torch.full((p.nlev * case.nij1,), -1, dtype=torch.int32, device=dev)
    cg = _abi.CGrid(nij1=case.nij1, reserved=0, **{k: g[k].data_ptr() for k in GRID_KEYS})
    co = _abi.CObs(nobs=o["elm"].numel(), hdxf_dtype=F64 if o["hdxf"].dtype == torch.float64 else F32,
                   **{k: o[k].data_ptr() for k in OBS_KEYS})
    cp = p.to_c()
    code = lib.sbletkf_analysis_noalloc(ctypes.byref(cp), ctypes.byref(cg), ctypes.byref(co), f3.data_ptr(),
                                        f2.data_ptr(), a3.data_ptr(), a2.data_ptr(),
                                        F64 if dtype == torch.float64 else F32, None, pst.data_ptr(),
                                        torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    return code, a3.cpu().numpy(), a2.cpu().numpy(), pst.cpu().numpy()


def _workspace(case, dev, dtype=torch.float64):
    an = Analysis(case.params, case.nij1, case.obs["elm"].numel(), device=dev)
    an.prepare_obs({k: v.to(dev) for k, v in case.obs.items()})
    g = {k: v.to(dev) for k, v in case.grid.items()}
    a3, a2 = an.da_main(g, case.fcst3d.to(dev, dtype), case.fcst2d.to(dev, dtype))
    out = a3.cpu().numpy(), a2.cpu().numpy()
    an.close()
    return out


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


def test_noalloc_rejects_sizes_beyond_its_limits(cuda):
    case = make_case(WORKLOADS[0].scaled(nlon=12, nlat=10, nlev=2, nmem=8, n_sst=40, n_ssh=10, n_prof=1, seed=503))
    big = dict(case.obs)
    n = _abi.NOALLOC_MAX_OBS + 1
    reps = -(-n // big["elm"].numel())
    big = {k: (v.repeat(1, reps)[:, :n] if v.dim() == 2 else v.repeat(reps)[:n]) for k, v in big.items()}
    case.obs = big
    code, _, _, _ = _noalloc(case, cuda)
    assert code == _abi.ERR_WORKSPACE
