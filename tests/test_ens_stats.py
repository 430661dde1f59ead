"""Ensemble mean and spread of the state (sbletkf_ensemble_mean_spread)
against the two-pass restatement of ensemble_mesp (common.f90:505-596) in
oracle/letkf_oracle.py: FP64 within 1e-12 relative, FP32 state within FP32
rounding."""
import numpy as np
import pytest
import torch

from oracle import letkf_oracle as O
from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case

pytestmark = pytest.mark.gpu


def _ref(x):
    """x [nv][k][...] -> mean, spread [nv][...] by the oracle's two-pass form."""
    nv, k = x.shape[:2]
    flat = x.reshape(nv, k, -1)
    m = np.empty((nv, flat.shape[2]))
    s = np.empty_like(m)
    for v in range(nv):
        m[v], s[v], _ = O.mean_spread_pert(flat[v])
    return m.reshape((nv,) + x.shape[2:]), s.reshape((nv,) + x.shape[2:])


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 2e-6)])
def test_ensemble_mean_spread(dtype, tol, cuda):
    from sbpom_letkf_v2_b200.analysis import ensemble_mean_spread
    wl = WORKLOADS[0].scaled(nlon=20, nlat=16, nlev=5, nmem=33, n_sst=10, n_ssh=5, n_prof=1, seed=4)
    case = make_case(wl)
    f3, f2 = case.fcst3d.to("cuda:0", dtype), case.fcst2d.to("cuda:0", dtype)
    m3, d3, m2, d2 = ensemble_mean_spread(case.params, f3, f2)
    r3m, r3s = _ref(f3.double().cpu().numpy())
    r2m, r2s = _ref(f2.double().cpu().numpy())
    for got, want in ((m3, r3m), (d3, r3s), (m2, r2m), (d2, r2s)):
        g = got.double().cpu().numpy()
        assert np.abs(g - want).max() <= tol * np.abs(want).max()
