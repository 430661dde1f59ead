"""Failure detection without a GPU fault: bad inputs and exhausted limits
become status bits (the reference STOPs, letkf/run/src/common.f90:1019-1038,
common_da.f90:196-201), never a trap, and the context stays usable."""
import numpy as np
import pytest
import torch

from sbpom_letkf_v2_b200._abi import ERR_EIG_NOCONV, ERR_NONFINITE, ERR_WORKSPACE, SBLETKFError
from sbpom_letkf_v2_b200.analysis import Analysis
from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case

pytestmark = pytest.mark.gpu


def _case(k=40):
    wl = WORKLOADS[0].scaled(nlon=16, nlat=12, nlev=4, nmem=k, n_sst=400, n_ssh=100, n_prof=4, seed=61)
    return make_case(wl, device="cuda:0", cov_infl_mul=1.1)


def _run(case, obs, params=None):
    p = params or case.params
    an = Analysis(p, case.nij1, max(1, obs["elm"].numel()), device="cuda:0")
    try:
        an.prepare_obs(obs)
        return an.da_main(case.grid, case.fcst3d, case.fcst2d, params=p)
    finally:
        an.close()


@pytest.mark.parametrize("what", ["dep_nan", "err_zero", "hdxf_inf"])
def test_bad_observation_values_raise_nonfinite(what, cuda):
    case = _case()
    obs = {k: v.clone() for k, v in case.obs.items()}
    if what == "dep_nan":
        obs["dep"][7] = float("nan")
    elif what == "err_zero":
        obs["err"][3] = 0.0
    else:
        obs["hdxf"][2, 11] = float("inf")
    with pytest.raises(SBLETKFError) as ei:
        _run(case, obs)
    assert ei.value.code & ERR_NONFINITE
    a3, _ = _run(case, case.obs)          # the context is still usable
    assert torch.isfinite(a3).all()


def test_sweep_cap_reports_no_convergence(cuda):
    case = _case()
    with pytest.raises(SBLETKFError) as ei:
        _run(case, case.obs, case.params.replace(max_sweeps=1))
    assert ei.value.code & ERR_EIG_NOCONV


def test_workspace_capacity_and_shapes_checked_on_host(cuda):
    case = _case()
    an = Analysis(case.params, case.nij1, 10, device="cuda:0")
    with pytest.raises(SBLETKFError) as ei:
        an.prepare_obs(case.obs)          # 500+ obs > max_nobs = 10
    assert ei.value.code == ERR_WORKSPACE
    small = {k: v[..., :10].contiguous() for k, v in case.obs.items()}
    an.prepare_obs(small)
    with pytest.raises(ValueError):
        an.da_main(case.grid, case.fcst3d[:, :, :2].contiguous(), case.fcst2d)
    an.close()


def test_point_status_marks_the_failing_points(cuda):
    case = _case()
    p = case.params.replace(max_sweeps=1)
    an = Analysis(p, case.nij1, case.obs["elm"].numel(), device="cuda:0")
    an.prepare_obs(case.obs)
    st = torch.zeros(p.nlev * case.nij1, dtype=torch.int32, device="cuda:0")
    an.da_main(case.grid, case.fcst3d, case.fcst2d, point_status=st, check=False)
    code = an.status()
    nobsl = an.count_nobsl(case.grid).reshape(-1)
    bad = (st & ERR_EIG_NOCONV) != 0
    assert code & ERR_EIG_NOCONV and bool(bad.any())
    assert bool((nobsl[bad] > 0).all())   # only points with observations run the eigensolve
    an.close()


@pytest.mark.parametrize("schedule", [Analysis.SCHED_PIPELINE, Analysis.SCHED_COLUMNS, Analysis.SCHED_POINT])
def test_prelatched_timeout_aborts_mixed_launch_and_context_stays_usable(schedule, cuda):
    """The path every tensor-core launch takes once a bounded wait has expired
    somewhere: with SBLETKF_ERR_TIMEOUT latched on the host before the launch,
    no CTA allocates tensor memory or issues a UMMA, every point is marked,
    the call reports the status, and the next call runs normally."""
    from sbpom_letkf_v2_b200._abi import ERR_TIMEOUT
    case = _case()
    p = case.params.replace(precision=1)
    P = p.nlev * case.nij1
    an = Analysis(p, case.nij1, case.obs["elm"].numel(), device="cuda:0")
    an.set_schedule(schedule)
    an.prepare_obs(case.obs)
    st = torch.zeros(P, dtype=torch.int32, device="cuda:0")
    an.latch_status(ERR_TIMEOUT)
    an.da_main(case.grid, case.fcst3d, case.fcst2d, point_status=st, check=False)
    assert an.status() & ERR_TIMEOUT
    assert bool(((st & ERR_TIMEOUT) != 0).all())
    st.zero_()
    a3, a2 = an.da_main(case.grid, case.fcst3d, case.fcst2d, point_status=st)   # raises on any status
    assert torch.isfinite(a3).all() and torch.isfinite(a2).all()
    assert bool((st == 0).all())
    an.close()
