"""Shape checks of the seeded workloads at full size (GPU generation)."""
import numpy as np
import pytest

from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case

pytestmark = pytest.mark.gpu


def test_uneven_workload_nobsl_histogram(cuda):
    """Workload 2 (400x300x40, k=64, 300k obs with 180k HF-radar obs in three
    100 km patches): local observation counts range from 0 to beyond 4,000,
    with points below 1,000, between 1,000 and 4,000 and above 4,000 (the
    dense SST field leaves no surface point with fewer than ~100)."""
    from sbpom_letkf_v2_b200.analysis import Analysis
    case = make_case(WORKLOADS[2], device="cuda:0")
    an = Analysis(case.params, case.nij1, case.obs["elm"].numel(), device="cuda:0")
    an.prepare_obs(case.obs)
    n = an.count_nobsl(case.grid).cpu().numpy().ravel()
    an.close()
    h = np.histogram(n, bins=[0, 1, 1000, 4000, 10 ** 7])[0]
    assert n.min() == 0 and n.max() > 4000
    assert all(c > 0 for c in h), h
    assert (n == 0).mean() > 0.3          # deep levels see no observation
