"""One analysis cycle (sbletkf_prepare_obs + sbletkf_analysis) captured in a
CUDA graph: the entry points make no host synchronisation and no allocation,
so a replay equals an eager call, also after the inputs change in place."""
import pytest
import torch

from sbpom_letkf_v2_b200.analysis import Analysis
from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_cycle_graph_replay_matches_eager(precision, cuda):
    wl = WORKLOADS[0].scaled(nlon=24, nlat=18, nlev=6, nmem=40, n_sst=600, n_ssh=200, n_prof=6, seed=77)
    case = make_case(wl, device="cuda:0", cov_infl_mul=1.1, alpha_rtpp=0.3)
    p = case.params.replace(precision=precision)
    an = Analysis(p, case.nij1, case.obs["elm"].numel(), device="cuda:0")
    obs = {k: v.clone() for k, v in case.obs.items()}
    f3, f2 = case.fcst3d.clone(), case.fcst2d.clone()
    a3 = torch.empty_like(f3)
    a2 = torch.empty_like(f2)

    def cycle():
        an.prepare_obs(obs)
        an.da_main(case.grid, f3, f2, anal3d=a3, anal2d=a2, check=False)

    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        cycle()                      # warm-up outside capture (kernel attributes, module load)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        cycle()
    for trial in range(2):
        if trial == 1:               # new departures and forecast, same buffers
            obs["dep"].mul_(0.5).add_(0.01)
            f3.add_(0.001)
        g.replay()
        torch.cuda.synchronize()
        assert an.status() == 0
        r3, r2 = a3.clone(), a2.clone()
        an.prepare_obs(obs)
        e3, e2 = an.da_main(case.grid, f3, f2)
        assert torch.equal(r3, e3) and torch.equal(r2, e2)
    del g
    an.close()
