"""Autotuner (sbpom_letkf_v2_b200/tune.py): candidate set, column sampling,
the JSON cache, and on a GPU a real tuning run whose choice reproduces the
analysis of the default configuration."""
import json

import numpy as np
import pytest
import torch

from sbpom_letkf_v2_b200 import tune
from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case


def _case(precision=1):
    wl = WORKLOADS[0].scaled(nlon=20, nlat=16, nlev=5, nmem=24, n_sst=300, n_ssh=60, n_prof=4, seed=21)
    case = make_case(wl, cov_infl_mul=1.1)
    return case, case.params.replace(precision=precision)


def test_candidates_and_key():
    case, p = _case(1)
    c = tune.candidates(p)
    assert len(c) == 3 * len(tune.TC_CANDIDATES)          # pipeline, columns, point x tc routing
    assert len(tune.candidates(p.replace(precision=0))) == 3
    assert len(tune.candidates(p.replace(nmem=120))) == 2 * len(tune.TC_CANDIDATES)   # no pipeline above 112
    assert len(tune.candidates(p.replace(iswitch_da=2, precision=0))) == 2
    assert tune.key(p, "B200") != tune.key(p.replace(nmem=32), "B200")


def test_column_sample_keeps_whole_columns():
    case, p = _case()
    uni = torch.rand(p.nlev * case.nij1, 3)
    g, f3, f2, u = tune.column_sample(case.grid, case.fcst3d, case.fcst2d, uni, p.nlev, 50)
    n = g["lon1"].numel()
    assert n <= 50 and g["depth1"].shape == (p.nlev, n) and f3.shape[-1] == n and f2.shape[-1] == n
    stride = case.nij1 // 50
    assert torch.equal(g["lon1"], case.grid["lon1"][::stride][:n])
    assert torch.equal(u.view(p.nlev, n, 3), uni.view(p.nlev, case.nij1, 3)[:, ::stride][:, :n])


def test_cache_round_trip_and_fastest_choice(tmp_path):
    case, p = _case()
    calls = []

    def fake(params, g, f3, f2, obs, uni, cand, reps):
        calls.append(cand)
        if cand["tc_max_cand"] == 3072.0:
            return None                                  # as if it had raised a status
        return 10.0 + cand["schedule"] + cand["tc_max_cand"] / 1e4
    path = str(tmp_path / "tune.json")
    r = tune.tune(p, case.grid, case.fcst3d, case.fcst2d, case.obs, cache=path, gpu_name="X", measure=fake)
    assert r["schedule"] == 0 and r["tc_max_cand"] == 0.0
    assert len(r["ms"]) == len(calls) - 3                # the failing candidates are dropped
    assert r["ms_width"] == {}                           # one CTA per point: no queue items to size
    n = len(calls)
    r2 = tune.tune(p, case.grid, case.fcst3d, case.fcst2d, case.obs, cache=path, gpu_name="X", measure=fake)
    assert len(calls) == n and r2 == r                   # served from the cache
    assert tune.key(p, "X") in json.load(open(path))


@pytest.mark.gpu
def test_gpu_tuning_choice_reproduces_the_analysis(tmp_path, cuda):
    from sbpom_letkf_v2_b200.analysis import Analysis
    case, p = _case(1)
    c = case.to("cuda:0")
    cfg = tune.tune(p, c.grid, c.fcst3d, c.fcst2d, c.obs, cache=str(tmp_path / "t.json"))
    assert cfg["schedule"] in (0, 1, 2) and len(cfg["ms"]) >= 1
    outs = []
    for use in (None, cfg):
        an = Analysis(p, c.nij1, c.obs["elm"].numel(), device="cuda:0")
        pp = tune.apply(an, p, use) if use else p
        an.prepare_obs(c.obs)
        a3, _ = an.da_main(c.grid, c.fcst3d, c.fcst2d, params=pp)
        outs.append(a3.double().cpu().numpy())
        an.close()
    m0, m1 = outs[0].mean(axis=1), outs[1].mean(axis=1)
    assert np.abs(m1 - m0).max() <= 1e-4 * np.abs(m0).max()


def test_item_width_stage_and_row_sample():
    """When a queue schedule wins, stage 2 times the item widths on whole
    latitude rows and keeps the fastest."""
    case, p = _case()
    calls = []

    def fake(params, g, f3, f2, obs, uni, cand, reps):
        calls.append((cand, g["lon1"].numel()))
        if "item_width" in cand:
            return 5.0 + abs(cand["item_width"] - 2)        # width 2 is fastest
        return 10.0 - cand["schedule"] + cand["tc_max_cand"] / 1e4   # the pipeline (2) wins
    r = tune.tune(p, case.grid, case.fcst3d, case.fcst2d, case.obs, cache=None, gpu_name="X", measure=fake)
    assert r["schedule"] == 2 and r["item_width"] == 2 and set(r["ms_width"]) == {str(w) for w in tune.WIDTHS}
    g, f3, f2, _ = tune.row_sample(case.grid, case.fcst3d, case.fcst2d, None, p.nlev, p.nlon, 3 * p.nlon + 5)
    n = g["lon1"].numel()
    assert n == 3 * p.nlon and f3.shape[-1] == n and g["depth1"].shape == (p.nlev, n)
    assert torch.equal(g["rj1"].view(3, p.nlon)[:, 0].diff(), torch.ones(2, dtype=g["rj1"].dtype))
    assert all(w == case.nij1 for c, w in calls if "item_width" in c)   # a small grid: every row
