"""Observation-space preprocessing (sbletkf_obs_operator) against the CPU
restatement oracle/obsop_oracle.py (set_obs / Trans_XtoY / akima_spline).

Tolerances: qc, idx, idy exactly equal; H(x) mean, spread, hdxf, dep, err
within 1e-12 relative (FP64 both sides, different summation order)."""
import numpy as np
import pytest
import torch

from oracle import obsop_oracle as OO
from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case

TOL = 1e-12


# ---- the restatement on known answers ---------------------------------------

def test_akima_zero_weight_rule_and_bilinear_planes():
    """On data with equal slopes both Akima weights vanish and the reference
    sets t = 0 (common.f90:348-354), so the interval's value is the
    zero-end-slope Hermite cubic y0 + (y1 - y0)(3u^2 - 2u^3); grid points are
    reproduced exactly; bilinear interpolation reproduces bilinear functions."""
    x = np.array([-900.0, -500.0, -300.0, -120.0, -60.0, -20.0, 0.0])
    y = 0.37 * x + 5.0
    for x5 in (-700.0, -301.0, -100.0, -1e-3):
        i = int(np.searchsorted(x, x5, side="right"))           # x[i-1] <= x5 < x[i]
        u = (x5 - x[i - 1]) / (x[i] - x[i - 1])
        want = y[i - 1] + (y[i] - y[i - 1]) * (3 * u * u - 2 * u ** 3)
        assert abs(OO.akima(x, y, x5) - want) <= 1e-12 * 400
    for j in range(len(x)):
        assert OO.akima(x, y, x[j]) == y[j]
    assert OO.akima(x, y, 1.0) is None and OO.akima(x, y, -901.0) is None
    f = lambda a, b: 2.0 + 0.5 * a - 0.25 * b + 0.125 * a * b
    assert abs(OO.bilinear(1.0, 2.0, 3.0, 4.0, 1.3, 3.8, f(1, 3), f(2, 3), f(1, 4), f(2, 4)) - f(1.3, 3.8)) < 1e-14
    assert OO.bilinear(1.0, 1.0, 3.0, 4.0, 1.0, 3.5, 0, 0, 0, 0) is None


def _raw_case(k=12, nobs=240, seed=3):
    wl = WORKLOADS[0].scaled(nlon=18, nlat=14, nlev=8, nmem=k, n_sst=10, n_ssh=5, n_prof=1, seed=seed)
    case = make_case(wl)
    p = case.params
    rng = np.random.default_rng(seed)
    g = case.grid
    grid = dict(lon=g["lon1"].numpy(), lat=g["lat1"].numpy(), fsm=(g["phi1"] != 1.0).double().numpy(),
                depth=g["depth1"].numpy())
    lon0, lat0 = grid["lon"].min(), grid["lat"].min()
    span_x = grid["lon"].max() - lon0
    span_y = grid["lat"].max() - lat0
    lon = lon0 - 0.05 * span_x + 1.1 * span_x * rng.random(nobs)   # a few outside the grid
    lat = lat0 - 0.05 * span_y + 1.1 * span_y * rng.random(nobs)
    elm = rng.choice(np.array([3073, 3332, 2819, 2820, 2567, 9999], np.int32), nobs, p=[.3, .2, .15, .15, .15, .05])
    lev = np.where(rng.random(nobs) < 0.4, 0.0, -rng.uniform(0.0, 5000.0, nobs))
    lev[rng.random(nobs) < 0.05] = 3.0                                # above the surface
    dat = rng.normal(10.0, 5.0, nobs)
    err = rng.uniform(0.05, 0.5, nobs)
    obs = dict(elm=elm, lon=lon, lat=lat, lev=lev, dat=dat, err=err)
    return case, p, grid, obs


@pytest.mark.gpu
@pytest.mark.parametrize("gross_qc,aoei", [(False, True), (True, False), (False, False)])
def test_obs_operator_matches_oracle(gross_qc, aoei, cuda):
    from sbpom_letkf_v2_b200.obsop import obs_operator
    case, p, grid, obs = _raw_case()
    ref = OO.set_obs(p, grid, obs, case.fcst3d.numpy().astype(np.float64), case.fcst2d.numpy().astype(np.float64),
                     gross_qc=gross_qc, aoei=aoei)
    dev = "cuda:0"
    gt = {k: torch.as_tensor(v, device=dev) for k, v in grid.items()}
    ot = {k: torch.as_tensor(v, device=dev) for k, v in obs.items()}
    r = obs_operator(p, gt, case.fcst3d.to(dev), case.fcst2d.to(dev), ot, gross_qc=gross_qc, aoei=aoei, stats=True)
    assert np.array_equal(r["idx"].cpu().numpy(), ref["idx"])
    assert np.array_equal(r["idy"].cpu().numpy(), ref["idy"])
    qc = r["qc"].cpu().numpy()
    assert np.array_equal(qc, ref["qc"])
    assert 0 < qc.sum() < qc.size                                      # both outcomes exercised
    ok = ~np.isnan(ref["hxmean"])
    for key in ("hxmean", "hxsprd", "dep"):
        got = r[key].cpu().numpy()
        assert np.array_equal(np.isnan(got), np.isnan(ref[key]))
        assert np.abs(got[ok] - ref[key][ok]).max() <= TOL * np.abs(ref[key][ok]).max()
    keep = ref["qc"] == 1
    assert np.abs(r["err"].cpu().numpy()[keep] - ref["err"][keep]).max() <= TOL
    hd = r["hdxf"].cpu().numpy()
    assert np.abs(hd[:, ok] - ref["hdxf"][:, ok]).max() <= TOL * np.abs(ref["hdxf"][:, ok]).max()
    # monit_dep sums over qc = 1, per variable
    st = r["stats"].cpu().numpy()
    assert st[:, 0].sum() == keep.sum()
    assert abs(st[:, 1].sum() - ref["dep"][keep].sum()) <= 1e-10 * max(1.0, np.abs(ref["dep"][keep]).sum())


@pytest.mark.gpu
def test_obs_operator_feeds_the_analysis(cuda):
    """set_obs on the GPU, then the analysis: the same as the oracle analysis of
    the oracle's preprocessed observations (FP64, <= 1e-10)."""
    from oracle import cref
    from sbpom_letkf_v2_b200.analysis import Analysis
    from sbpom_letkf_v2_b200.obsop import analysis_obs, obs_operator
    case, p, grid, obs = _raw_case(k=16, nobs=300, seed=9)
    f3, f2 = case.fcst3d.numpy().astype(np.float64), case.fcst2d.numpy().astype(np.float64)
    ref = OO.set_obs(p, grid, obs, f3, f2)
    keep = ref["qc"] == 1
    ob_ref = dict(elm=obs["elm"][keep], idx=ref["idx"][keep], idy=ref["idy"][keep], lon=obs["lon"][keep],
                  lat=obs["lat"][keep], lev=obs["lev"][keep], err=ref["err"][keep], dep=ref["dep"][keep],
                  hdxf=ref["hdxf"][:, keep])
    g_np = {k: v.numpy() for k, v in case.grid.items()}
    a_ref = cref.da_main(p, g_np, ob_ref, f3, f2, rsize=8)
    dev = "cuda:0"
    r = obs_operator(p, {k: torch.as_tensor(v, device=dev) for k, v in grid.items()},
                     torch.as_tensor(f3, device=dev), torch.as_tensor(f2, device=dev),
                     {k: torch.as_tensor(v, device=dev) for k, v in obs.items()})
    ob = analysis_obs(obs, r, hdxf_dtype=torch.float64)
    an = Analysis(p, case.nij1, int(ob["elm"].numel()), device=dev)
    an.prepare_obs(ob)
    a3, a2 = an.da_main({k: v.to(dev) for k, v in case.grid.items()}, torch.as_tensor(f3, device=dev),
                        torch.as_tensor(f2, device=dev))
    an.close()
    e3 = np.abs(a3.cpu().numpy() - a_ref["anal3d"]).max() / np.abs(a_ref["anal3d"]).max()
    e2 = np.abs(a2.cpu().numpy() - a_ref["anal2d"]).max() / np.abs(a_ref["anal2d"]).max()
    assert e3 <= 1e-10 and e2 <= 1e-10
