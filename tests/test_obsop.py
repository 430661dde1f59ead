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


# ---- observation-space monitors (monit_mean / monit_sprd) --------------------

def test_monit_sums_known_answers():
    """The restatement of monit_mean / monit_sprd on a hand-made set: undef
    hx and unknown elements are skipped, SSH has no surface / interior split."""
    from sbpom_letkf_v2_b200.params import LETKFParams
    p = LETKFParams(nmem=4, nlon=4, nlat=4, nlev=6, nv3d=4, nv2d=1)
    obs = dict(elm=[3073, 3073, 3332, 2567, 3073, 9999], lev=[0.0, -10.0, -5.0, 0.0, 0.0, 0.0],
               dat=[10.0, 11.0, 35.0, 0.5, 9.0, 1.0])
    hx = [9.0, 8.0, 34.5, 0.25, None, 3.0]
    st = OO.monit_sums(p, obs, hx, True)
    t, s, z = p.iv3d_t, p.iv3d_s, p.nv3d + p.iv2d_z
    assert st[t].tolist() == [[2, 4.0, 10.0], [1, 1.0, 1.0], [1, 3.0, 9.0]]
    assert st[s].tolist() == [[1, 0.5, 0.25], [0, 0, 0], [1, 0.5, 0.25]]
    assert st[z].tolist() == [[1, 0.25, 0.0625], [0, 0, 0], [0, 0, 0]]
    assert st.sum() == st[[t, s, z]].sum()
    sp = OO.monit_sums(p, obs, hx, False)
    assert sp[t, 0].tolist() == [2, 17.0, 145.0]


@pytest.mark.gpu
def test_write_ens_monitors_match_the_oracle(cuda):
    """The monitors write_ens_mpi prints (common_io.f90:917-1045) on the GPU:
    ensemble mean / spread fields of the forecast and of an analysis, H of
    each, monit_mean (O-B, O-A) and monit_sprd; against the restatement:
    counts exact, H and the sums within 1e-12 relative."""
    from sbpom_letkf_v2_b200.obsop import MONIT_DEPARTURE, MONIT_VALUE, obs_monitor, write_ens_monitors
    case, p, grid, obs = _raw_case(k=12, nobs=400, seed=5)
    f3, f2 = case.fcst3d.double(), case.fcst2d.double()
    a3 = 0.6 * f3 + 0.4 * f3.mean(1, keepdim=True) + 0.01      # an analysis-like state: spread shrunk, mean moved
    a2 = 0.6 * f2 + 0.4 * f2.mean(1, keepdim=True) - 0.02
    dev = "cuda:0"
    gt = {k: torch.as_tensor(v, device=dev) for k, v in grid.items()}
    ot = {k: torch.as_tensor(v, device=dev) for k, v in obs.items()}
    res = write_ens_monitors(p, gt, ot, f3.to(dev), f2.to(dev), a3.to(dev), a2.to(dev))
    k = p.nmem
    for name, s3, s2 in (("fcst", f3, f2), ("anal", a3, a2)):
        x3, x2 = s3.numpy(), s2.numpy()
        m3, m2 = x3.mean(1), x2.mean(1)
        d3 = np.sqrt(((x3 - m3[:, None]) ** 2).sum(1) / (k - 1))
        d2 = np.sqrt(((x2 - m2[:, None]) ** 2).sum(1) / (k - 1))
        for key, f3f, f2f, mode in (("hxmean", m3, m2, MONIT_DEPARTURE), ("hxsprd", d3, d2, MONIT_VALUE)):
            ref = OO.hx_of_field(p, grid, obs, f3f, f2f)
            want = np.array([np.nan if h is None else h for h in ref])
            got = res[name][key].cpu().numpy()
            assert np.array_equal(np.isnan(got), np.isnan(want))
            ok = ~np.isnan(want)
            assert 0 < ok.sum() < ok.size
            assert np.abs(got[ok] - want[ok]).max() <= TOL * np.abs(want[ok]).max()
            st = obs_monitor(p, ot, res[name][key], mode).cpu().numpy()
            sr = OO.monit_sums(p, obs, ref, mode == MONIT_DEPARTURE)
            assert np.array_equal(st[..., 0], sr[..., 0])
            for j in (1, 2):
                assert np.abs(st[..., j] - sr[..., j]).max() <= TOL * max(1.0, np.abs(sr[..., j]).max())
        m, s = res[name]["mean"], res[name]["sprd"]
        sr = OO.monit_sums(p, obs, OO.hx_of_field(p, grid, obs, m3, m2), True)
        n = sr[..., 0]
        with np.errstate(invalid="ignore", divide="ignore"):
            bias = np.where(n > 0, sr[..., 1] / n, np.nan)
        assert np.array_equal(m["n"].numpy(), n.astype(np.int64))
        assert np.allclose(m["bias"].numpy(), bias, rtol=1e-12, atol=1e-14, equal_nan=True)
        assert s["n"].sum() > 0
