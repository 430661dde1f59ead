"""GPU parity on the benchmark workloads themselves, against the C oracle in
binary64 (oracle/letkf_ref.c), through the C ABI.

* workload 0 (64x48x12, k=20, 3k obs) in full;
* workloads 1 and 2 (400x300x40, k=100 / k=64) on a column sample (every
  197th column, all 40 levels; 197 is prime to nlon, so the sample spans
  every longitude);
* workload 4 (128x96x20, k=128 particles, nmonte=100) on a column sample:
  resampling indices bit-exact for SR, MR and LPFGM;
* the mixed path's transform W (letkf_core, common_letkf.f90:191-208) against
  the oracle on sampled workload-1 points, through sbletkf_core_batched.

A column sample is analysed by passing those columns as the grid (nij1 = the
sample size, observations global), which is how a rank of the reference's
MPI decomposition sees its points (common_mpi.f90:314); every point is
independent of the others, so the sampled analysis equals the full one there.

Tolerances: FP64 path <= 1e-10 relative (max |error| / max |field| per
variable); mixed path <= 1e-4 relative on the analysis mean and spread and on
W; nobsl exactly equal; PF indices bit-exact.
"""
import numpy as np
import pytest
import torch

from oracle import cref
from oracle import letkf_oracle as O
from sbpom_letkf_v2_b200.analysis import core_batched
from sbpom_letkf_v2_b200.params import DA_LPF, DA_LPFGM, RM_MR, RM_SR
from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case, pf_uniforms
from tests._util import field_relerr, incr_relerr
from tests.test_gpu_parity import _mean_spread_err, run_gpu

pytestmark = pytest.mark.gpu
TOL64 = 1e-10
TOL_MIXED = 1e-4


def _columns(case, cols, uniforms=None):
    """numpy grid / obs / forecast of the columns `cols` (and the uniforms of
    those points, point ids k*ncol + j)."""
    dev = case.fcst3d.device
    ct = torch.as_tensor(np.asarray(cols), device=dev)
    g = {k: (v.index_select(v.dim() - 1, ct)).cpu().numpy() for k, v in case.grid.items()}
    ob = {k: v.cpu().numpy() for k, v in case.obs.items()}
    f3 = case.fcst3d.index_select(3, ct).cpu().numpy()
    f2 = case.fcst2d.index_select(2, ct).cpu().numpy()
    return g, ob, f3, f2


def _check_fp64(r, ref, f3):
    assert (r["status"] == 0).all()
    assert np.array_equal(r["nobsl"], ref["nobsl"])
    assert field_relerr(r["anal3d"], ref["anal3d"]) <= TOL64
    assert field_relerr(r["anal2d"], ref["anal2d"]) <= TOL64
    assert incr_relerr(r["anal3d"], ref["anal3d"], f3) <= TOL64


def _check_mixed(r, ref):
    assert (r["status"] == 0).all()
    em, es = _mean_spread_err(r["anal3d"], ref["anal3d"])
    em2, es2 = _mean_spread_err(r["anal2d"], ref["anal2d"])
    assert max(em, em2) <= TOL_MIXED and max(es, es2) <= TOL_MIXED
    return max(em, em2), max(es, es2)


def test_workload0_in_full_fp64_and_mixed(cuda):
    case = make_case(WORKLOADS[0])
    g = {k: v.numpy() for k, v in case.grid.items()}
    ob = {k: v.numpy() for k, v in case.obs.items()}
    f3, f2 = case.fcst3d.numpy(), case.fcst2d.numpy()
    ref = cref.da_main(case.params, g, ob, f3, f2, rsize=8)
    assert ref["nobsl"].max() > 0
    _check_fp64(run_gpu(case.params, g, ob, f3, f2), ref, f3)
    _check_mixed(run_gpu(case.params.replace(precision=1), g, ob, f3, f2), ref)


@pytest.fixture(scope="module")
def workload1(cuda):
    case = make_case(WORKLOADS[1], device=cuda)
    cols = np.arange(0, case.nij1, 197)
    g, ob, f3, f2 = _columns(case, cols)
    ref = cref.da_main(case.params, g, ob, f3, f2, rsize=8)
    yield case, g, ob, f3, f2, ref
    del case
    torch.cuda.empty_cache()


def test_workload1_sampled_columns_fp64(workload1):
    case, g, ob, f3, f2, ref = workload1
    assert ref["nobsl"].max() > 1000 and (ref["nobsl"] == 0).any()
    _check_fp64(run_gpu(case.params, g, ob, f3, f2, dev=case.fcst3d.device), ref, f3)


def test_workload1_sampled_columns_mixed(workload1):
    case, g, ob, f3, f2, ref = workload1
    _check_mixed(run_gpu(case.params.replace(precision=1), g, ob, f3, f2, dev=case.fcst3d.device), ref)


def test_workload1_mixed_transform_w_against_letkf_core(workload1):
    """W and wvec of the mixed path (tensor-core Gram, FP64 eigensolve) on 48
    sampled workload-1 points with observations, against the oracle's
    letkf_core; the FP64 path is held to 1e-10 on the same points."""
    case, g, ob, f3, f2, ref = workload1
    p = case.params
    so = O.sort_obs(ob, p.nlon, p.nlat)
    rng = np.random.default_rng(17)
    nob = ref["nobsl"]
    pts = [(k, i) for k, i in zip(*np.nonzero(nob > p.nmem))]
    pick = [pts[j] for j in rng.choice(len(pts), size=48, replace=False)]
    blocks = []
    for k, i in pick:
        cand, dist = O.column_candidates(p, g, so, i)
        _, h, rd, rl, dp, _, _ = O.obs_local(p, so, cand, dist, k, g["depth1"][k, i])
        assert h.shape[0] == nob[k, i]
        blocks.append((h, rd, rl, dp))
    dev = case.fcst3d.device
    nobl = torch.tensor([b[0].shape[0] for b in blocks], dtype=torch.int64, device=dev)
    hd = torch.tensor(np.concatenate([b[0].T.reshape(-1) for b in blocks]), device=dev)
    cat = lambda j: torch.tensor(np.concatenate([b[j] for b in blocks]), device=dev)
    out = {}
    for prec in (0, 1):
        wv, wm = core_batched(p.replace(precision=prec), nobl, hd, cat(1), cat(2), cat(3))
        ew = ev = 0.0
        for q, (h, rd, rl, dp) in enumerate(blocks):
            rv, rm = O.letkf_core(p, h, rd, rl, dp)
            ew = max(ew, np.abs(wm[q].cpu().numpy().T - rm).max() / np.abs(rm).max())
            ev = max(ev, np.abs(wv[q].cpu().numpy() - rv).max() / np.abs(rv).max())
        out[prec] = (ew, ev)
    assert out[0][0] <= TOL64 and out[0][1] <= TOL64
    assert out[1][0] <= TOL_MIXED and out[1][1] <= TOL_MIXED
    print(f"mixed W rel err {out[1][0]:.2e}, wvec {out[1][1]:.2e}; fp64 W {out[0][0]:.2e}")


@pytest.fixture(scope="module")
def workload2(cuda):
    case = make_case(WORKLOADS[2], device=cuda)
    cols = np.arange(0, case.nij1, 197)
    g, ob, f3, f2 = _columns(case, cols)
    ref = cref.da_main(case.params, g, ob, f3, f2, rsize=8)
    yield case, g, ob, f3, f2, ref
    del case
    torch.cuda.empty_cache()


def test_workload2_sampled_columns_fp64_and_mixed(workload2):
    """The uneven workload: the sample holds points with more than 12288
    search-box candidates, which the mixed kernel routes to the FP64 Gram."""
    case, g, ob, f3, f2, ref = workload2
    assert ref["nobsl"].max() > 12288 and (ref["nobsl"] == 0).any()
    dev = case.fcst3d.device
    _check_fp64(run_gpu(case.params, g, ob, f3, f2, dev=dev), ref, f3)
    _check_mixed(run_gpu(case.params.replace(precision=1), g, ob, f3, f2, dev=dev), ref)


@pytest.mark.parametrize("da,rm,stride", [(DA_LPF, RM_SR, 61), (DA_LPF, RM_MR, 307), (DA_LPFGM, RM_SR, 61)])
def test_workload4_k128_nmonte100_indices_bit_exact(da, rm, stride, cuda):
    wl = WORKLOADS[4]
    case = make_case(wl, device=cuda, iswitch_da=da, rm=rm, nmonte=100)
    assert case.params.nmem == 128 and case.params.nmonte == 100
    cols = np.arange(0, case.nij1, stride)
    g, ob, f3, f2 = _columns(case, cols)
    P = case.params.nlev * cols.size
    uni = pf_uniforms(P, 100, 128, rm, seed=23).numpy()
    ref = cref.da_main(case.params, g, ob, f3, f2, uniforms=uni, rsize=8, want_src=True)
    r = run_gpu(case.params, g, ob, f3, f2, uni=uni, want_src=True, dev=case.fcst3d.device)
    assert (r["status"] == 0).all()
    assert np.array_equal(r["nobsl"], ref["nobsl"])
    has = ref["nobsl"].reshape(-1) > 0
    assert has.sum() > 100
    assert np.array_equal(r["src"][has], ref["src"][has])
    assert field_relerr(r["anal3d"], ref["anal3d"]) <= TOL64
    assert field_relerr(r["anal2d"], ref["anal2d"]) <= TOL64
