"""Known answers of the local transforms, derived from the reference's
semantics (letkf/run/src/common_letkf.f90:37-210, common_lpfgm.f90:89-263):

* nobsl = 0: W = sqrt(rho) I, wvec = 0                       (letkf_core_noobs)
* one observation y (sum_j y_j = 0), weight w = rloc/rdiag:
    A = alpha I + w y y^T, alpha = (k-1)/rho
    W = sqrt(k-1) [alpha^-1/2 (I - u u^T) + (alpha + w|y|^2)^-1/2 u u^T], u = y/|y|
    wvec = w dep y / (alpha + w |y|^2)
* W symmetric and W^2 = (k-1) Pa; W 1 = sqrt(rho) 1 because Y 1 = 0
* PF with equal likelihoods (cwgt = i/k): every particle drawn once by SR
  for a uniform u whose offset u/k^2 is far above rounding (u = 0 puts every
  draw on a cwgt boundary), so with diagonal priority W_LPF = I
* diagonal-priority resampling matrix: 0/1 columns summing to one, and a
  drawn particle keeps its own column

Each property is checked on the oracle (CPU) and on the GPU's batched core
(sbletkf_core_batched) at 1e-12 (FP64) or exactly (PF)."""
import numpy as np
import pytest
import torch

from oracle import letkf_oracle as O
from sbpom_letkf_v2_b200.params import DA_LPF, RM_MR, RM_SR, LETKFParams

TOL = 1e-12


def _params(k, **kw):
    base = dict(nmem=k, nlon=8, nlat=8, nlev=2, nv3d=4, nv2d=1, cov_infl_mul=1.3, nmonte=1)
    base.update(kw)
    return LETKFParams(**base)


def _rand_block(rng, n, k):
    h = rng.standard_normal((n, k))
    h -= h.mean(axis=1, keepdims=True)          # Y 1 = 0 as for H(x) perturbations
    rd = rng.uniform(0.05, 0.5, n)
    rl = rng.uniform(0.1, 1.0, n)
    dp = rng.standard_normal(n)
    return h, rd, rl, dp


def _single_obs_closed_form(p, y, rd, rl, d):
    k = p.nmem
    alpha = (k - 1) / p.cov_infl_mul
    w = rl / rd
    ny2 = float(y @ y)
    u = y / np.sqrt(ny2)
    uu = np.outer(u, u)
    lam1 = alpha + w * ny2
    W = np.sqrt(k - 1) * ((np.eye(k) - uu) / np.sqrt(alpha) + uu / np.sqrt(lam1))
    wvec = w * d * y / lam1
    return wvec, W


# ---- oracle ---------------------------------------------------------------

def test_oracle_noobs_and_single_observation():
    p = _params(16)
    ev, em = O.letkf_core_noobs(p)
    assert np.array_equal(ev, np.zeros(16)) and np.allclose(em, np.sqrt(1.3) * np.eye(16), rtol=0, atol=0)
    rng = np.random.default_rng(3)
    h, rd, rl, dp = _rand_block(rng, 1, 16)
    wv, wm = O.letkf_core(p, h, rd, rl, dp)
    cv, cm = _single_obs_closed_form(p, h[0], rd[0], rl[0], dp[0])
    assert np.abs(wm - cm).max() <= TOL * np.abs(cm).max()
    assert np.abs(wv - cv).max() <= TOL * np.abs(cv).max()


@pytest.mark.parametrize("n", [3, 40])
def test_oracle_w_symmetric_square_and_ones(n):
    p = _params(20)
    h, rd, rl, dp = _rand_block(np.random.default_rng(n), n, 20)
    wv, wm, ev, evec, pa = O.letkf_core(p, h, rd, rl, dp, return_eig=True)
    assert np.abs(wm - wm.T).max() <= TOL * np.abs(wm).max()
    assert np.abs(wm @ wm - (p.nmem - 1) * pa).max() <= 1e-11 * np.abs(wm @ wm).max()
    assert np.abs(wm @ np.ones(20) - np.sqrt(p.cov_infl_mul)).max() <= 1e-11


def test_oracle_pf_equal_likelihoods_identity():
    k = 24
    p = _params(k, iswitch_da=DA_LPF, rm=RM_SR, dp=True)
    h = np.tile(np.linspace(-1, 1, 5)[:, None], (1, k))   # same value for every particle
    dp = np.zeros(5)
    wgt = O.pf_weight_gauss_likelihood(dp, h, np.ones(5), np.ones(5))
    assert np.allclose(O.cumulative(wgt), np.arange(1, k + 1) / k, rtol=0, atol=1e-15)
    for u in (0.25, 0.37, 0.999):
        _, wm, _ = O.lpf_core(p, h, np.ones(5), np.ones(5), dp, np.array([u]))
        assert np.array_equal(wm, np.eye(k))


# ---- GPU batched core ---------------------------------------------------------

def _gpu_core(p, blocks, uniforms=None):
    from sbpom_letkf_v2_b200.analysis import core_batched
    dev = "cuda:0"
    nob = torch.tensor([b[0].shape[0] for b in blocks], dtype=torch.int64, device=dev)
    cat = lambda j: torch.tensor(np.concatenate([b[j] for b in blocks]) if blocks else np.zeros(0), device=dev)
    hd = torch.tensor(np.concatenate([b[0].T.reshape(-1) for b in blocks]), device=dev)
    uni = None if uniforms is None else torch.tensor(uniforms, device=dev)
    wv, wm = core_batched(p, nob, hd, cat(1), cat(2), cat(3), uniforms=uni)
    return wv.cpu().numpy(), wm.cpu().numpy().transpose(0, 2, 1)   # W(i,j) at [q][i][j]


@pytest.mark.gpu
@pytest.mark.parametrize("k", [8, 20, 100])
def test_gpu_core_known_answers(k, cuda):
    p = _params(k)
    rng = np.random.default_rng(k)
    blocks = [(np.zeros((0, k)), np.zeros(0), np.zeros(0), np.zeros(0)), _rand_block(rng, 1, k),
              _rand_block(rng, 5, k), _rand_block(rng, 3 * k, k)]
    wv, wm = _gpu_core(p, blocks)
    assert np.array_equal(wv[0], np.zeros(k))
    assert np.abs(wm[0] - np.sqrt(p.cov_infl_mul) * np.eye(k)).max() <= TOL
    h, rd, rl, dp = blocks[1]
    cv, cm = _single_obs_closed_form(p, h[0], rd[0], rl[0], dp[0])
    assert np.abs(wm[1] - cm).max() <= TOL * np.abs(cm).max()
    assert np.abs(wv[1] - cv).max() <= TOL * np.abs(cv).max()
    for q in (2, 3):
        W = wm[q]
        _, _, _, _, pa = O.letkf_core(p, *blocks[q], return_eig=True)
        assert np.abs(W - W.T).max() <= TOL * np.abs(W).max()
        assert np.abs(W @ W - (k - 1) * pa).max() <= 1e-11 * np.abs(W @ W).max()
        assert np.abs(W @ np.ones(k) - np.sqrt(p.cov_infl_mul)).max() <= 1e-11


@pytest.mark.gpu
def test_gpu_pf_equal_likelihoods_and_dp_structure(cuda):
    k = 32
    p = _params(k, iswitch_da=DA_LPF, rm=RM_SR, dp=True)
    h = np.tile(np.linspace(-1, 1, 5)[:, None], (1, k))
    blk = (h, np.ones(5), np.ones(5), np.zeros(5))
    _, wm = _gpu_core(p, [blk, blk, blk], uniforms=np.array([[0.25], [0.37], [0.999]]))
    for q in range(3):
        assert np.array_equal(wm[q], np.eye(k))
    # random likelihoods, MR, one draw: a 0/1 matrix, one particle per member,
    # and every drawn particle keeps its own member (diagonal priority)
    pm = _params(k, iswitch_da=DA_LPF, rm=RM_MR, dp=True)
    rng = np.random.default_rng(5)
    blocks = [_rand_block(rng, 6, k) for _ in range(4)]
    uni = rng.random((4, 1, k))
    _, wm = _gpu_core(pm, blocks, uniforms=uni)
    for q in range(4):
        W = wm[q]                                   # W(i,j): particle i -> member j
        assert set(np.unique(W)) <= {0.0, 1.0}
        assert np.array_equal(W.sum(axis=0), np.ones(k))
        drawn = W.sum(axis=1) > 0
        assert np.all(np.diag(W)[drawn] == 1.0)
        _, wo, _ = O.lpf_core(pm, *blocks[q], uni[q])
        assert np.array_equal(W, wo)
