"""FP64 CPU oracle of the sbPOM-LETKF analysis step (LETKF, LPF, LPFGM).

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg may import this module, and only as the checker;
the product path (sbpom_letkf_v2_b200) never does.

A restatement, in numpy/scipy binary64, of the reference's Fortran with
r_size = kind(0d0); every function cites the lines it follows (paths relative
to the reference project, ``src/`` = ``letkf/run/src/``).  The reference
cannot be compiled here (no Fortran compiler, MPI or netCDF) and ships no
tests, fixtures or golden vectors for this path, so the LETKF / LPF
arithmetic is **parity unpinned**: it is pinned only by analytic known
answers (tests/test_oracle_*.py) and by agreement with the independent C
restatement in oracle/letkf_ref.c.  MT19937 is pinned by its published known
answer (oracle/mt19937.py).

Evaluation order follows the Fortran where it matters for bit-exactness: the
PF log-likelihood is accumulated serially in obs order as
``ll - (((0.5*d)*d)*rloc)/rdiag`` (src/common_lpfgm.f90:64-69), sums are
left-to-right, and LAPACK ``dsyev('V','U')`` is the eigensolver
(src/common.f90:1016).
"""
from __future__ import annotations

import dataclasses

import numpy as np
import scipy.linalg.lapack as lapack

# ---------------------------------------------------------------------------
# numerics helpers (src/common.f90)
# ---------------------------------------------------------------------------


def nint(x):
    """Fortran NINT: nearest integer, halves away from zero."""
    x = np.asarray(x, dtype=np.float64)
    t = np.trunc(x)
    frac = np.abs(x - t)
    return (t + np.sign(x) * (frac >= 0.5)).astype(np.int64)


def distance_2p(lona, lata, lonb, latb, pi, re):
    """Great-circle distance, spherical law of cosines (src/common.f90:79-101)."""
    cosd = (np.sin(pi * lata / 180.0) * np.sin(pi * latb / 180.0)
            + np.cos(pi * lata / 180.0) * np.cos(pi * latb / 180.0) * np.cos(pi * (lonb - lona) / 180.0))
    cosd = np.minimum(1.0, cosd)
    cosd = np.maximum(-1.0, cosd)
    return re * np.arccos(cosd)


def mtx_eigen(a):
    """dsyev('V','U') then descending order with negative-eigenvalue
    reconditioning (src/common.f90:992-1050).  Returns (eval, evec, np)."""
    n = a.shape[0]
    w, v, info = lapack.dsyev(np.asarray(a, dtype=np.float64), compute_v=1, lower=0)
    if info != 0:
        raise RuntimeError(f"***Error: DSYEV, INFO: {info}")
    npos = n
    if w[n - 1] < 0:
        raise RuntimeError("***Error (mtx_eigen): All Eigenvalues are Negative")
    w = w.copy()
    v = v.copy()
    neg = w < 0.0
    npos -= int(neg.sum())
    w[neg] = 0.0
    v[:, neg] = 0.0
    return w[::-1].copy(), v[:, ::-1].copy(), npos


# ---------------------------------------------------------------------------
# observation bucketing (src/common_obs.f90:266-377)
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class SortedObs:
    perm: np.ndarray        # sorted position -> input index
    cellstart: np.ndarray   # [nlon*nlat+1] first sorted position of cell (j-1)*nlon+(i-1)
    nobsgrd: np.ndarray     # [nlon, nlat] cumulative counts as in the reference
    elm: np.ndarray
    lon: np.ndarray
    lat: np.ndarray
    lev: np.ndarray
    err: np.ndarray
    dep: np.ndarray
    hdxf: np.ndarray        # [nobs_sorted, nmem] float64


def sort_obs(obs: dict, nlon: int, nlat: int) -> SortedObs:
    """Row-major (idy, then idx) cell order, stable within a cell, and the
    cumulative count nobsgrd(i,j) (src/common_obs.f90:274-377)."""
    idx = np.asarray(obs["idx"], dtype=np.int64)
    idy = np.asarray(obs["idy"], dtype=np.int64)
    if idx.size and (idx.min() < 1 or idx.max() > nlon - 1 or idy.min() < 1 or idy.max() > nlat - 1):
        raise ValueError("obs cell index outside [1,nlon-1]x[1,nlat-1]")
    key = (idy - 1) * nlon + (idx - 1)
    perm = np.argsort(key, kind="stable")
    counts = np.bincount(key, minlength=nlon * nlat)
    cellstart = np.zeros(nlon * nlat + 1, dtype=np.int64)
    np.cumsum(counts, out=cellstart[1:])
    nobsgrd = cellstart[1:].reshape(nlat, nlon).T.copy()
    nobsgrd[:, nlat - 1] = 0          # row nlat is never filled (loop j=1..nlat-1)
    hdxf = np.asarray(obs["hdxf"], dtype=np.float64)     # [nmem][nobs]
    return SortedObs(perm=perm, cellstart=cellstart, nobsgrd=nobsgrd,
                     elm=np.asarray(obs["elm"])[perm], lon=np.asarray(obs["lon"], np.float64)[perm],
                     lat=np.asarray(obs["lat"], np.float64)[perm], lev=np.asarray(obs["lev"], np.float64)[perm],
                     err=np.asarray(obs["err"], np.float64)[perm], dep=np.asarray(obs["dep"], np.float64)[perm],
                     hdxf=np.ascontiguousarray(hdxf[:, perm].T))


def obs_local_sub(so: SortedObs, nlon, imin, imax, jmin, jmax):
    """Candidate sorted positions, rows jmin..jmax, cells imin..imax
    (src/common_da.f90:297-348, expressed with cellstart instead of nobsgrd)."""
    parts = []
    for j in range(jmin, jmax + 1):
        ib = so.cellstart[(j - 1) * nlon + (imin - 1)]
        ie = so.cellstart[(j - 1) * nlon + imax]
        if ie > ib:
            parts.append(np.arange(ib, ie))
    return np.concatenate(parts) if parts else np.zeros(0, dtype=np.int64)


def search_box(p, g, i):
    """imin..jmax of point i (src/common_da.f90:158-161)."""
    imin = max(int(nint(g["ri1"][i] - p.dist_zero / g["dlon1"][i])), 1)
    imax = min(int(nint(g["ri1"][i] + p.dist_zero / g["dlon1"][i])), p.nlon)
    jmin = max(int(nint(g["rj1"][i] - p.dist_zero / g["dlat1"][i])), 1)
    jmax = min(int(nint(g["rj1"][i] + p.dist_zero / g["dlat1"][i])), p.nlat)
    return imin, imax, jmin, jmax


def column_candidates(p, g, so: SortedObs, i):
    """Horizontal part of obs_local for point i: candidate positions within the
    cutoff and their distances (the distance does not depend on the level)."""
    imin, imax, jmin, jmax = search_box(p, g, i)
    cand = obs_local_sub(so, p.nlon, imin, imax, jmin, jmax)
    dist = distance_2p(so.lon[cand], so.lat[cand], g["lon1"][i], g["lat1"][i], p.pi, p.re)
    return cand, dist


def obs_local(p, so: SortedObs, cand, dist, k, rdep):
    """Local obs of level k (0-based) from the column candidates, in
    candidate order (src/common_da.f90:209-293)."""
    elm = so.elm[cand]
    is_z = elm == p.id_z_obs
    if k < p.nlev - 1:
        dlev = np.where(is_z, np.abs(rdep), np.abs(so.lev[cand] - rdep))
    else:
        dlev = np.where(is_z, 0.0, np.abs(so.lev[cand] - rdep))
    keep = ~(p.dist_zerov < dlev) & ~(p.dist_zero < dist)
    sel = cand[keep]
    d = dist[keep]
    dl = dlev[keep]
    rdiag = so.err[sel] ** 2
    if p.sigma_obsv <= 0.0:
        rloc = np.exp(-0.5 * (d / p.sigma_obs) ** 2)
    else:
        rloc = np.exp(-0.5 * ((d / p.sigma_obs) ** 2 + (dl / p.sigma_obsv) ** 2))
    return sel, so.hdxf[sel], rdiag, rloc, so.dep[sel], d, dl


# ---------------------------------------------------------------------------
# transform cores
# ---------------------------------------------------------------------------


def letkf_core_noobs(p):
    """W = sqrt(rho) I, wvec = 0 (src/common_letkf.f90:37-57)."""
    k = p.nmem
    return np.zeros(k), np.eye(k) * np.sqrt(p.cov_infl_mul)


def letkf_core(p, hdxf, rdiag, rloc, dep, infl=None, return_eig=False):
    """Local ensemble transform (src/common_letkf.f90:61-210), binary64.
    hdxf is [nobsl, nmem]."""
    k = p.nmem
    infl = p.cov_infl_mul if infl is None else infl
    rlinv = hdxf * rloc[:, None] / rdiag[:, None]                 # :93-97
    work1 = rlinv.T @ hdxf                                        # :114-116
    work1[np.diag_indices(k)] += float(k - 1) / infl              # :124-126
    ev, evec, _ = mtx_eigen(work1)                                # :132
    pa = (evec / ev[None, :]) @ evec.T                            # :139-150
    work2 = pa @ rlinv.T                                          # :162-166
    wvec = work2 @ dep                                            # :178-184
    wmat = (evec * np.sqrt(float(k - 1) / ev)[None, :]) @ evec.T  # :191-202
    if return_eig:
        return wvec, wmat, ev, evec, pa
    return wvec, wmat


def pf_weight_gauss_likelihood(dep, hdxf, rloc, rdiag):
    """Normalised Gaussian-likelihood weights (src/common_lpfgm.f90:38-77):
    serial FP64 accumulation in obs order, max-subtracted exp, normalise."""
    n, k = hdxf.shape
    ll = np.zeros(k)
    for i in range(n):
        d = dep[i] - hdxf[i, :]
        ll = ll - (((0.5 * d) * d) * rloc[i]) / rdiag[i]
    llmax = ll.max()
    ex = np.exp(ll - llmax)
    s = 0.0
    for j in range(k):
        s = s + ex[j]
    return ex / s


def cumulative(wgt):
    """cwgt(i) = cwgt(i-1) + wgt(i), serial (src/common_lpfgm.f90:252-255)."""
    c = np.empty_like(wgt)
    acc = 0.0
    for i in range(wgt.size):
        acc = wgt[i] if i == 0 else acc + wgt[i]
        c[i] = acc
    return c


def resampling_rand(p, u):
    """The draw's rand(1..k) from its uniforms (src/common_lpfgm.f90:110-134).
    SR: u is a scalar; MR: u is [k]."""
    k = p.nmem
    if p.rm == 0:
        r = np.empty(k)
        r1 = (u + 1.0 - 1.0) / float(k)          # i = 1: rand(1) is overwritten first
        r[0] = r1
        base = u if p.sr_textbook else r1        # reference: later i use the new rand(1)
        for i in range(2, k + 1):
            r[i - 1] = (base + float(i) - 1.0) / float(k)
        return r
    return np.sort(np.asarray(u, dtype=np.float64))


def resampling_src(p, cwgt, rand):
    """src[j] = 0-based particle taken by member j for one draw
    (src/common_lpfgm.f90:136-195)."""
    k = p.nmem
    inum = np.empty(k, dtype=np.int64)
    for j in range(k):
        hit = np.nonzero(rand[j] <= cwgt)[0]
        inum[j] = hit[0] if hit.size else k - 1
    if not p.dp:
        return inum
    src = np.full(k, -1, dtype=np.int64)
    used = np.zeros(k, dtype=bool)
    pending = inum.copy()
    for i in range(k):                     # diagonal priority (:156-165)
        kk = pending[i]
        if used[kk]:
            continue
        src[kk] = kk
        used[kk] = True
        pending[i] = -1
    for i in range(k):                     # remaining rows to unused columns (:168-181)
        if pending[i] < 0:
            continue
        free = np.nonzero(~used)[0]
        if free.size:
            src[free[0]] = pending[i]
            used[free[0]] = True
        pending[i] = -1
    return src


def lpf_core(p, hdxf, rdiag, rloc, dep, uniforms):
    """LPF transform (src/common_lpfgm.f90:213-263).  uniforms: [nmonte] (SR)
    or [nmonte, k] (MR).  Returns (wvec, W, src[nmonte, k])."""
    k = p.nmem
    wgt = pf_weight_gauss_likelihood(dep, hdxf, rloc, rdiag)
    cwgt = cumulative(wgt)
    wmat = np.zeros((k, k))
    srcs = np.empty((p.nmonte, k), dtype=np.int64)
    for d in range(p.nmonte):
        src = resampling_src(p, cwgt, resampling_rand(p, uniforms[d]))
        srcs[d] = src
        rs = np.zeros((k, k))
        rs[src, np.arange(k)] = 1.0
        wmat = wmat + rs / float(p.nmonte)
    return np.zeros(k), wmat, srcs


def gm_core(p, hdxf, rdiag, rloc, dep):
    """Gaussian-mixture shift matrix (src/common_lpfgm.f90:279-405)."""
    k = p.nmem
    rlinv = hdxf * rloc[:, None] / rdiag[:, None]
    work1 = rlinv.T @ hdxf
    work1[np.diag_indices(k)] += float(k - 1) / p.cov_infl_gm
    ev, evec, _ = mtx_eigen(work1)
    pa = (evec / ev[None, :]) @ evec.T
    work2 = pa @ rlinv.T
    wmat = work2 @ (dep[:, None] - hdxf)
    wmat[np.diag_indices(k)] += 1.0
    return np.zeros(k), wmat


def lpfgm_core_noobs(p):
    """W = I, wvec = 0 (src/common_lpfgm.f90:422-440)."""
    return np.zeros(p.nmem), np.eye(p.nmem)


def lpfgm_core(p, hdxf, rdiag, rloc, dep, uniforms):
    """LPF (iswitch_da=2) or LPFGM (=3) (src/common_lpfgm.f90:444-494)."""
    _, w_lpf, srcs = lpf_core(p, hdxf, rdiag, rloc, dep, uniforms)
    if p.iswitch_da == 2:
        return np.zeros(p.nmem), w_lpf, srcs
    _, w_gm = gm_core(p, hdxf, rdiag, rloc, dep)
    return np.zeros(p.nmem), w_gm @ w_lpf, srcs


# ---------------------------------------------------------------------------
# ensemble update (src/common_da.f90:354-533)
# ---------------------------------------------------------------------------


def mean_spread_pert(x):
    """x [nmem, nvd] -> mean, spread (k-1 denominator), perturbation
    (src/common_da.f90:354-401)."""
    k = x.shape[0]
    m = np.zeros(x.shape[1])
    for j in range(k):
        m = m + x[j]
    m = m / float(k)
    s = np.zeros(x.shape[1])
    for j in range(k):
        s = s + (x[j] - m) * (x[j] - m)
    s = np.sqrt(s / float(k - 1))
    return m, s, x - m[None, :]


def analysis_ensemble(fm, dxf, wvec, wmat):
    """anal(j,v) = xm_v + sum_i dxf(i,v)(wvec(i)+W(i,j)) (src/common_da.f90:407-432)."""
    return fm[None, :] + (wvec[:, None] + wmat).T @ dxf


def update_point(p, x, wvec, wmat, xs_f=None):
    """Analysis of one point's [nmem, nvd] block with RTPP / RTPS
    (src/common_da.f90:88-113)."""
    fm, fs, dxf = mean_spread_pert(x)
    anal = analysis_ensemble(fm, dxf, wvec, wmat)
    am, asp, dxa = mean_spread_pert(anal)
    if 0.0 < p.alpha_rtpp:
        anal = am[None, :] + p.alpha_rtpp * dxf + (1.0 - p.alpha_rtpp) * dxa
    if 0.0 < p.alpha_rtps:
        fac = np.where(asp == 0.0, 0.0, p.alpha_rtps * fs / np.where(asp == 0.0, 1.0, asp) + (1.0 - p.alpha_rtps))
        anal = am[None, :] + dxa * fac[None, :]
    return anal


def round_off(p, anal3d, phi1):
    """T/S clamp for k >= 2 where phi1 /= 1 (src/common_da.f90:506-533).
    anal3d [nv3d][nmem][nlev][nij1], in place."""
    sea = phi1 != 1.0
    for iv, lo, hi in ((p.iv3d_t, p.tmin, p.tmax), (p.iv3d_s, p.smin, p.smax)):
        blk = anal3d[iv, :, 1:, :]
        clamped = np.minimum(np.maximum(blk, lo), hi)
        blk[...] = np.where(sea[None, None, :], clamped, blk)


# ---------------------------------------------------------------------------
# the analysis step (src/common_da.f90:22-124)
# ---------------------------------------------------------------------------


@dataclasses.dataclass
class OracleResult:
    anal3d: np.ndarray
    anal2d: np.ndarray
    nobsl: np.ndarray                 # [nlev, nij1]
    wvec: dict                        # (k, i) -> wvec  (only for points in `keep`)
    wmat: dict
    src: dict                         # (k, i) -> [nmonte, nmem] (PF)


def da_main(p, grid, obs, fcst3d, fcst2d, uniforms=None, points=None, keep=()):
    """Analysis of every point (or only `points`, a list of (k, i) 0-based).

    grid: lon1 lat1 ri1 rj1 dlon1 dlat1 phi1 [nij1], depth1 [nlev][nij1].
    obs: elm idx idy lon lat lev err dep [nobs], hdxf [nmem][nobs].
    fcst3d [nv3d][nmem][nlev][nij1], fcst2d [nv2d][nmem][nij1] (any float dtype).
    uniforms: [P][nmonte] (SR) or [P][nmonte][nmem] (MR), P index k*nij1+i.
    Returns FP64 analyses of the same layout."""
    g = {kk: np.asarray(v, dtype=np.float64) for kk, v in grid.items()}
    f3 = np.asarray(fcst3d, dtype=np.float64)
    f2 = np.asarray(fcst2d, dtype=np.float64)
    nij1 = g["lon1"].size
    nobs = int(np.asarray(obs["elm"]).size)
    if nobs == 0:                                         # :57-61
        return OracleResult(f3.copy(), f2.copy(), np.zeros((p.nlev, nij1), np.int64), {}, {}, {})
    so = sort_obs(obs, p.nlon, p.nlat)
    a3 = np.zeros_like(f3)
    a2 = np.zeros_like(f2)
    nobsl = np.full((p.nlev, nij1), -1, dtype=np.int64)
    wv, wm, srcd = {}, {}, {}
    keep = set(keep)
    if points is None:
        cols = {i: list(range(p.nlev)) for i in range(nij1)}
    else:
        cols = {}
        for (k, i) in points:
            cols.setdefault(i, []).append(k)
    for i, levs in cols.items():
        cand, dist = column_candidates(p, g, so, i)
        for k in levs:
            rdep = g["depth1"][k, i]
            sel, hdxf, rdiag, rloc, dep, _, _ = obs_local(p, so, cand, dist, k, rdep)
            n = sel.size
            nobsl[k, i] = n
            pidx = k * nij1 + i
            src = None
            if p.iswitch_da == 1:
                wvec, wmat = letkf_core_noobs(p) if n == 0 else letkf_core(p, hdxf, rdiag, rloc, dep)
            else:
                if n == 0:
                    wvec, wmat = lpfgm_core_noobs(p)
                else:
                    wvec, wmat, src = lpfgm_core(p, hdxf, rdiag, rloc, dep, uniforms[pidx])
            if (k, i) in keep:
                wv[(k, i)], wm[(k, i)] = wvec, wmat
                if src is not None:
                    srcd[(k, i)] = src
            x = f3[:, :, k, i].T                          # [nmem, nv3d]
            a3[:, :, k, i] = update_point(p, x, wvec, wmat).T
            if k == p.nlev - 1 and f2.shape[0] > 0:
                a2[:, :, i] = update_point(p, f2[:, :, i].T, wvec, wmat).T
    if p.roff:
        round_off(p, a3, g["phi1"])
    return OracleResult(a3, a2, nobsl, wv, wm, srcd)


def count_nobsl(p, grid, obs):
    """nobsl of every point [nlev, nij1] (src/common_da.f90:133-205)."""
    g = {kk: np.asarray(v, dtype=np.float64) for kk, v in grid.items()}
    nij1 = g["lon1"].size
    out = np.zeros((p.nlev, nij1), dtype=np.int64)
    if np.asarray(obs["elm"]).size == 0:
        return out
    so = sort_obs(obs, p.nlon, p.nlat)
    for i in range(nij1):
        cand, dist = column_candidates(p, g, so, i)
        for k in range(p.nlev):
            out[k, i] = obs_local(p, so, cand, dist, k, g["depth1"][k, i])[0].size
    return out
