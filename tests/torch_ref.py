"""FP64 torch restatement of the LETKF analysis, differentiable by autograd
through torch.linalg.eigh: the reference for the backward kernel.

TEST INFRASTRUCTURE ONLY.  Observation selection (which obs a point uses,
their distances and level differences) comes from the oracle
(oracle/letkf_oracle.py, letkf/run/src/common_da.f90:133-293) and is a fixed
set; everything that depends on dep, rdiag, rho and sigma_obs is torch:

  rloc = exp(-((d/sigma)^2 + (dlev/sigma_v)^2)/2)            common_da.f90:283-287
  letkf_core: A = Y^T diag(rloc/rdiag) Y + (k-1)/rho I       common_letkf.f90:93-126
              Pa, wvec = Pa Y^T R^-1 dep, W = sqrt(k-1) A^-1/2  :139-202
  update, RTPP / RTPS, T/S round-off                          common_da.f90:88-113, 506-533

method="eigh": points with 0 < nobsl < k-1 use the observation-space form of
the same transform (N = alpha I + Z Z^T), because A then has a repeated
eigenvalue (k-1)/rho whose eigh gradient is undefined; N's eigenvalues are
distinct.  Near-repeated eigenvalues (rank-deficient local Y, common with
smooth fields and k = 50) still make the eigh gradient overflow, so
method="ns" computes A^-1/2 with the coupled Newton-Schulz iteration
(Higham, Functions of Matrices, 2008, eq. 6.35) on A / tr(A), run to FP64
convergence, and wvec with torch.linalg.solve: both differentiate stably.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from oracle import letkf_oracle as O


class Selection:
    """Per-point local observation sets (input obs indices, distances, dlev)."""

    def __init__(self, p, grid: dict, obs: dict):
        g = {k: np.asarray(v, np.float64) for k, v in grid.items()}
        self.nij1 = g["lon1"].size
        so = O.sort_obs(obs, p.nlon, p.nlat)
        self.pts = {}
        for i in range(self.nij1):
            cand, dist = O.column_candidates(p, g, so, i)
            for k in range(p.nlev):
                sel, _, _, _, _, d, dl = O.obs_local(p, so, cand, dist, k, g["depth1"][k, i])
                self.pts[(k, i)] = (so.perm[sel], d, dl)


NS_ITERS = 60


def _inv_sqrt_ns(A):
    """A^-1/2 of an SPD matrix by the coupled Newton-Schulz iteration."""
    k = A.shape[0]
    eye = torch.eye(k, dtype=torch.float64)
    c = torch.trace(A)
    Y, Z = A / c, eye
    for _ in range(NS_ITERS):
        T = 0.5 * (3.0 * eye - Z @ Y)
        Y, Z = Y @ T, T @ Z
    return Z / torch.sqrt(c)


def _transform(Y, w, d, k, rho, method="eigh"):
    """(wvec, W) of one point; Y [n, k]."""
    n = Y.shape[0]
    alpha = (k - 1) / rho
    if n == 0:
        return torch.zeros(k, dtype=torch.float64), torch.eye(k, dtype=torch.float64) * torch.sqrt(rho)
    if method == "ns":
        A = Y.T @ (w[:, None] * Y) + alpha * torch.eye(k, dtype=torch.float64)
        wvec = torch.linalg.solve(A, Y.T @ (w * d))
        return wvec, math.sqrt(k - 1) * _inv_sqrt_ns(A)
    if n >= k - 1:
        A = Y.T @ (w[:, None] * Y) + alpha * torch.eye(k, dtype=torch.float64)
        lam, V = torch.linalg.eigh(A)
        pa = (V / lam[None, :]) @ V.T
        wvec = pa @ (Y.T @ (w * d))
        W = (V * torch.sqrt((k - 1) / lam)[None, :]) @ V.T
        return wvec, W
    sw = torch.sqrt(w)
    Z = sw[:, None] * Y
    N = Z @ Z.T + alpha * torch.eye(n, dtype=torch.float64)
    lam, Q = torch.linalg.eigh(N)
    wvec = Z.T @ (Q @ ((Q.T @ (sw * d)) / lam))
    g = -1.0 / (torch.sqrt(alpha * lam) * (torch.sqrt(lam) + torch.sqrt(alpha)))
    ZQ = Z.T @ Q
    W = math.sqrt(k - 1) * (torch.eye(k, dtype=torch.float64) / torch.sqrt(alpha) + (ZQ * g[None, :]) @ ZQ.T)
    return wvec, W


def _update(p, x, wvec, W):
    """x [k, nv] -> analysis [k, nv] with RTPP / RTPS (common_da.f90:88-113)."""
    k = x.shape[0]
    fm = x.mean(0)
    dxf = x - fm
    fs = torch.sqrt((dxf * dxf).sum(0) / (k - 1))
    anal = fm[None, :] + (wvec[:, None] + W).T @ dxf
    am = anal.mean(0)
    dxa = anal - am
    asp = torch.sqrt((dxa * dxa).sum(0) / (k - 1))
    if p.alpha_rtpp > 0.0:
        anal = am[None, :] + p.alpha_rtpp * dxf + (1.0 - p.alpha_rtpp) * dxa
    if p.alpha_rtps > 0.0:
        fac = p.alpha_rtps * fs / asp + (1.0 - p.alpha_rtps)
        anal = am[None, :] + dxa * fac[None, :]
    return anal


def analysis(p, sel: Selection, grid: dict, obs: dict, fcst3d, fcst2d, dep, rdiag, rho, sigma, method="eigh"):
    """anal3d [nv3d][k][nlev][nij1], anal2d [nv2d][k][nij1] as differentiable
    FP64 tensors of dep [nobs], rdiag [nobs], rho and sigma (0-dim)."""
    k = p.nmem
    f3 = torch.as_tensor(np.asarray(fcst3d), dtype=torch.float64)
    f2 = torch.as_tensor(np.asarray(fcst2d), dtype=torch.float64)
    hd = torch.as_tensor(np.asarray(obs["hdxf"], np.float64).T.copy())  # [nobs, k]
    phi = np.asarray(grid["phi1"], np.float64)
    a3 = [[[None] * sel.nij1 for _ in range(p.nlev)] for _ in range(p.nv3d)]
    a2 = [[None] * sel.nij1 for _ in range(p.nv2d)]
    for (kl, i), (idx, d, dl) in sel.pts.items():
        it = torch.as_tensor(idx, dtype=torch.long)
        dd = torch.as_tensor(d)
        q = (dd / sigma) ** 2
        if p.sigma_obsv > 0.0:
            q = q + torch.as_tensor((dl / p.sigma_obsv) ** 2)
        rloc = torch.exp(-0.5 * q)
        w = rloc / rdiag[it]
        wvec, W = _transform(hd[it], w, dep[it], k, rho, method)
        an = _update(p, f3[:, :, kl, i].T, wvec, W)          # [k, nv3d]
        if p.roff and kl >= 1 and phi[i] != 1.0:
            cols = []
            for v in range(p.nv3d):
                c = an[:, v]
                if v == p.iv3d_t:
                    c = torch.clamp(c, p.tmin, p.tmax)
                if v == p.iv3d_s:
                    c = torch.clamp(c, p.smin, p.smax)
                cols.append(c)
            an = torch.stack(cols, 1)
        for v in range(p.nv3d):
            a3[v][kl][i] = an[:, v]
        if kl == p.nlev - 1 and p.nv2d > 0:
            an2 = _update(p, f2[:, :, i].T, wvec, W)
            for v in range(p.nv2d):
                a2[v][i] = an2[:, v]
    A3 = torch.stack([torch.stack([torch.stack(a3[v][kl], 1) for kl in range(p.nlev)], 1)
                      for v in range(p.nv3d)], 0)                       # [nv3d][k][nlev][nij1]
    A2 = torch.stack([torch.stack(a2[v], 1) for v in range(p.nv2d)], 0) if p.nv2d else f2.clone()
    return A3, A2


def mean_cost(a3, a2, t3, t2):
    """J = sum over variables and points of (ensemble mean - truth)^2."""
    return ((a3.mean(1) - t3) ** 2).sum() + ((a2.mean(1) - t2) ** 2).sum()
