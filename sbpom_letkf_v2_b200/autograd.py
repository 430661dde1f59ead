"""Differentiable analysis step.

``LETKFFunction`` wraps ``sbletkf_analysis`` (forward) and ``sbletkf_backward``
(the vector-Jacobian product) as a ``torch.autograd.Function``: the analysis
ensemble is differentiable with respect to the observation departures
``dep``, the observation error variances ``rdiag`` (= err**2,
letkf/run/src/common_da.f90:280), the multiplicative inflation
``cov_infl_mul`` (rho, common_letkf.f90:124-126) and the horizontal
localization scale ``sigma_obs`` (common_da.f90:283-287).  The cutoff
``dist_zero`` stays at its value in the given parameters, so the local
observation sets are fixed and the map is smooth.  The reference has no
gradient; this is a new capability of the same analysis.
"""
from __future__ import annotations

import torch

from .analysis import Analysis
from .params import LETKFParams


class LETKFFunction(torch.autograd.Function):
    """(dep, rdiag, cov_infl_mul, sigma_obs) -> (anal3d, anal2d)."""

    @staticmethod
    def forward(ctx, dep, rdiag, cov_infl_mul, sigma_obs, analysis: Analysis, obs: dict, grid: dict,
                fcst3d, fcst2d, params: LETKFParams):
        if params.iswitch_da != 1:
            raise ValueError("LETKFFunction differentiates the LETKF analysis (iswitch_da = 1)")
        p = params.replace(cov_infl_mul=float(cov_infl_mul), sigma_obs=float(sigma_obs),
                           dist_zero=params.dist_zero)
        o = dict(obs)
        o["dep"] = dep.detach().to(torch.float64)
        o["err"] = torch.sqrt(rdiag.detach().to(torch.float64))
        analysis.prepare_obs(o, params=p)
        a3, a2 = analysis.da_main(grid, fcst3d, fcst2d, params=p)
        ctx.state = (analysis, o, grid, fcst3d, fcst2d, p)
        ctx.like = tuple(t if isinstance(t, torch.Tensor) else None
                         for t in (dep, rdiag, cov_infl_mul, sigma_obs))
        return a3, a2

    @staticmethod
    def backward(ctx, g3, g2):
        analysis, o, grid, f3, f2, p = ctx.state
        g3 = torch.zeros_like(f3) if g3 is None else g3.to(f3.dtype)
        g2 = torch.zeros_like(f2) if g2 is None else g2.to(f2.dtype)
        analysis.prepare_obs(o, params=p)  # the workspace may have served other calls since
        grads = analysis.backward(grid, f3, f2, g3, g2, params=p)
        out = tuple(None if t is None else g.reshape(t.shape).to(t.device, t.dtype)
                    for g, t in zip(grads, ctx.like))
        return out + (None,) * 6


def letkf_analysis(analysis: Analysis, obs: dict, grid: dict, fcst3d, fcst2d, params: LETKFParams,
                   dep=None, rdiag=None, cov_infl_mul=None, sigma_obs=None):
    """Differentiable ``da_main``: any of dep, rdiag (err**2), cov_infl_mul,
    sigma_obs given as tensors with requires_grad receive gradients.  Missing
    ones are taken from ``obs`` / ``params``."""
    dev = analysis.device
    dep = obs["dep"].to(dev, torch.float64) if dep is None else dep
    rdiag = (obs["err"].to(dev, torch.float64) ** 2) if rdiag is None else rdiag
    rho = torch.tensor(params.cov_infl_mul, dtype=torch.float64) if cov_infl_mul is None else cov_infl_mul
    sig = torch.tensor(params.sigma_obs, dtype=torch.float64) if sigma_obs is None else sigma_obs
    return LETKFFunction.apply(dep, rdiag, rho, sig, analysis, obs, grid, fcst3d, fcst2d, params)
