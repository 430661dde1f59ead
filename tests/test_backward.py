"""Gradients of the LETKF analysis (sbletkf_backward / LETKFFunction).

References: the FP64 torch restatement differentiated by autograd
(tests/torch_ref.py; through torch.linalg.eigh at k = 12, through a
Newton-Schulz A^-1/2 at k = 50 where near-repeated eigenvalues make the eigh
gradient overflow) and central finite differences with h = 1e-6 (relative) of
the FP64 forward.  Cost J = sum (mean anal - truth)^2.
Tolerances (relative to the largest gradient component of each kind):
  backward vs torch autograd   1e-8
  backward vs central FD       1e-6, plus the FD rounding floor
                               4 k eps |J| / (2h): the forward is accurate to
                               its Jacobi tolerance k eps, and the difference
                               quotient amplifies that by 1/(2h)
"""
import numpy as np
import pytest
import torch

from sbpom_letkf_v2_b200.synthetic import WORKLOADS, make_case
from tests import torch_ref as T

TOL_AD = 1e-8
TOL_FD = 1e-6
H_REL = 1e-6
EPS = 2.220446049250313e-16


def _fd_ok(fd, g, gmax, J, h2, k):
    """h2: the difference quotient's denominator (2h)."""
    return abs(fd - g) <= TOL_FD * gmax + 4.0 * k * EPS * abs(J) / h2


def _case(k=12, seed=901, **kw):
    wl = WORKLOADS[0].scaled(nlon=16, nlat=12, nlev=5, nmem=k, n_sst=30, n_ssh=8, n_prof=8, seed=seed)
    return make_case(wl, cov_infl_mul=1.1, sigma_obs=50e3, **kw)


def _np(case):
    return ({k: v.numpy() for k, v in case.grid.items()}, {k: v.numpy() for k, v in case.obs.items()})


def _torch_grads(case, p=None, method="eigh"):
    p = p or case.params
    g, ob = _np(case)
    sel = T.Selection(p, g, ob)
    dep = torch.tensor(ob["dep"], requires_grad=True)
    rd = torch.tensor(ob["err"] ** 2, requires_grad=True)
    rho = torch.tensor(p.cov_infl_mul, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(p.sigma_obs, dtype=torch.float64, requires_grad=True)
    a3, a2 = T.analysis(p, sel, g, ob, case.fcst3d.numpy(), case.fcst2d.numpy(), dep, rd, rho, sig, method)
    J = T.mean_cost(a3, a2, case.truth3d.double(), case.truth2d.double())
    J.backward()
    return dict(J=float(J.detach()), dep=dep.grad.numpy(), rdiag=rd.grad.numpy(), rho=float(rho.grad),
                sigma=float(sig.grad), a3=a3.detach().numpy(), a2=a2.detach().numpy())


def _rel(a, b):
    a, b = np.atleast_1d(a), np.atleast_1d(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


# ---- CPU: the torch reference itself -------------------------------------

def test_torch_reference_forward_matches_oracle():
    from oracle import letkf_oracle as O
    case = _case(alpha_rtpp=0.5)
    g, ob = _np(case)
    r = _torch_grads(case)
    ref = O.da_main(case.params, g, ob, case.fcst3d.numpy(), case.fcst2d.numpy())
    assert _rel(r["a3"], ref.anal3d) <= 1e-12
    assert _rel(r["a2"], ref.anal2d) <= 1e-12


def test_torch_reference_gradient_vs_fd():
    case = _case()
    p = case.params
    g, ob = _np(case)
    sel = T.Selection(p, g, ob)
    r = _torch_grads(case)

    def J(dep=None, rd=None, rho=None, sig=None):
        dep = torch.tensor(ob["dep"]) if dep is None else dep
        rd = torch.tensor(ob["err"] ** 2) if rd is None else rd
        rho = torch.tensor(p.cov_infl_mul, dtype=torch.float64) if rho is None else rho
        sig = torch.tensor(p.sigma_obs, dtype=torch.float64) if sig is None else sig
        with torch.no_grad():
            a3, a2 = T.analysis(p, sel, g, ob, case.fcst3d.numpy(), case.fcst2d.numpy(), dep, rd, rho, sig)
            return float(T.mean_cost(a3, a2, case.truth3d.double(), case.truth2d.double()))

    h = H_REL * p.cov_infl_mul
    fd = (J(rho=torch.tensor(p.cov_infl_mul + h, dtype=torch.float64))
          - J(rho=torch.tensor(p.cov_infl_mul - h, dtype=torch.float64))) / (2 * h)
    assert _fd_ok(fd, r["rho"], abs(r["rho"]), r["J"], 2 * h, p.nmem)
    h = H_REL * p.sigma_obs
    fd = (J(sig=torch.tensor(p.sigma_obs + h, dtype=torch.float64))
          - J(sig=torch.tensor(p.sigma_obs - h, dtype=torch.float64))) / (2 * h)
    assert _fd_ok(fd, r["sigma"], abs(r["sigma"]), r["J"], 2 * h, p.nmem)
    o = int(np.argmax(np.abs(r["dep"])))
    d0 = torch.tensor(ob["dep"])
    h = H_REL * max(1.0, abs(float(d0[o])))
    dp, dm = d0.clone(), d0.clone()
    dp[o] += h
    dm[o] -= h
    fd = (J(dep=dp) - J(dep=dm)) / (2 * h)
    assert _fd_ok(fd, r["dep"][o], np.abs(r["dep"]).max(), r["J"], 2 * h, p.nmem)


# ---- GPU: sbletkf_backward -------------------------------------------------

def _gpu_grads(case, p=None, dev="cuda:0"):
    from sbpom_letkf_v2_b200.analysis import Analysis
    from sbpom_letkf_v2_b200.autograd import letkf_analysis
    p = p or case.params
    c = case.to(dev)
    an = Analysis(p, c.nij1, c.obs["elm"].numel(), device=dev)
    dep = c.obs["dep"].clone().requires_grad_(True)
    rd = (c.obs["err"] ** 2).clone().requires_grad_(True)
    rho = torch.tensor(p.cov_infl_mul, dtype=torch.float64, requires_grad=True)
    sig = torch.tensor(p.sigma_obs, dtype=torch.float64, requires_grad=True)
    f3, f2 = c.fcst3d.double(), c.fcst2d.double()
    a3, a2 = letkf_analysis(an, c.obs, c.grid, f3, f2, p, dep=dep, rdiag=rd, cov_infl_mul=rho, sigma_obs=sig)
    J = ((a3.mean(1) - c.truth3d.double()) ** 2).sum() + ((a2.mean(1) - c.truth2d.double()) ** 2).sum()
    J.backward()
    out = dict(J=float(J.detach()), dep=dep.grad.cpu().numpy(), rdiag=rd.grad.cpu().numpy(),
               rho=float(rho.grad), sigma=float(sig.grad))

    def Jf(dep_v=None, rd_v=None, rho_v=None, sig_v=None):
        with torch.no_grad():
            b3, b2 = letkf_analysis(an, c.obs, c.grid, f3, f2, p,
                                    dep=c.obs["dep"] if dep_v is None else dep_v,
                                    rdiag=c.obs["err"] ** 2 if rd_v is None else rd_v,
                                    cov_infl_mul=torch.tensor(p.cov_infl_mul if rho_v is None else rho_v,
                                                              dtype=torch.float64),
                                    sigma_obs=torch.tensor(p.sigma_obs if sig_v is None else sig_v,
                                                           dtype=torch.float64))
            return float(((b3.mean(1) - c.truth3d.double()) ** 2).sum() + ((b2.mean(1) - c.truth2d.double()) ** 2).sum())

    out["Jf"] = Jf
    out["obs"] = c.obs
    out["an"] = an
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("relax,k", [("none", 12), ("rtpp", 12), ("rtps", 12), ("rtpp", 50)])
def test_backward_matches_torch_autograd(relax, k, cuda):
    kw = {"none": {}, "rtpp": {"alpha_rtpp": 0.5}, "rtps": {"alpha_rtps": 0.7}}[relax]
    case = _case(k=k, **kw)
    ref = _torch_grads(case, method="eigh" if k <= 12 else "ns")
    got = _gpu_grads(case)
    assert abs(got["J"] - ref["J"]) <= 1e-12 * abs(ref["J"])
    assert _rel(got["dep"], ref["dep"]) <= TOL_AD
    assert _rel(got["rdiag"], ref["rdiag"]) <= TOL_AD
    assert _rel(got["rho"], ref["rho"]) <= TOL_AD
    assert _rel(got["sigma"], ref["sigma"]) <= TOL_AD
    got["an"].close()


@pytest.mark.gpu
@pytest.mark.parametrize("k", [12, 50])
def test_backward_vs_central_fd(k, cuda):
    case = _case(k=k, seed=950 + k)
    p = case.params
    got = _gpu_grads(case)
    Jf, obs, J = got["Jf"], got["obs"], got["J"]
    h = H_REL * p.cov_infl_mul
    fd = (Jf(rho_v=p.cov_infl_mul + h) - Jf(rho_v=p.cov_infl_mul - h)) / (2 * h)
    assert _fd_ok(fd, got["rho"], abs(got["rho"]), J, 2 * h, k), (fd, got["rho"])
    h = H_REL * p.sigma_obs
    fd = (Jf(sig_v=p.sigma_obs + h) - Jf(sig_v=p.sigma_obs - h)) / (2 * h)
    assert _fd_ok(fd, got["sigma"], abs(got["sigma"]), J, 2 * h, k), (fd, got["sigma"])
    for key, base in (("dep", obs["dep"]), ("rdiag", obs["err"] ** 2)):
        g = got[key]
        for o in np.argsort(-np.abs(g))[:3]:
            h = H_REL * max(1e-3, abs(float(base[o])))
            bp, bm = base.clone(), base.clone()
            bp[o] += h
            bm[o] -= h
            if key == "dep":
                fd = (Jf(dep_v=bp) - Jf(dep_v=bm)) / (2 * h)
            else:
                fd = (Jf(rd_v=bp) - Jf(rd_v=bm)) / (2 * h)
            assert _fd_ok(fd, g[o], np.abs(g).max(), J, 2 * h, k), (key, o, fd, g[o])
    got["an"].close()


@pytest.mark.gpu
def test_backward_without_observations_is_zero(cuda):
    from sbpom_letkf_v2_b200.analysis import Analysis
    case = _case().to("cuda:0")
    p = case.params
    empty = {k: v[..., :0] for k, v in case.obs.items()}
    an = Analysis(p, case.nij1, 1, device="cuda:0")
    an.prepare_obs(empty)
    g3 = torch.ones_like(case.fcst3d)
    g2 = torch.ones_like(case.fcst2d)
    gd, gr, gi, gs = an.backward(case.grid, case.fcst3d, case.fcst2d, g3, g2)
    assert gd.numel() == 0 and gr.numel() == 0 and float(gi) == 0.0 and float(gs) == 0.0
    an.close()


@pytest.mark.gpu
def test_backward_rejects_pf_and_large_k(cuda):
    from sbpom_letkf_v2_b200._abi import SBLETKFError
    from sbpom_letkf_v2_b200.analysis import Analysis
    from sbpom_letkf_v2_b200.params import DA_LPF
    for kw, k in (({"iswitch_da": DA_LPF}, 12), ({}, 128)):
        case = _case(k=k, **kw).to("cuda:0")
        an = Analysis(case.params, case.nij1, case.obs["elm"].numel(), device="cuda:0")
        an.prepare_obs(case.obs)
        with pytest.raises(SBLETKFError):
            an.backward(case.grid, case.fcst3d, case.fcst2d, torch.ones_like(case.fcst3d),
                        torch.ones_like(case.fcst2d))
        an.close()
