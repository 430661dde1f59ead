"""Seeded synthetic analysis-step inputs for the five benchmark workloads.

The reference reads a sbPOM grid file, a member ensemble and observation files
that are not available here; this module stands in for them with seeded fields
of the same shapes, value ranges and error model:

* grid: regular 0.25 deg lat/lon, ``dx = re cos(lat) dlon``, ``dy = re dlat``
  in metres (as ``grid.nc`` dx/dy, common_pom.f90:81-85), uniform sigma levels
  ``z_e(kk) = -(kk-1)/(nlev-1)`` and ``depth1(i,k) = z_e(nlev-k+1) * h``
  (common_pom.f90:100-106), so k = nlev is the surface and k = 1 the bottom;
  smooth bathymetry 200-5000 m with about 10 % land (h = 1).
* ensemble: smooth background (T 2-28 C, S 33-35 psu, |U|,|V| < 1 m/s,
  SSH +-0.5 m) plus member perturbations with a 150 km Gaussian horizontal
  correlation (FFT-filtered white noise), FP32 storage.
* observations: seeded locations, element ids of common_setting.f90:56-60,
  ``hdxf = H(x_m) - mean_m H(x_m)`` with bilinear horizontal / linear vertical
  interpolation, ``dep = H(truth) + N(0, sigma_o^2) - mean_m H(x_m)`` and the
  observation error std in ``err`` (rdiag = err^2).

All tensors are built with torch on ``device`` so the 4.8M-point workload can
be generated directly in device memory.
"""
from __future__ import annotations

import dataclasses
import math

import torch

from .params import (ID_S_OBS, ID_T_OBS, ID_U_OBS, ID_V_OBS, ID_Z_OBS, DA_LETKF,
                     DA_LPF, RM_SR, LETKFParams)

IV_U, IV_V, IV_T, IV_S = 0, 1, 2, 3      # 3D variable order (common_setting.f90:42-45)
IV_Z = 0                                 # 2D: zeta (:46)
PROFILE_DEPTHS = (10.0, 20.0, 30.0, 50.0, 75.0, 100.0, 150.0, 200.0, 300.0, 500.0)


@dataclasses.dataclass
class Workload:
    """One benchmark workload: grid, ensemble, observation mix and DA options."""

    name: str
    nlon: int
    nlat: int
    nlev: int
    nmem: int
    n_sst: int
    n_ssh: int
    n_prof: int                 # profiles; each has len(PROFILE_DEPTHS) obs
    n_hf: int = 0               # HF-radar surface currents (half U, half V)
    hf_patches: int = 3
    hf_radius_km: float = 100.0
    lon0: float = 120.0
    lat0: float = 10.0
    ddeg: float = 0.25
    sigma_obs: float = 200.0e3
    sigma_obsv: float = 100.0
    cov_infl_mul: float = 1.1
    iswitch_da: int = DA_LETKF
    rm: int = RM_SR
    nmonte: int = 1
    corr_km: float = 150.0
    seed: int = 1000

    @property
    def nobs(self) -> int:
        return self.n_sst + self.n_ssh + self.n_prof * len(PROFILE_DEPTHS) + self.n_hf

    @property
    def npoints(self) -> int:
        return self.nlon * self.nlat * self.nlev

    def params(self, **kw) -> LETKFParams:
        base = dict(nmem=self.nmem, nlon=self.nlon, nlat=self.nlat, nlev=self.nlev,
                    nv3d=4, nv2d=1, iv3d_t=IV_T, iv3d_s=IV_S, iswitch_da=self.iswitch_da,
                    nmonte=self.nmonte, rm=self.rm, dp=True, cov_infl_mul=self.cov_infl_mul,
                    alpha_rtpp=0.0, alpha_rtps=0.0, sigma_obs=self.sigma_obs,
                    sigma_obsv=self.sigma_obsv, roff=True)
        base.update(kw)
        return LETKFParams(**base)

    def scaled(self, **kw) -> "Workload":
        return dataclasses.replace(self, **kw)


# The five workloads.  The 300-row grids start at 30 S so every latitude stays
# below 45 deg and the local search boxes stay near 53 x 53 cells.
WORKLOADS = {
    0: Workload("plain-fp64-small 64x48x12 k=20 3k obs", 64, 48, 12, 20,
                n_sst=2000, n_ssh=800, n_prof=20, seed=1000),
    1: Workload("production 400x300x40 k=100 200k obs", 400, 300, 40, 100,
                n_sst=150_000, n_ssh=45_000, n_prof=500, lat0=-30.0, seed=1001),
    2: Workload("uneven-batching 400x300x40 k=64 300k obs", 400, 300, 40, 64,
                n_sst=120_000, n_ssh=0, n_prof=0, n_hf=180_000, lat0=-30.0, seed=1002),
    3: Workload("differentiation 128x96x20 k=50 20k obs", 128, 96, 20, 50,
                n_sst=13_337, n_ssh=5_333, n_prof=133, seed=1003),
    4: Workload("local-pf 128x96x20 k=128 20k obs", 128, 96, 20, 128,
                n_sst=13_337, n_ssh=5_333, n_prof=133, iswitch_da=DA_LPF, rm=RM_SR,
                nmonte=100, seed=1003),
}

SIGMA_O = {ID_T_OBS: 0.5, ID_Z_OBS: 0.05, "prof_t": 0.3, "prof_s": 0.05, "hf": 0.1}


@dataclasses.dataclass
class Case:
    """Inputs of one analysis call (reference array layouts, see sbletkf.h)."""

    workload: Workload
    params: LETKFParams
    grid: dict          # lon1 lat1 ri1 rj1 dlon1 dlat1 phi1 [nij1] f64, depth1 [nlev][nij1] f64
    obs: dict           # elm idx idy [nobs] i32, lon lat lev err dep [nobs] f64, hdxf [nmem][nobs]
    fcst3d: torch.Tensor  # [nv3d][nmem][nlev][nij1]
    fcst2d: torch.Tensor  # [nv2d][nmem][nij1]
    truth3d: torch.Tensor  # [nv3d][nlev][nij1]
    truth2d: torch.Tensor  # [nv2d][nij1]

    @property
    def nij1(self) -> int:
        return self.workload.nlon * self.workload.nlat

    def to(self, device) -> "Case":
        mv = lambda d: {k: v.to(device) for k, v in d.items()}
        return dataclasses.replace(self, grid=mv(self.grid), obs=mv(self.obs),
                                   fcst3d=self.fcst3d.to(device), fcst2d=self.fcst2d.to(device),
                                   truth3d=self.truth3d.to(device), truth2d=self.truth2d.to(device))

    def numpy(self) -> dict:
        d = {f"grid_{k}": v.cpu().numpy() for k, v in self.grid.items()}
        d.update({f"obs_{k}": v.cpu().numpy() for k, v in self.obs.items()})
        d["fcst3d"] = self.fcst3d.cpu().numpy()
        d["fcst2d"] = self.fcst2d.cpu().numpy()
        return d


def _smooth_fields(n: int, nlat: int, nlon: int, sig_y: float, sig_x: float,
                   gen: torch.Generator, device) -> torch.Tensor:
    """n unit-variance fields with a Gaussian correlation (periodic FFT filter)."""
    out = torch.empty(n, nlat, nlon, dtype=torch.float32, device=device)
    ky = torch.fft.fftfreq(nlat, device=device).view(-1, 1) * 2 * math.pi
    kx = torch.fft.rfftfreq(nlon, device=device).view(1, -1) * 2 * math.pi
    filt = torch.exp(-0.25 * ((ky * sig_y) ** 2 + (kx * sig_x) ** 2))
    chunk = max(1, int(2 ** 26 // (nlat * nlon)))
    for s in range(0, n, chunk):
        e = min(n, s + chunk)
        w = torch.randn(e - s, nlat, nlon, generator=gen, device=device, dtype=torch.float32)
        f = torch.fft.irfft2(torch.fft.rfft2(w) * filt, s=(nlat, nlon))
        f = f - f.mean(dim=(1, 2), keepdim=True)
        out[s:e] = f / f.std(dim=(1, 2), keepdim=True).clamp_min(1e-12)
    return out


def _grid(wl: Workload, gen, device):
    nlon, nlat, nlev = wl.nlon, wl.nlat, wl.nlev
    re, pi = 6371.3e3, 4.0 * math.atan(1.0)
    i1 = torch.arange(1, nlon + 1, device=device, dtype=torch.float64)
    j1 = torch.arange(1, nlat + 1, device=device, dtype=torch.float64)
    jj, ii = torch.meshgrid(j1, i1, indexing="ij")          # [nlat][nlon]
    lon = wl.lon0 + (ii - 1) * wl.ddeg
    lat = wl.lat0 + (jj - 1) * wl.ddeg
    dlon = re * torch.cos(lat * pi / 180.0) * wl.ddeg * pi / 180.0
    dlat = torch.full_like(lat, re * wl.ddeg * pi / 180.0)
    cell_km = re * wl.ddeg * pi / 180.0 / 1e3
    sm = _smooth_fields(2, nlat, nlon, 600.0 / cell_km, 600.0 / cell_km, gen, device).double()
    basin = torch.sigmoid(1.2 * sm[0])
    h = 200.0 + 4800.0 * basin
    land = sm[1] < torch.quantile(sm[1].flatten().float(), 0.10).double()
    h = torch.where(land, torch.ones_like(h), h)
    z_e = -torch.arange(nlev, device=device, dtype=torch.float64) / max(nlev - 1, 1)
    # depth1(i,k) = z_e(nlev-k+1)*h ; 0-based k0 -> z_e index nlev-1-k0
    zk = z_e.flip(0)                                         # [nlev], zk[nlev-1]=0
    depth = zk.view(-1, 1) * h.reshape(1, -1)                # [nlev][nij1]
    g = dict(lon1=lon.reshape(-1), lat1=lat.reshape(-1), ri1=ii.reshape(-1), rj1=jj.reshape(-1),
             dlon1=dlon.reshape(-1), dlat1=dlat.reshape(-1), phi1=h.reshape(-1),
             depth1=depth.contiguous())
    return g, land.reshape(-1)


def _background(wl, g, device):
    """Smooth T, S, U, V [nv3d][nlev][nij1] and SSH [nij1] backgrounds (FP64)."""
    lat = g["lat1"].view(1, -1)
    lon = g["lon1"].view(1, -1)
    z = g["depth1"]
    ph = (lat - wl.lat0) / max(wl.nlat * wl.ddeg, 1e-9)
    pl = (lon - wl.lon0) / max(wl.nlon * wl.ddeg, 1e-9)
    tsurf = 10.0 + 16.0 * torch.cos(lat * math.pi / 180.0 * 1.6).clamp_min(0.0) + 1.5 * torch.sin(6.0 * pl)
    t = 2.0 + (tsurf - 2.0) * torch.exp(z / 700.0)
    s = 34.0 + 0.6 * torch.sin(3.0 * pl + 2.0 * ph) * torch.exp(z / 400.0) - 0.3 * torch.exp(z / 150.0)
    u = 0.6 * torch.sin(2 * math.pi * ph * 2.0) * torch.exp(z / 500.0)
    v = 0.5 * torch.cos(2 * math.pi * pl * 3.0) * torch.exp(z / 500.0)
    ssh = 0.35 * torch.sin(2 * math.pi * (pl + ph)) * torch.cos(math.pi * ph)
    return torch.stack([u, v, t, s]), ssh.view(-1)


def _members(wl, g, nmem, gen, device, bg3, bg2):
    """Background plus correlated perturbations, [nv3d][nmem][nlev][nij1] FP32."""
    nlon, nlat, nlev = wl.nlon, wl.nlat, wl.nlev
    cell_km = 6371.3 * wl.ddeg * math.pi / 180.0
    coslat = math.cos(math.radians(wl.lat0 + 0.5 * nlat * wl.ddeg))
    sy = wl.corr_km / cell_km
    sx = wl.corr_km / (cell_km * max(coslat, 0.2))
    z = g["depth1"].float()                                  # [nlev][nij1]
    h = g["phi1"].float().view(1, -1).clamp_min(1.0)
    sig = (z / h)                                            # [-1,0]
    amp3 = [0.10 * torch.exp(z / 500.0) + 0.02, 0.10 * torch.exp(z / 500.0) + 0.02,
            0.60 * torch.exp(z / 400.0) + 0.10, 0.10 * torch.exp(z / 400.0) + 0.02]
    x3 = torch.empty(4, nmem, nlev, nlon * nlat, dtype=torch.float32, device=device)
    for v in range(4):
        f = _smooth_fields(2 * nmem, nlat, nlon, sy, sx, gen, device).view(nmem, 2, -1)
        for m in range(nmem):
            x3[v, m] = bg3[v].float() + amp3[v] * (f[m, 0].view(1, -1) + 0.5 * f[m, 1].view(1, -1) * (2 * sig + 1))
    f2 = _smooth_fields(nmem, nlat, nlon, sy, sx, gen, device).view(nmem, -1)
    x2 = (bg2.float().view(1, -1) + 0.05 * f2).view(1, nmem, -1)
    return x3, x2


def _interp(field3, field2, g, wl, ox, oy, olev, var3, is_2d):
    """H(x): bilinear horizontal, linear-in-depth vertical, for a batch of members.

    field3 [nmem][nv3d][nlev][nij1] not used directly; field3 is [nv3d][M][nlev][nij1],
    field2 [nv2d][M][nij1].  ox, oy fractional 1-based indices.  Returns [M][nobs] FP64.
    """
    nlon = wl.nlon
    ix = ox.floor().long()
    iy = oy.floor().long()
    fx = (ox - ix).double()
    fy = (oy - iy).double()
    corners = [(0, 0, (1 - fx) * (1 - fy)), (1, 0, fx * (1 - fy)), (0, 1, (1 - fx) * fy), (1, 1, fx * fy)]
    M = field3.shape[1]
    out = torch.zeros(M, ox.numel(), dtype=torch.float64, device=ox.device)
    depth = g["depth1"]
    nlev = depth.shape[0]
    for dx, dy, w in corners:
        col = (iy - 1 + dy) * nlon + (ix - 1 + dx)
        d = depth[:, col]                                    # [nlev][nobs], increasing in k
        lev = olev.clamp(min=d[0])                           # below bottom -> bottom
        # first k with d[k] >= lev
        kk = torch.searchsorted(d.t().contiguous(), lev.view(-1, 1)).view(-1).clamp(1, nlev - 1)
        d0 = d.gather(0, (kk - 1).view(1, -1)).view(-1)
        d1 = d.gather(0, kk.view(1, -1)).view(-1)
        a = torch.where(d1 > d0, (lev - d0) / (d1 - d0), torch.ones_like(lev)).clamp(0, 1)
        vals = torch.zeros(M, ox.numel(), dtype=torch.float64, device=ox.device)
        for v in range(field3.shape[0]):
            sel = (var3 == v) & ~is_2d
            if sel.any():
                c, k0, k1, aa = col[sel], kk[sel] - 1, kk[sel], a[sel]
                f0 = field3[v][:, k0, c].double()
                f1 = field3[v][:, k1, c].double()
                vals[:, sel] = f0 + (f1 - f0) * aa
        if is_2d.any():
            vals[:, is_2d] = field2[IV_Z][:, col[is_2d]].double()
        out += vals * w
    return out


def make_case(wl: Workload | int, device="cpu", seed: int | None = None, **param_kw) -> Case:
    """Build one seeded analysis-call input set for workload ``wl``."""
    if isinstance(wl, int):
        wl = WORKLOADS[wl]
    seed = wl.seed if seed is None else seed
    device = torch.device(device)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    g, land = _grid(wl, gen, device)
    bg3, bg2 = _background(wl, g, device)
    x3, x2 = _members(wl, g, wl.nmem, gen, device, bg3, bg2)
    t3, t2 = _members(wl, g, 1, gen, device, bg3, bg2)
    nlon, nlat = wl.nlon, wl.nlat

    def uni(n):
        return torch.rand(n, generator=gen, device=device, dtype=torch.float64)

    def locs(n):
        return 1.0 + uni(n) * (nlon - 1.0 - 1e-9), 1.0 + uni(n) * (nlat - 1.0 - 1e-9)

    ox, oy, olev, elm, err, var3, is2d = [], [], [], [], [], [], []

    def add(x, y, lv, e, sg, v3, two_d):
        n = x.numel()
        ox.append(x); oy.append(y); olev.append(lv)
        elm.append(torch.full((n,), e, dtype=torch.int32, device=device))
        err.append(torch.full((n,), sg, dtype=torch.float64, device=device))
        var3.append(torch.full((n,), v3, dtype=torch.int64, device=device))
        is2d.append(torch.full((n,), two_d, dtype=torch.bool, device=device))

    if wl.n_sst:
        x, y = locs(wl.n_sst)
        add(x, y, torch.zeros_like(x), ID_T_OBS, SIGMA_O[ID_T_OBS], IV_T, False)
    if wl.n_ssh:
        x, y = locs(wl.n_ssh)
        add(x, y, torch.zeros_like(x), ID_Z_OBS, SIGMA_O[ID_Z_OBS], 0, True)
    if wl.n_prof:
        px, py = locs(wl.n_prof)
        nl = len(PROFILE_DEPTHS)
        x = px.repeat_interleave(nl)
        y = py.repeat_interleave(nl)
        dep_std = torch.tensor(PROFILE_DEPTHS, dtype=torch.float64, device=device).repeat(wl.n_prof)
        col = (y.floor().long() - 1) * nlon + (x.floor().long() - 1)
        hloc = g["phi1"][col].clamp_min(2.0)
        lv = -torch.minimum(dep_std, 0.9 * hloc)
        is_t = (torch.arange(x.numel(), device=device) % 2) == 0
        for sel, e, sg, v3 in ((is_t, ID_T_OBS, SIGMA_O["prof_t"], IV_T),
                               (~is_t, ID_S_OBS, SIGMA_O["prof_s"], IV_S)):
            add(x[sel], y[sel], lv[sel], e, sg, v3, False)
    if wl.n_hf:
        cell_km = 6371.3 * wl.ddeg * math.pi / 180.0
        sea = torch.nonzero(~land).view(-1)
        cidx = sea[torch.randint(0, sea.numel(), (wl.hf_patches,), generator=gen, device=device)]
        cx = (cidx % nlon).double() + 1.0
        cy = (cidx // nlon).double() + 1.0
        per = [wl.n_hf // wl.hf_patches + (1 if p < wl.n_hf % wl.hf_patches else 0) for p in range(wl.hf_patches)]
        for p in range(wl.hf_patches):
            n = per[p]
            r = wl.hf_radius_km / cell_km * torch.sqrt(uni(n))
            th = 2 * math.pi * uni(n)
            x = (cx[p] + r * torch.cos(th)).clamp(1.0, nlon - 1e-6)
            y = (cy[p] + r * torch.sin(th)).clamp(1.0, nlat - 1e-6)
            half = torch.arange(n, device=device) % 2 == 0
            add(x[half], y[half], torch.zeros(int(half.sum()), dtype=torch.float64, device=device),
                ID_U_OBS, SIGMA_O["hf"], IV_U, False)
            add(x[~half], y[~half], torch.zeros(int((~half).sum()), dtype=torch.float64, device=device),
                ID_V_OBS, SIGMA_O["hf"], IV_V, False)

    ox, oy, olev = torch.cat(ox), torch.cat(oy), torch.cat(olev)
    elm, err, var3, is2d = torch.cat(elm), torch.cat(err), torch.cat(var3), torch.cat(is2d)
    # shuffle so the input order is unrelated to the cell order
    perm = torch.randperm(ox.numel(), generator=gen, device=device)
    ox, oy, olev, elm, err, var3, is2d = (a[perm] for a in (ox, oy, olev, elm, err, var3, is2d))
    ox = ox.clamp(1.0, nlon - 1e-6)
    oy = oy.clamp(1.0, nlat - 1e-6)

    hx = _interp(x3, x2, g, wl, ox, oy, olev, var3, is2d)          # [nmem][nobs] f64
    ht = _interp(t3, t2, g, wl, ox, oy, olev, var3, is2d)[0]
    hmean = hx.mean(dim=0)
    hdxf = (hx - hmean).float()
    noise = torch.randn(ox.numel(), generator=gen, device=device, dtype=torch.float64) * err
    dep = ht + noise - hmean
    obs = dict(elm=elm, idx=ox.floor().int(), idy=oy.floor().int(),
               lon=wl.lon0 + (ox - 1.0) * wl.ddeg, lat=wl.lat0 + (oy - 1.0) * wl.ddeg,
               lev=olev, err=err, dep=dep, hdxf=hdxf.contiguous())
    params = wl.params(**param_kw)
    return Case(workload=wl, params=params, grid=g, obs=obs, fcst3d=x3, fcst2d=x2,
                truth3d=t3[:, 0].contiguous(), truth2d=t2[:, 0].contiguous())


def pf_uniforms(npoints: int, nmonte: int, nmem: int, rm: int, device="cpu", seed: int = 7) -> torch.Tensor:
    """Seeded resampling uniforms: [P][nmonte] (SR) or [P][nmonte][nmem] (MR)."""
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    shape = (npoints, nmonte) if rm == RM_SR else (npoints, nmonte, nmem)
    return torch.rand(shape, generator=gen, device=device, dtype=torch.float64)
