"""CPU restatement of the observation-space preprocessing (set_obs).

TEST INFRASTRUCTURE ONLY: the checker of sbletkf_obs_operator.  Parity
unpinned (the reference has no tests for this path either).  Follows

  obs_id_uniform          letkf/run/src/common.f90:112-168
  bilinear_interpolation  common.f90:246-269
  akima_spline            common.f90:276-385
  Trans_XtoY              common.f90:391-500
  set_obs                 common_obs.f90:24-265 and 380-399 (mean, spread,
                          dYf, innovation, gross-error QC, AOEI)

Arrays use the library's layouts: global grid arrays [nlat*nlon] with the
longitude index fastest (column c = (j-1)*nlon + (i-1)), depth [nlev][ncol]
with level 0 the dummy bottom layer and nlev-1 the surface, state
[nv3d][nmem][nlev][ncol] and [nv2d][nmem][ncol].  `None` marks the
reference's undef.

One deviation, documented: akima_spline with the target exactly on the top
grid point falls out of its search loop and then reads past the array
(common.f90:306-343 with i = ndim+1); here that case returns y(ndim), the
value the loop had already assigned.
"""
from __future__ import annotations

import math

import numpy as np

UNDEF = None


def obs_id_uniform(lono, lato, glon, glat, nlon, nlat):
    """Cell indices (1-based; 0 when outside) from the first grid row / column."""
    lon_row = glon[:nlon]                      # lon(:,1)
    lat_col = glat[::nlon][:nlat]              # lat(1,:)
    idx = np.zeros(len(lono), np.int32)
    idy = np.zeros(len(lono), np.int32)
    for o in range(len(lono)):
        for j in range(1, nlat):
            lo, hi = min(lat_col[j - 1], lat_col[j]), max(lat_col[j - 1], lat_col[j])
            if lato[o] < lo or hi <= lato[o]:
                continue
            idy[o] = j
            break
        for i in range(1, nlon):
            lo, hi = min(lon_row[i - 1], lon_row[i]), max(lon_row[i - 1], lon_row[i])
            if lono[o] < lo or hi <= lono[o]:
                continue
            idx[o] = i
            break
    return idx, idy


def bilinear(x0, x1, y0, y1, x, y, f00, f10, f01, f11):
    if x0 == x1 or y0 == y1:
        return UNDEF
    return ((y1 - y) / (y1 - y0) * ((x1 - x) / (x1 - x0) * f00 + (x - x0) / (x1 - x0) * f10)
            + (y - y0) / (y1 - y0) * ((x1 - x) / (x1 - x0) * f01 + (x - x0) / (x1 - x0) * f11))


def akima(x, y, x5):
    """Akima (1970) spline value at x5 of the points (x[0..ndim-1], y)."""
    ndim = len(x)
    if x5 < x[0] or x[ndim - 1] < x5:
        return UNDEF
    i = None
    y5 = UNDEF
    for ii in range(1, ndim + 1):                      # Fortran i = 1..ndim
        if x5 == x[ii - 1]:
            y5 = y[ii - 1]
            continue
        if x5 < x[ii - 1]:
            i = ii
            break
    if i is None:                                      # x5 == x(ndim): see module docstring
        return y5
    X = lambda k: x[k - 1]
    Y = lambda k: y[k - 1]
    d = [0.0] * 6                                      # dydx(1..5)

    def slope(m):
        return (Y(i - 3 + m) - Y(i - 4 + m)) / (X(i - 3 + m) - X(i - 4 + m))
    if i == 2:
        for m in range(3, 6):
            d[m] = slope(m)
        d[2] = 2.0 * d[3] - d[4]
        d[1] = 2.0 * d[2] - d[3]
    elif i == 3:
        for m in range(2, 6):
            d[m] = slope(m)
        d[1] = 2.0 * d[2] - d[3]
    elif i == ndim:
        for m in range(1, 4):
            d[m] = slope(m)
        d[4] = 2.0 * d[3] - d[2]
        d[5] = 2.0 * d[4] - d[3]
    elif i == ndim - 1:
        for m in range(1, 5):
            d[m] = slope(m)
        d[5] = 2.0 * d[4] - d[3]
    else:
        for m in range(1, 6):
            d[m] = slope(m)
    dd = [0.0] + [abs(d[m + 1] - d[m]) for m in range(1, 5)]
    t = [0.0, 0.0, 0.0]
    for m in (1, 2):
        wk = dd[m + 2] + dd[m]
        t[m] = 0.0 if wk == 0 else (dd[m + 2] * d[m + 1] + dd[m] * d[m + 2]) / wk
    dx21 = X(i) - X(i - 1)
    dx = x5 - X(i - 1)
    return (Y(i - 1) + dx * t[1] + dx * dx * (3.0 * d[3] - 2.0 * t[1] - t[2]) / dx21
            + dx * dx * dx * (t[1] + t[2] - 2.0 * d[3]) / dx21 / dx21)


def trans_xtoy(p, g, obs, idx, idy, s3, s2, m):
    """H(x) of member m for every observation (None = undef)."""
    nlon, nlat, nlev = p.nlon, p.nlat, p.nlev
    vmap = {2819: p.iv3d_u, 2820: p.iv3d_v, 3073: p.iv3d_t, 3332: p.iv3d_s}
    out = []
    for o in range(len(obs["elm"])):
        i, j = int(idx[o]), int(idy[o])
        if i < 1 or nlon - 1 < i or j < 1 or nlat - 1 < j:
            out.append(UNDEF)
            continue
        c00, c10, c01, c11 = (j - 1) * nlon + i - 1, (j - 1) * nlon + i, j * nlon + i - 1, j * nlon + i
        if any(g["fsm"][c] == 0.0 for c in (c00, c10, c01, c11)):
            out.append(UNDEF)
            continue
        x0, x1, y0, y1 = g["lon"][c00], g["lon"][c10], g["lat"][c00], g["lat"][c01]
        lo, la, lv = obs["lon"][o], obs["lat"][o], obs["lev"][o]
        e = int(obs["elm"][o])
        if e == p.id_z_obs:
            f = [s2[p.iv2d_z, m, c] for c in (c00, c10, c01, c11)]
            out.append(bilinear(x0, x1, y0, y1, lo, la, *f))
            continue
        if e not in vmap:
            out.append(UNDEF)
            continue
        v = vmap[e]
        dep = g["depth"]
        cs = (c00, c10, c01, c11)
        if 0.0 < lv:
            out.append(UNDEF)
        elif any(lv < dep[1, c] for c in cs):
            out.append(UNDEF)
        elif any(dep[nlev - 1, c] < lv for c in cs):
            f = [s3[v, m, nlev - 1, c] for c in cs]
            out.append(bilinear(x0, x1, y0, y1, lo, la, *f))
        else:
            f = [akima(dep[1:, c], s3[v, m, 1:, c], lv) for c in cs]
            out.append(UNDEF if any(a is UNDEF for a in f) else bilinear(x0, x1, y0, y1, lo, la, *f))
    return out


GROSS = {"z": (-1.0, 1.0), "t": (-5.0, 5.0), "s": (-2.0, 2.0), "u": (-2.0, 2.0), "v": (-2.0, 2.0)}


def set_obs(p, g, obs, s3, s2, gross_qc=False, aoei=True):
    """idx, idy, qc, hxmean, hxsprd, hdxf [nmem][nobs], dep, err (FP64, NaN
    where undef) for the raw observations obs{elm, lon, lat, lev, dat, err}.
    gross_qc / aoei are the reference's LGE_IO / AOEI switches (defaults
    .false. / .true., common_setting.f90:103-108); the gross-error check
    runs only with AOEI off, as in common_obs.f90:186."""
    nobs, k = len(obs["elm"]), p.nmem
    idx, idy = obs_id_uniform(obs["lon"], obs["lat"], g["lon"], g["lat"], p.nlon, p.nlat)
    hx = np.full((k, nobs), np.nan)
    qc = np.ones(nobs, np.int32)
    for m in range(k):
        h = trans_xtoy(p, g, obs, idx, idy, s3, s2, m)
        for o in range(nobs):
            if h[o] is UNDEF:
                qc[o] = 0
            else:
                hx[m, o] = h[o]
    mean = np.full(nobs, np.nan)
    sprd = np.full(nobs, np.nan)
    hdxf = np.full((k, nobs), np.nan)
    dep = np.full(nobs, np.nan)
    err = np.asarray(obs["err"], np.float64).copy()
    for o in range(nobs):
        if qc[o] != 1:
            continue
        mean[o] = hx[:, o].sum() / k
        sprd[o] = math.sqrt(((hx[:, o] - mean[o]) ** 2).sum() / (k - 1))
        hdxf[:, o] = hx[:, o] - mean[o]
        dep[o] = obs["dat"][o] - mean[o]
        if gross_qc and not aoei:                      # LGE_IO .and. .not. AOEI (common_obs.f90:186)
            e = int(obs["elm"][o])
            key = {p.id_z_obs: "z", 3073: "t", 3332: "s", 2819: "u", 2820: "v"}.get(e)
            if key is not None:
                lo, hi = GROSS[key]
                if dep[o] < lo or hi < dep[o]:
                    qc[o] = 0
            elif abs(dep[o]) > 10.0 * err[o]:
                qc[o] = 0
        if aoei and qc[o] == 1:                        # common_obs.f90:385-397
            err[o] = math.sqrt(max(err[o] * err[o], dep[o] * dep[o] - sprd[o] * sprd[o]))
    return dict(idx=idx, idy=idy, qc=qc, hxmean=mean, hxsprd=sprd, hdxf=hdxf, dep=dep, err=err)


def monit_sums(p, obs, hx, departure):
    """monit_mean (common.f90:681-840, departure=True: v = dat - hx) and
    monit_sprd (:846-978, v = hx): for every observation with hx defined
    (not None / NaN), count, sum v and sum v^2 under its variable, and for the
    3D variables under surface (lev == 0) or interior.  Serial, in
    observation order.  Returns [nv3d+nv2d][all, surface, interior][count,
    sum, sum of squares]."""
    nvt = p.nv3d + p.nv2d
    st = np.zeros((nvt, 3, 3))
    vmap = {2819: p.iv3d_u, 2820: p.iv3d_v, 3073: p.iv3d_t, 3332: p.iv3d_s, p.id_z_obs: p.nv3d + p.iv2d_z}
    for o in range(len(obs["elm"])):
        h = hx[o]
        if h is UNDEF or h is None or (isinstance(h, float) and math.isnan(h)):
            continue
        e = int(obs["elm"][o])
        if e not in vmap:
            continue
        ivd = vmap[e]
        v = obs["dat"][o] - h if departure else h
        st[ivd, 0] += (1.0, v, v * v)
        if e == p.id_z_obs:
            continue
        st[ivd, 1 if obs["lev"][o] == 0.0 else 2] += (1.0, v, v * v)
    return st


def hx_of_field(p, g, obs, f3, f2):
    """Trans_XtoY of one state field f3 [nv3d][nlev][ncell], f2 [nv2d][ncell]
    (write_ens_mpi, common_io.f90:967-985): a list with UNDEF where undefined."""
    idx, idy = obs_id_uniform(obs["lon"], obs["lat"], g["lon"], g["lat"], p.nlon, p.nlat)
    return trans_xtoy(p, g, obs, idx, idy, np.asarray(f3)[:, None], np.asarray(f2)[:, None], 0)
