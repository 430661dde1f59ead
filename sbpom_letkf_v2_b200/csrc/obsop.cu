// obsop.cu -- observation-space preprocessing: the observation operator H(x)
// for every member, the ensemble mean / spread in observation space, dYf,
// the innovation, gross-error QC and AOEI (set_obs, letkf/run/src/
// common_obs.f90:24-265, 380-399; Trans_XtoY, common.f90:391-500).
//
// One warp per observation, lanes over members (k <= 128, 4 per lane).
//  1. cell indices as obs_id_uniform (common.f90:112-168): the first grid
//     row / column band [min, max) holding the location, warp-parallel scan;
//  2. Trans_XtoY: outside the inner cells or a land corner -> undef; SSH by
//     bilinear interpolation of the 2D field; 3D elements undef above the
//     surface or below the bottom of any corner, surface level when above
//     the top level of any corner, otherwise an Akima spline (Akima 1970, as
//     akima_spline, common.f90:276-385) over levels 2..nlev of each corner
//     followed by bilinear interpolation (bilinear_interpolation,
//     common.f90:246-269);
//  3. any undef member -> qc = 0 (read_ens_mpi, common_io.f90:832-838);
//  4. mean, spread (k-1), hdxf = H(x_m) - mean, dep = obs - mean;
//  5. optional gross-error check (LGE_IO, only with AOEI off) and AOEI
//     err = sqrt(max(err^2, dep^2 - sprd^2)) (Minamide & Zhang 2017);
//  6. optional monitor sums of dep per variable over qc = 1 (monit_dep,
//     common.f90:602-675).
// Undef outputs are NaN.  The Akima search that lands exactly on the top
// level returns that level's value (the reference's loop then reads past its
// array).
#include "internal.cuh"

namespace sbl {
namespace {

constexpr int kMemPerLane = 4;  // members per lane (k <= 128)

struct GlobalGrid {
  const double *lon, *lat, *fsm, *depth;  // [nlat*nlon], depth [nlev][nlat*nlon]
};

__device__ __forceinline__ double bilinear(double x0, double x1, double y0, double y1, double x, double y,
                                           double f00, double f10, double f01, double f11) {
  return (y1 - y) / (y1 - y0) * ((x1 - x) / (x1 - x0) * f00 + (x - x0) / (x1 - x0) * f10) +
         (y - y0) / (y1 - y0) * ((x1 - x) / (x1 - x0) * f01 + (x - x0) / (x1 - x0) * f11);
}

// Interval of an Akima evaluation: Fortran index i (2..ndim) with
// x(i-1) <= x5 < x(i), or 0 for "exactly the last point" (value y(ndim)).
// x(q) = depth level q (0-based), q = 1..ndim.
__device__ __forceinline__ int akima_interval(const double *depth, long long ncol, long long c, int ndim, double x5) {
  for (int q = 1; q <= ndim; ++q) {
    const double xq = depth[(long long)q * ncol + c];
    if (x5 == xq) continue;
    if (x5 < xq) return q;
  }
  return 0;
}

template <typename ST>
__device__ __forceinline__ double akima_eval(const double *depth, const ST *yv, long long ncol, long long c,
                                             int ndim, int i, double x5) {
  // X(q) = depth level q, Y(q) = state level q (Fortran points q = 1..ndim)
  auto X = [&](int q) { return depth[(long long)q * ncol + c]; };
  auto Y = [&](int q) { return (double)yv[(long long)q * ncol + c]; };
  if (i == 0) return Y(ndim);
  double d[6];
  auto slope = [&](int m) { return (Y(i - 3 + m) - Y(i - 4 + m)) / (X(i - 3 + m) - X(i - 4 + m)); };
  if (i == 2) {
    for (int m = 3; m <= 5; ++m) d[m] = slope(m);
    d[2] = 2.0 * d[3] - d[4];
    d[1] = 2.0 * d[2] - d[3];
  } else if (i == 3) {
    for (int m = 2; m <= 5; ++m) d[m] = slope(m);
    d[1] = 2.0 * d[2] - d[3];
  } else if (i == ndim) {
    for (int m = 1; m <= 3; ++m) d[m] = slope(m);
    d[4] = 2.0 * d[3] - d[2];
    d[5] = 2.0 * d[4] - d[3];
  } else if (i == ndim - 1) {
    for (int m = 1; m <= 4; ++m) d[m] = slope(m);
    d[5] = 2.0 * d[4] - d[3];
  } else {
    for (int m = 1; m <= 5; ++m) d[m] = slope(m);
  }
  double dd[5];
  for (int m = 1; m <= 4; ++m) dd[m] = fabs(d[m + 1] - d[m]);
  double t[3];
  for (int m = 1; m <= 2; ++m) {
    const double wk = dd[m + 2] + dd[m];
    t[m] = (wk == 0.0) ? 0.0 : (dd[m + 2] * d[m + 1] + dd[m] * d[m + 2]) / wk;
  }
  const double dx21 = X(i) - X(i - 1), dx = x5 - X(i - 1);
  return Y(i - 1) + dx * t[1] + dx * dx * (3.0 * d[3] - 2.0 * t[1] - t[2]) / dx21 +
         dx * dx * dx * (t[1] + t[2] - 2.0 * d[3]) / dx21 / dx21;
}

// First band j in 1..n-1 with min(a[j-1],a[j]) <= x < max(a[j-1],a[j]) (a[q] =
// base[q*stride]), 0 when none: warp-parallel, first match wins.
__device__ __forceinline__ int first_band(const double *base, long long stride, int n, double x) {
  const int lane = threadIdx.x & 31;
  for (int b0 = 1; b0 < n; b0 += 32) {
    const int j = b0 + lane;
    bool hit = false;
    if (j < n) {
      const double a0 = base[(long long)(j - 1) * stride], a1 = base[(long long)j * stride];
      const double lo = fmin(a0, a1), hi = fmax(a0, a1);
      hit = !(x < lo || hi <= x);
    }
    const unsigned m = __ballot_sync(0xffffffffu, hit);
    if (m) return b0 + __ffs(m) - 1;
  }
  return 0;
}

template <typename ST>
__global__ void k_obs_operator(const sbletkf_params p, const GlobalGrid g, const ST *__restrict__ s3,
                               const ST *__restrict__ s2, sbletkf_obs_in ob, int flags, sbletkf_obs_out out,
                               double *__restrict__ stats) {
  const int lane = threadIdx.x & 31;
  const long long o = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (o >= ob.nobs) return;
  const int nlon = p.nlon, nlat = p.nlat, nlev = p.nlev, k = p.nmem;
  const long long ncol = (long long)nlon * nlat;
  const double lono = ob.lon[o], lato = ob.lat[o], levo = ob.lev[o];
  const int elm = ob.elm[o];
  const int ix = first_band(g.lon, 1, nlon, lono);                 // lon(:,1)
  const int iy = first_band(g.lat, nlon, nlat, lato);              // lat(1,:)

  // ---- Trans_XtoY: which branch (the same for every member)
  int branch = 0;  // 0 undef, 1 SSH bilinear, 2 surface bilinear, 3 Akima + bilinear
  int var = -1;
  long long c[4] = {0, 0, 0, 0};
  if (ix >= 1 && ix <= nlon - 1 && iy >= 1 && iy <= nlat - 1) {
    c[0] = (long long)(iy - 1) * nlon + (ix - 1);
    c[1] = c[0] + 1;
    c[2] = c[0] + nlon;
    c[3] = c[2] + 1;
    bool land = false;
    for (int q = 0; q < 4; ++q) land |= g.fsm[c[q]] == 0.0;
    if (!land) {
      if (elm == p.id_z_obs) {
        branch = (p.iv2d_z >= 0 && p.iv2d_z < p.nv2d) ? 1 : 0;
        var = p.iv2d_z;
      } else {
        var = elm == 2819 ? p.iv3d_u : elm == 2820 ? p.iv3d_v : elm == 3073 ? p.iv3d_t : elm == 3332 ? p.iv3d_s : -1;
        if (var >= 0 && var < p.nv3d && !(0.0 < levo)) {
          bool below = false, above = false;
          for (int q = 0; q < 4; ++q) {
            below |= levo < g.depth[1 * ncol + c[q]];
            above |= g.depth[(long long)(nlev - 1) * ncol + c[q]] < levo;
          }
          branch = below ? 0 : above ? 2 : 3;
        }
      }
    }
  }
  const double x0 = branch ? g.lon[c[0]] : 0.0, x1 = branch ? g.lon[c[1]] : 1.0;
  const double y0 = branch ? g.lat[c[0]] : 0.0, y1 = branch ? g.lat[c[2]] : 1.0;
  if (branch && (x0 == x1 || y0 == y1)) branch = 0;  // bilinear_interpolation -> undef
  int ai[4] = {0, 0, 0, 0};
  if (branch == 3)
    for (int q = 0; q < 4; ++q) ai[q] = akima_interval(g.depth, ncol, c[q], nlev - 1, levo);

  // ---- H(x_m), lanes over members
  double hx[kMemPerLane];
  double sum = 0.0;
#pragma unroll
  for (int t = 0; t < kMemPerLane; ++t) {
    const int m = lane + 32 * t;
    hx[t] = 0.0;
    if (m >= k || branch == 0) continue;
    double f[4];
    if (branch == 1) {
      const ST *y = s2 + ((long long)var * k + m) * ncol;
      for (int q = 0; q < 4; ++q) f[q] = (double)y[c[q]];
    } else {
      const ST *y = s3 + ((long long)var * k + m) * nlev * ncol;
      for (int q = 0; q < 4; ++q)
        f[q] = branch == 2 ? (double)y[(long long)(nlev - 1) * ncol + c[q]]
                           : akima_eval(g.depth, y, ncol, c[q], nlev - 1, ai[q], levo);
    }
    hx[t] = bilinear(x0, x1, y0, y1, lono, lato, f[0], f[1], f[2], f[3]);
    sum += hx[t];
  }
  int qc = branch != 0;
  const double nan = __longlong_as_double(0x7ff8000000000000LL);
  double mean = nan, sprd = nan, dep = nan, err = ob.err[o];
  if (qc) {
    mean = warp_sum(sum) / (double)k;
    double q2 = 0.0;
#pragma unroll
    for (int t = 0; t < kMemPerLane; ++t)
      if (lane + 32 * t < k) q2 += (hx[t] - mean) * (hx[t] - mean);
    q2 = warp_sum(q2);
    sprd = k > 1 ? sqrt(q2 / (double)(k - 1)) : nan;
    dep = ob.dat[o] - mean;
    const bool aoei = flags & SBLETKF_OBSOP_AOEI;
    if ((flags & SBLETKF_OBSOP_GROSS_QC) && !aoei) {  // common_obs.f90:186-217
      double lo = 0.0, hi = 0.0;
      bool known = true;
      if (elm == p.id_z_obs) { lo = -1.0; hi = 1.0; }
      else if (elm == 3073) { lo = -5.0; hi = 5.0; }
      else if (elm == 3332 || elm == 2819 || elm == 2820) { lo = -2.0; hi = 2.0; }
      else known = false;
      if (known ? (dep < lo || hi < dep) : fabs(dep) > 10.0 * err) qc = 0;
    }
    if (aoei && qc) err = sqrt(fmax(err * err, dep * dep - sprd * sprd));
  }
#pragma unroll
  for (int t = 0; t < kMemPerLane; ++t) {
    const int m = lane + 32 * t;
    if (m < k && out.hdxf) out.hdxf[(long long)m * ob.nobs + o] = branch ? hx[t] - mean : nan;
  }
  if (lane == 0) {
    if (out.idx) out.idx[o] = ix;
    if (out.idy) out.idy[o] = iy;
    if (out.qc) out.qc[o] = qc;
    if (out.hxmean) out.hxmean[o] = mean;
    if (out.hxsprd) out.hxsprd[o] = sprd;
    if (out.dep) out.dep[o] = dep;
    if (out.err) out.err[o] = err;
    if (stats && qc) {
      const int ivd = elm == p.id_z_obs ? p.nv3d + p.iv2d_z : var;
      if (ivd >= 0 && ivd < p.nv3d + p.nv2d) {
        atomicAdd(stats + 3 * ivd, 1.0);
        atomicAdd(stats + 3 * ivd + 1, dep);
        atomicAdd(stats + 3 * ivd + 2, dep * dep);
      }
    }
  }
}

}  // namespace

int launch_obs_operator(const sbletkf_params *p, const double *glon, const double *glat, const double *gfsm,
                        const double *gdepth, const void *s3, const void *s2, int dtype, const sbletkf_obs_in *obs,
                        int flags, const sbletkf_obs_out *out, double *stats, cudaStream_t s) {
  if (obs->nobs == 0) return SBLETKF_OK;
  const GlobalGrid g{glon, glat, gfsm, gdepth};
  const int wpb = 8;
  const unsigned nb = (unsigned)((obs->nobs + wpb - 1) / wpb);
  if (dtype == SBLETKF_F64)
    k_obs_operator<double><<<nb, 32 * wpb, 0, s>>>(*p, g, (const double *)s3, (const double *)s2, *obs, flags,
                                                   *out, stats);
  else
    k_obs_operator<float><<<nb, 32 * wpb, 0, s>>>(*p, g, (const float *)s3, (const float *)s2, *obs, flags, *out,
                                                  stats);
  return cuda_status(cudaGetLastError());
}

}  // namespace sbl
