// obs_prep.cu -- observation bucketing (letkf/run/src/common_obs.f90:266-377).
//
// The reference sorts the observations by latitude row (idy), then by
// longitude cell (idx), keeping the input order inside a cell, and records
// the cumulative count nobsgrd(i,j).  Here: a counting sort by cell key with
// a per-cell stable fix-up, an exclusive scan giving cellstart[] (so
// nobsgrd(i,j) = cellstart[(j-1)*nlon + i]), and one gather that writes the
// sorted obs arrays and the hdxf rows ([nobs][ldh], zero padded) in FP64 and
// FP32.
#include "internal.cuh"

namespace sbl {
namespace {

__global__ void k_obs_key(int nobs, const int32_t *__restrict__ idx, const int32_t *__restrict__ idy, int nlon,
                          int nlat, int32_t *__restrict__ key, int32_t *__restrict__ cnt, int *status) {
  int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= nobs) return;
  int x = idx[o], y = idy[o];
  if (x < 1 || x > nlon - 1 || y < 1 || y > nlat - 1) {
    key[o] = -1;
    atomicOr(status, SBLETKF_ERR_OBS_CELL);
    return;
  }
  int kk = (y - 1) * nlon + (x - 1);
  key[o] = kk;
  atomicAdd(&cnt[kk], 1);
}

// Exclusive scan of n counts into start[0..n], one CTA of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan(int n, const int32_t *__restrict__ cnt, int32_t *__restrict__ start) {
  __shared__ int ws[40];
  const int per = (n + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * per, e = min(n, b + per);
  int s = 0;
  for (int t = b; t < e; ++t) s += cnt[t];
  int excl;
  int total = block_excl_scan(s, excl, ws);
  for (int t = b; t < e; ++t) {
    start[t] = excl;
    excl += cnt[t];
  }
  if (threadIdx.x == 0) start[n] = total;
}

__global__ void k_scatter(int nobs, const int32_t *__restrict__ key, const int32_t *__restrict__ start,
                          int32_t *__restrict__ fill, int32_t *__restrict__ out) {
  int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= nobs) return;
  int kk = key[o];
  if (kk < 0) return;
  int pos = start[kk] + atomicAdd(&fill[kk], 1);
  out[pos] = o;
}

// Restores input order inside each cell (the reference's sort is stable).
__global__ void k_cell_sort(int ncell, const int32_t *__restrict__ start, int32_t *__restrict__ perm) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  int b = start[c], e = start[c + 1];
  for (int t = b + 1; t < e; ++t) {
    int v = perm[t], u = t - 1;
    while (u >= b && perm[u] > v) {
      perm[u + 1] = perm[u];
      --u;
    }
    perm[u + 1] = v;
  }
}

template <typename HT>
__global__ void k_gather(int nobs, int nmem, int ldh, const int32_t *__restrict__ nvalid,
                         const int32_t *__restrict__ perm, const int32_t *__restrict__ elm,
                         const double *__restrict__ lon, const double *__restrict__ lat,
                         const double *__restrict__ lev, const double *__restrict__ err,
                         const double *__restrict__ dep, const HT *__restrict__ hdxf, int32_t *__restrict__ s_elm,
                         double *__restrict__ s_lon, double *__restrict__ s_lat, double *__restrict__ s_lev,
                         double *__restrict__ s_rdiag, double *__restrict__ s_dep, double *__restrict__ h64,
                         float *__restrict__ h32, int *__restrict__ status) {
  const int lane = threadIdx.x & 31;
  const long long s = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (s >= nobs) return;
  double *row64 = h64 + s * ldh;
  float *row32 = h32 + s * ldh;
  if (s >= *nvalid) {  // positions of rejected obs: zero rows
    for (int m = lane; m < ldh; m += 32) {
      row64[m] = 0.0;
      row32[m] = 0.0f;
    }
    return;
  }
  const int o = perm[s];
  if (lane == 0) {
    s_elm[s] = elm[o];
    s_lon[s] = lon[o];
    s_lat[s] = lat[o];
    s_lev[s] = lev[o];
    s_rdiag[s] = err[o] * err[o];  // rdiag = obserr**2 (common_da.f90:280)
    s_dep[s] = dep[o];
    // an observation the analysis cannot use: non-finite values or err <= 0
    // (rdiag divides the localization weight, common_da.f90:280-287)
    if (!isfinite(lon[o]) || !isfinite(lat[o]) || !isfinite(lev[o]) || !isfinite(dep[o]) || !(err[o] > 0.0) ||
        !isfinite(err[o]))
      atomicOr(status, SBLETKF_ERR_NONFINITE);
  }
  bool bad = false;
  for (int m = lane; m < ldh; m += 32) {
    double v = m < nmem ? (double)hdxf[(long long)m * nobs + o] : 0.0;
    bad |= !isfinite(v);
    row64[m] = v;
    row32[m] = (float)v;
  }
  if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(status, SBLETKF_ERR_NONFINITE);
}

}  // namespace

int launch_prepare_obs(sbletkf_workspace *ws, const sbletkf_params *p, const sbletkf_obs *obs, cudaStream_t s) {
  const int nobs = obs->nobs;
  const int ncell = p->nlon * p->nlat;
  cudaError_t e = cudaMemsetAsync(ws->d_cellcnt, 0, sizeof(int32_t) * ncell, s);
  if (e != cudaSuccess) return cuda_status(e);
  const int tb = 256;
  if (nobs > 0)
    k_obs_key<<<(nobs + tb - 1) / tb, tb, 0, s>>>(nobs, obs->idx, obs->idy, p->nlon, p->nlat, ws->d_tmp,
                                                 ws->d_cellcnt, ws->d_status);
  k_scan<<<1, 1024, 0, s>>>(ncell, ws->d_cellcnt, ws->d_cellstart);
  e = cudaMemsetAsync(ws->d_cellcnt, 0, sizeof(int32_t) * ncell, s);
  if (e != cudaSuccess) return cuda_status(e);
  if (nobs > 0) {
    k_scatter<<<(nobs + tb - 1) / tb, tb, 0, s>>>(nobs, ws->d_tmp, ws->d_cellstart, ws->d_cellcnt, ws->d_perm);
    k_cell_sort<<<(ncell + tb - 1) / tb, tb, 0, s>>>(ncell, ws->d_cellstart, ws->d_perm);
    const int wpb = tb / 32;
    const int nb = (nobs + wpb - 1) / wpb;
    if (obs->hdxf_dtype == SBLETKF_F64)
      k_gather<double><<<nb, tb, 0, s>>>(nobs, p->nmem, ws->ldh, ws->d_cellstart + ncell, ws->d_perm, obs->elm,
                                         obs->lon, obs->lat, obs->lev, obs->err, obs->dep,
                                         (const double *)obs->hdxf, ws->d_elm, ws->d_lon, ws->d_lat, ws->d_lev,
                                         ws->d_rdiag, ws->d_dep, ws->d_hdxf64, ws->d_hdxf32, ws->d_status);
    else
      k_gather<float><<<nb, tb, 0, s>>>(nobs, p->nmem, ws->ldh, ws->d_cellstart + ncell, ws->d_perm, obs->elm,
                                        obs->lon, obs->lat, obs->lev, obs->err, obs->dep,
                                        (const float *)obs->hdxf, ws->d_elm, ws->d_lon, ws->d_lat, ws->d_lev,
                                        ws->d_rdiag, ws->d_dep, ws->d_hdxf64, ws->d_hdxf32, ws->d_status);
  }
  return cuda_status(cudaGetLastError());
}

}  // namespace sbl
