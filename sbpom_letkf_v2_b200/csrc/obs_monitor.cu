// obs_monitor.cu -- observation-space monitors of a forecast or an analysis:
// monit_mean (letkf/run/src/common.f90:681-840) and monit_sprd (:846-978),
// which write_ens_mpi calls on H(mean) and H(spread) of the forecast and of
// the analysis (common_io.f90:1039-1045).
//
// For every observation whose hx is defined (not NaN, the reference's undef),
// the value v = dat - hx (departure, monit_mean) or v = hx (monit_sprd) is
// counted and summed, with its square, under its variable (element id ->
// iv3d_u / iv3d_v / iv3d_t / iv3d_s, SSH -> nv3d + iv2d_z), and for the 3D
// variables also under "surface" (lev == 0) or "interior".  The means and
// RMS values follow on the host.  Block-local sums in shared memory, then
// one set of atomic adds per block.
#include "internal.cuh"

namespace sbl {
namespace {

constexpr int kMonThreads = 256;
constexpr int kMonCells = kNvMax * 3 * 3;  // [variable][all, surface, interior][count, sum, sum of squares]

__global__ void __launch_bounds__(kMonThreads) k_obs_monitor(const sbletkf_params p, int nobs,
                                                             const int32_t *__restrict__ elm,
                                                             const double *__restrict__ lev,
                                                             const double *__restrict__ dat,
                                                             const double *__restrict__ hx, int mode,
                                                             double *__restrict__ stats) {
  __shared__ double acc[kMonCells];
  for (int c = threadIdx.x; c < kMonCells; c += blockDim.x) acc[c] = 0.0;
  __syncthreads();
  const int nvt = p.nv3d + p.nv2d;
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < nobs; o += gridDim.x * blockDim.x) {
    const double h = hx[o];
    if (isnan(h)) continue;  // undef (common.f90:724, 878)
    const int e = elm[o];
    int ivd = -1;
    if (e == p.id_z_obs) ivd = p.nv3d + p.iv2d_z;
    else if (e == 2819) ivd = p.iv3d_u;
    else if (e == 2820) ivd = p.iv3d_v;
    else if (e == 3073) ivd = p.iv3d_t;
    else if (e == 3332) ivd = p.iv3d_s;
    if (ivd < 0 || ivd >= nvt) continue;
    const double v = mode == SBLETKF_MONIT_DEPARTURE ? dat[o] - h : h;
    const double v2 = v * v;
    double *a = acc + ivd * 9;
    atomicAdd(a, 1.0);
    atomicAdd(a + 1, v);
    atomicAdd(a + 2, v2);
    if (e == p.id_z_obs) continue;  // 2D: no surface / interior split
    double *b = a + (lev[o] == 0.0 ? 3 : 6);
    atomicAdd(b, 1.0);
    atomicAdd(b + 1, v);
    atomicAdd(b + 2, v2);
  }
  __syncthreads();
  for (int c = threadIdx.x; c < nvt * 9; c += blockDim.x)
    if (acc[c] != 0.0) atomicAdd(stats + c, acc[c]);
}

}  // namespace

int launch_obs_monitor(const sbletkf_params *p, int nobs, const int32_t *elm, const double *lev, const double *dat,
                       const double *hx, int mode, double *stats, cudaStream_t s) {
  if (nobs == 0) return SBLETKF_OK;
  const int blocks = (nobs + kMonThreads - 1) / kMonThreads;
  k_obs_monitor<<<blocks < 1184 ? blocks : 1184, kMonThreads, 0, s>>>(*p, nobs, elm, lev, dat, hx, mode, stats);
  return cuda_status(cudaGetLastError());
}

}  // namespace sbl

extern "C" int sbletkf_obs_monitor(const sbletkf_params *p, int32_t nobs, const int32_t *elm, const double *lev,
                                   const double *dat, const double *hx, int32_t mode, double *stats, void *stream) {
  if (!p || nobs < 0 || !stats) return SBLETKF_ERR_ARG;
  if (p->nv3d < 0 || p->nv2d < 0 || p->nv3d + p->nv2d > sbl::kNvMax) return SBLETKF_ERR_ARG;
  if (mode != SBLETKF_MONIT_DEPARTURE && mode != SBLETKF_MONIT_VALUE) return SBLETKF_ERR_ARG;
  if (nobs > 0 && (!elm || !lev || !hx || (mode == SBLETKF_MONIT_DEPARTURE && !dat))) return SBLETKF_ERR_ARG;
  return sbl::launch_obs_monitor(p, nobs, elm, lev, dat, hx, mode, stats, static_cast<cudaStream_t>(stream));
}
