// internal.cuh -- shared device/host declarations of libsbletkf (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sbletkf.h"

namespace sbl {

constexpr int kNvMax = 8;        // nv3d + nv2d limit
constexpr int kRowMax = 1024;    // grid rows of one local search box
constexpr int kThreads = 256;    // CTA size of the per-point kernels
constexpr int kChunk = 32;       // local obs rows staged per Gram step
constexpr int kDualMax = 64;     // local obs handled by the observation-space transform
constexpr int kListCap = kThreads + 64 + 64;  // streaming step + max(kDualMax, chunk) + chunk

// Sorted observation arrays owned by the workspace (cell order of
// common_obs.f90:266-377).  hdxf rows are padded to ldh with zeros.
struct ObsView {
  int32_t nobs;
  int32_t ldh;                   // row stride of hdxf64 / hdxf32 (elements)
  const int32_t *elm;
  const double *lon, *lat, *lev, *rdiag, *dep;
  const double *hdxf64;          // [nobs][ldh]
  const float *hdxf32;           // [nobs][ldh]
  const int32_t *cellstart;      // [nlon*nlat+1]
  const int32_t *perm;           // sorted position -> caller's index
};

struct GridView {
  int32_t nij1;
  const double *lon1, *lat1, *ri1, *rj1, *dlon1, *dlat1, *phi1, *depth1;
};

__host__ __device__ inline int round_up(int a, int b) { return (a + b - 1) / b * b; }

// Barrier of the kThreads threads (warps 0..7) that analyse one point.  In
// the 256-thread kernels that is the whole CTA (the same as __syncthreads);
// in the warp-specialised analysis kernel it is the consumer warps only, the
// producer warps synchronise on barrier 2.
__device__ __forceinline__ void cta_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kThreads) : "memory"); }

// Fortran NINT: nearest integer, halves away from zero (round() semantics).
__device__ __forceinline__ long long fnint(double x) { return llround(x); }

// distance_2p (letkf/run/src/common.f90:79-101) with the oracle's evaluation
// order and no FMA contraction, so only sin/cos/acos may differ in an ulp.
__device__ __forceinline__ double distance_2p(double lona, double lata, double lonb, double latb,
                                              double pi, double re) {
  double ra = __ddiv_rn(__dmul_rn(pi, lata), 180.0);
  double rb = __ddiv_rn(__dmul_rn(pi, latb), 180.0);
  double rl = __ddiv_rn(__dmul_rn(pi, __dsub_rn(lonb, lona)), 180.0);
  double t1 = __dmul_rn(sin(ra), sin(rb));
  double t2 = __dmul_rn(__dmul_rn(cos(ra), cos(rb)), cos(rl));
  double c = __dadd_rn(t1, t2);
  c = fmin(1.0, c);
  c = fmax(-1.0, c);
  return __dmul_rn(re, acos(c));
}

// Localization weight (common_da.f90:283-287).
__device__ __forceinline__ double loc_weight(double dist, double dlev, double so, double sv) {
  double q = __ddiv_rn(dist, so);
  q = __dmul_rn(q, q);
  if (sv > 0.0) {
    double r = __ddiv_rn(dlev, sv);
    q = __dadd_rn(q, __dmul_rn(r, r));
  }
  return exp(__dmul_rn(-0.5, q));
}

// dlev rule of count_nobsl / obs_local (common_da.f90:176-184).
__device__ __forceinline__ double dlev_of(int elm, double olev, double rdep, int k, int nlev, int id_z) {
  if (elm == id_z) return (k < nlev - 1) ? fabs(rdep) : 0.0;
  return fabs(__dsub_rn(olev, rdep));
}

// Search box of point i (common_da.f90:158-161).
__device__ __forceinline__ void search_box(const sbletkf_params &p, const GridView &g, int i, int &imin,
                                           int &imax, int &jmin, int &jmax) {
  double dz = p.dist_zero;
  long long a = fnint(__dsub_rn(g.ri1[i], __ddiv_rn(dz, g.dlon1[i])));
  long long b = fnint(__dadd_rn(g.ri1[i], __ddiv_rn(dz, g.dlon1[i])));
  long long c = fnint(__dsub_rn(g.rj1[i], __ddiv_rn(dz, g.dlat1[i])));
  long long d = fnint(__dadd_rn(g.rj1[i], __ddiv_rn(dz, g.dlat1[i])));
  imin = (int)(a > 1 ? (a < p.nlon ? a : p.nlon) : 1);
  imax = (int)(b < p.nlon ? (b > 1 ? b : 1) : p.nlon);
  jmin = (int)(c > 1 ? (c < p.nlat ? c : p.nlat) : 1);
  jmax = (int)(d < p.nlat ? (d > 1 ? d : 1) : p.nlat);
  // every index is now inside the grid; an empty box has imin > imax or jmin > jmax
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ int warp_incl_scan(int v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one int per thread; returns the block total.
// `ws` is shared scratch of >= nwarps+1 ints.
__device__ __forceinline__ int block_excl_scan(int v, int &excl, int *ws) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int inc = warp_incl_scan(v);
  if (lane == 31) ws[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int t = lane < nw ? ws[lane] : 0;
    int ti = warp_incl_scan(t);
    if (lane < nw) ws[lane] = ti - t;
    if (lane == nw - 1) ws[nw] = ti;
  }
  __syncthreads();
  excl = ws[wid] + inc - v;
  int total = ws[nw];
  __syncthreads();
  return total;
}

__device__ __forceinline__ void latch(int *status, int32_t *point_status, long long pid, int bits) {
  if (bits) {
    atomicOr(status, bits);
    if (point_status) atomicOr(&point_status[pid], bits);
  }
}

template <typename T>
__device__ __forceinline__ double ld_state(const void *base, long long off) {
  return (double)reinterpret_cast<const T *>(base)[off];
}

}  // namespace sbl

// Opaque workspace of the C ABI.
struct sbletkf_workspace {
  int device;
  sbletkf_params p;
  int32_t nij1, max_nobs, nobs, ncell, ldh;
  int prepared;
  int32_t *d_elm;
  double *d_lon, *d_lat, *d_lev, *d_rdiag, *d_dep;
  double *d_hdxf64;
  float *d_hdxf32;
  int32_t *d_perm, *d_cellstart, *d_cellcnt, *d_tmp;
  int32_t *d_status;
  int32_t *h_status;  // pinned
  double *d_gscratch; // backward scalar accumulators [2]
  // analysis schedule (SBLETKF_SCHED_*): -1 automatic, 0 one CTA per point,
  // 1 persistent column queue with warm-started eigensolves (d_queue counter,
  // d_slab k x k FP64 per CTA), 2 the pipelined column queue
  int schedule = 0;
  int item_width = 0;  // columns per queue item: 0 automatic, else 1..8
  int nslab = 0;
  int32_t *d_queue = nullptr;
  double *d_slab = nullptr;
  // pipelined schedule: per CTA and slot, the local-obs list of a point
  // (sorted-obs index and rloc), list_cap entries each
  int32_t *d_list_idx = nullptr;
  double *d_list_rloc = nullptr;
  long long list_cap = 0;
  sbl::ObsView obs_view() const {
    sbl::ObsView v;
    v.nobs = nobs; v.ldh = ldh; v.elm = d_elm; v.lon = d_lon; v.lat = d_lat; v.lev = d_lev;
    v.rdiag = d_rdiag; v.dep = d_dep; v.hdxf64 = d_hdxf64; v.hdxf32 = d_hdxf32;
    v.cellstart = d_cellstart; v.perm = d_perm;
    return v;
  }
};

namespace sbl {
// host helpers implemented in abi.cu
int check_params(const sbletkf_params *p);
int cuda_status(cudaError_t e);
GridView grid_view(const sbletkf_grid *g);
// launchers
int launch_prepare_obs(sbletkf_workspace *ws, const sbletkf_params *p, const sbletkf_obs *obs, cudaStream_t s);
int launch_analysis(sbletkf_workspace *ws, const sbletkf_params *p, const GridView &g, const void *f3,
                    const void *f2, void *a3, void *a2, int dtype, const double *uni, int32_t *src,
                    int32_t *pst, cudaStream_t s);
int launch_count(sbletkf_workspace *ws, const sbletkf_params *p, const GridView &g, int32_t *nobsl,
                 cudaStream_t s);
bool pipeline_supported(const sbletkf_params *p);
// Columns per item of the column queue: the workspace's setting, or 8 when
// the grid gives at least 32 such items per CTA, narrower otherwise (the
// dynamic queue balances the CTAs only to within about one item).
inline int queue_item_width(const sbletkf_workspace *ws, long long nij1, int ctas) {
  if (ws->item_width > 0) return ws->item_width;
  const long long per = nij1 / ((long long)ctas * 32);
  return per >= 8 ? 8 : per < 1 ? 1 : (int)per;
}
int launch_analysis_ws(sbletkf_workspace *ws, const sbletkf_params *p, const GridView &g, const void *f3,
                       const void *f2, void *a3, void *a2, int dtype, const double *uni, int32_t *src, int32_t *pst,
                       cudaStream_t s);
int launch_core_batched(const sbletkf_params *p, int32_t npts, const int64_t *off, const double *hdxf,
                        const double *rdiag, const double *rloc, const double *dep, double *wvec,
                        double *wmat, const double *uni, int32_t *src, int32_t *pst, int *d_status,
                        cudaStream_t s);
int launch_obs_operator(const sbletkf_params *p, const double *glon, const double *glat, const double *gfsm,
                        const double *gdepth, const void *s3, const void *s2, int dtype, const sbletkf_obs_in *obs,
                        int flags, const sbletkf_obs_out *out, double *stats, cudaStream_t s);
int launch_obs_monitor(const sbletkf_params *p, int nobs, const int32_t *elm, const double *lev, const double *dat,
                       const double *hx, int mode, double *stats, cudaStream_t s);
int launch_ens_mesp(const sbletkf_params *p, int nij1, const void *s3, const void *s2, int dtype, void *m3, void *sd3,
                    void *m2, void *sd2, cudaStream_t s);
int launch_backward(sbletkf_workspace *ws, const sbletkf_params *p, const GridView &g, const void *f3,
                    const void *f2, int dtype, const void *ga3, const void *ga2, double *gdep,
                    double *grdiag, double *ginfl, double *gsig, cudaStream_t s);
}  // namespace sbl
