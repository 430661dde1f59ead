// abi.cu -- C ABI of libsbletkf (declared in include/sbletkf.h).
#include <stdio.h>
#include <string.h>

#include "point.cuh"

namespace sbl {

// Device-side error word of the workspace-free entry points.
__device__ int g_core_status;

int cuda_status(cudaError_t e) { return e == cudaSuccess ? SBLETKF_OK : SBLETKF_ERR_CUDA; }

int check_params(const sbletkf_params *p) {
  if (!p) return SBLETKF_ERR_ARG;
  if (p->nmem < 2 || p->nmem > 128) return SBLETKF_ERR_ARG;
  if (p->nlon < 2 || p->nlat < 2 || p->nlev < 1) return SBLETKF_ERR_ARG;
  if (p->nv3d < 0 || p->nv2d < 0 || p->nv3d + p->nv2d > kNvMax) return SBLETKF_ERR_ARG;
  if (p->iswitch_da < SBLETKF_DA_LETKF || p->iswitch_da > SBLETKF_DA_LPFGM) return SBLETKF_ERR_ARG;
  if (p->rm != SBLETKF_RM_SR && p->rm != SBLETKF_RM_MR) return SBLETKF_ERR_ARG;
  if (p->nmonte < 1 || p->max_sweeps < 1) return SBLETKF_ERR_ARG;
  if (!(p->cov_infl_mul > 0.0) || !(p->cov_infl_gm > 0.0) || !(p->sigma_obs > 0.0)) return SBLETKF_ERR_ARG;
  if (p->precision != SBLETKF_PREC_FP64 && p->precision != SBLETKF_PREC_MIXED) return SBLETKF_ERR_ARG;
  return SBLETKF_OK;
}

GridView grid_view(const sbletkf_grid *g) {
  GridView v;
  v.nij1 = g->nij1;
  v.lon1 = g->lon1; v.lat1 = g->lat1; v.ri1 = g->ri1; v.rj1 = g->rj1;
  v.dlon1 = g->dlon1; v.dlat1 = g->dlat1; v.phi1 = g->phi1; v.depth1 = g->depth1;
  return v;
}

static bool grid_ok(const sbletkf_grid *g) {
  return g && g->nij1 > 0 && g->lon1 && g->lat1 && g->ri1 && g->rj1 && g->dlon1 && g->dlat1 && g->phi1 &&
         g->depth1;
}

// status |= bits (sbletkf_latch_status)
__global__ void k_latch(int32_t *status, int32_t bits) { atomicOr(status, bits); }

static bool same_shape(const sbletkf_workspace *ws, const sbletkf_params *p) {
  return ws->p.nmem == p->nmem && ws->p.nlon == p->nlon && ws->p.nlat == p->nlat && ws->p.nlev == p->nlev;
}

}  // namespace sbl

using namespace sbl;

extern "C" {

int32_t sbletkf_abi_version(void) { return SBLETKF_ABI_VERSION; }

int sbletkf_workspace_create(const sbletkf_params *p, int32_t nij1, int32_t max_nobs, int32_t device,
                             sbletkf_workspace **out) {
  if (!out) return SBLETKF_ERR_ARG;
  *out = nullptr;
  int st = check_params(p);
  if (st) return st;
  if (nij1 < 1 || max_nobs < 0) return SBLETKF_ERR_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return SBLETKF_ERR_CUDA;
  sbletkf_workspace *ws = new sbletkf_workspace();
  memset(ws, 0, sizeof(*ws));
  ws->device = device;
  ws->p = *p;
  ws->nij1 = nij1;
  ws->max_nobs = max_nobs;
  ws->ncell = p->nlon * p->nlat;
  ws->ldh = kp_of_r(r_for_k(p->nmem));
  const size_t no = (size_t)(max_nobs > 0 ? max_nobs : 1);
  cudaError_t e = cudaSuccess;
  auto alloc = [&](void **ptr, size_t bytes) {
    if (e == cudaSuccess) e = cudaMalloc(ptr, bytes);
  };
  alloc((void **)&ws->d_elm, sizeof(int32_t) * no);
  alloc((void **)&ws->d_lon, sizeof(double) * no);
  alloc((void **)&ws->d_lat, sizeof(double) * no);
  alloc((void **)&ws->d_lev, sizeof(double) * no);
  alloc((void **)&ws->d_rdiag, sizeof(double) * no);
  alloc((void **)&ws->d_dep, sizeof(double) * no);
  alloc((void **)&ws->d_hdxf64, sizeof(double) * no * ws->ldh);
  alloc((void **)&ws->d_hdxf32, sizeof(float) * no * ws->ldh);
  alloc((void **)&ws->d_perm, sizeof(int32_t) * no);
  alloc((void **)&ws->d_tmp, sizeof(int32_t) * no);
  alloc((void **)&ws->d_cellstart, sizeof(int32_t) * (ws->ncell + 1));
  alloc((void **)&ws->d_cellcnt, sizeof(int32_t) * ws->ncell);
  alloc((void **)&ws->d_status, sizeof(int32_t) * 4);
  alloc((void **)&ws->d_gscratch, sizeof(double) * 8);
  {  // persistent schedule: one CTA per SM, two k x k FP64 matrices each
    int nsm = 0;
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    ws->nslab = nsm;
    alloc((void **)&ws->d_queue, sizeof(int32_t) * 4);
    alloc((void **)&ws->d_slab, sizeof(double) * (size_t)p->nmem * p->nmem * (size_t)(nsm > 0 ? nsm : 1));
    ws->schedule = SBLETKF_SCHED_AUTO;
    if (pipeline_supported(p)) {  // the pipelined schedule's per-CTA local-obs lists
      ws->list_cap = (long long)no;
      const size_t nl = (size_t)2 * (size_t)(nsm > 0 ? nsm : 1) * (size_t)ws->list_cap;
      alloc((void **)&ws->d_list_idx, sizeof(int32_t) * nl);
      alloc((void **)&ws->d_list_rloc, sizeof(double) * nl);
    }
  }
  if (e == cudaSuccess) e = cudaMallocHost((void **)&ws->h_status, sizeof(int32_t) * 4);
  if (e == cudaSuccess) e = cudaMemset(ws->d_status, 0, sizeof(int32_t) * 4);
  if (e == cudaSuccess) e = cudaMemset(ws->d_cellstart, 0, sizeof(int32_t) * (ws->ncell + 1));
  if (e != cudaSuccess) {
    sbletkf_workspace_destroy(ws);
    return SBLETKF_ERR_CUDA;
  }
  *out = ws;
  return SBLETKF_OK;
}

int sbletkf_workspace_destroy(sbletkf_workspace *ws) {
  if (!ws) return SBLETKF_OK;
  cudaSetDevice(ws->device);
  void *ptrs[] = {ws->d_elm, ws->d_lon, ws->d_lat, ws->d_lev, ws->d_rdiag, ws->d_dep, ws->d_hdxf64,
                  ws->d_hdxf32, ws->d_perm, ws->d_tmp, ws->d_cellstart, ws->d_cellcnt, ws->d_status,
                  ws->d_gscratch, ws->d_queue, ws->d_slab, ws->d_list_idx, ws->d_list_rloc};
  for (void *q : ptrs)
    if (q) cudaFree(q);
  if (ws->h_status) cudaFreeHost(ws->h_status);
  delete ws;
  return SBLETKF_OK;
}

int sbletkf_prepare_obs(sbletkf_workspace *ws, const sbletkf_params *p, const sbletkf_obs *obs, void *stream) {
  if (!ws || !obs) return SBLETKF_ERR_ARG;
  int st = check_params(p);
  if (st) return st;
  if (!same_shape(ws, p)) return SBLETKF_ERR_ARG;
  if (obs->nobs < 0 || obs->nobs > ws->max_nobs) return SBLETKF_ERR_WORKSPACE;
  if (obs->nobs > 0 && (!obs->elm || !obs->idx || !obs->idy || !obs->lon || !obs->lat || !obs->lev ||
                        !obs->err || !obs->dep || !obs->hdxf))
    return SBLETKF_ERR_ARG;
  if (obs->hdxf_dtype != SBLETKF_F32 && obs->hdxf_dtype != SBLETKF_F64) return SBLETKF_ERR_ARG;
  if (cudaSetDevice(ws->device) != cudaSuccess) return SBLETKF_ERR_CUDA;
  st = launch_prepare_obs(ws, p, obs, (cudaStream_t)stream);
  if (st) return st;
  ws->nobs = obs->nobs;
  ws->prepared = 1;
  return SBLETKF_OK;
}

int sbletkf_analysis(sbletkf_workspace *ws, const sbletkf_params *p, const sbletkf_grid *grid, const void *fcst3d,
                     const void *fcst2d, void *anal3d, void *anal2d, int32_t state_dtype, const double *uniforms,
                     int32_t *resample_src, int32_t *point_status, void *stream) {
  if (!ws || !ws->prepared) return SBLETKF_ERR_ARG;
  int st = check_params(p);
  if (st) return st;
  if (!same_shape(ws, p) || !grid_ok(grid) || grid->nij1 != ws->nij1) return SBLETKF_ERR_ARG;
  if (state_dtype != SBLETKF_F32 && state_dtype != SBLETKF_F64) return SBLETKF_ERR_ARG;
  if (p->nv3d > 0 && (!fcst3d || !anal3d)) return SBLETKF_ERR_ARG;
  if (p->nv2d > 0 && (!fcst2d || !anal2d)) return SBLETKF_ERR_ARG;
  if (p->iswitch_da != SBLETKF_DA_LETKF && !uniforms && ws->nobs > 0) return SBLETKF_ERR_ARG;
  if (cudaSetDevice(ws->device) != cudaSuccess) return SBLETKF_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  if (ws->nobs == 0) {  // common_da.f90:57-61: analysis = forecast, no round-off
    const size_t es = state_dtype == SBLETKF_F64 ? 8 : 4;
    const size_t n3 = (size_t)p->nv3d * p->nmem * p->nlev * grid->nij1;
    const size_t n2 = (size_t)p->nv2d * p->nmem * grid->nij1;
    cudaError_t e = cudaSuccess;
    if (n3) e = cudaMemcpyAsync(anal3d, fcst3d, n3 * es, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && n2) e = cudaMemcpyAsync(anal2d, fcst2d, n2 * es, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && point_status)
      e = cudaMemsetAsync(point_status, 0, sizeof(int32_t) * (size_t)p->nlev * grid->nij1, s);
    return cuda_status(e);
  }
  return launch_analysis(ws, p, grid_view(grid), fcst3d, fcst2d, anal3d, anal2d, state_dtype, uniforms,
                         resample_src, point_status, s);
}

int sbletkf_workspace_set_schedule(sbletkf_workspace *ws, int32_t schedule) {
  if (!ws || (schedule != SBLETKF_SCHED_AUTO && schedule != SBLETKF_SCHED_POINT &&
              schedule != SBLETKF_SCHED_COLUMNS && schedule != SBLETKF_SCHED_PIPELINE))
    return SBLETKF_ERR_ARG;
  if (schedule == SBLETKF_SCHED_PIPELINE && !ws->d_list_idx) return SBLETKF_ERR_UNSUPPORTED;
  ws->schedule = schedule;
  return SBLETKF_OK;
}

int sbletkf_workspace_set_item_width(sbletkf_workspace *ws, int32_t width) {
  if (!ws || width < 0 || width > 8) return SBLETKF_ERR_ARG;
  ws->item_width = width;
  return SBLETKF_OK;
}

int sbletkf_count_nobsl(sbletkf_workspace *ws, const sbletkf_params *p, const sbletkf_grid *grid, int32_t *nobsl,
                        void *stream) {
  if (!ws || !ws->prepared || !nobsl) return SBLETKF_ERR_ARG;
  int st = check_params(p);
  if (st) return st;
  if (!same_shape(ws, p) || !grid_ok(grid) || grid->nij1 != ws->nij1) return SBLETKF_ERR_ARG;
  if (cudaSetDevice(ws->device) != cudaSuccess) return SBLETKF_ERR_CUDA;
  if (ws->nobs == 0)
    return cuda_status(cudaMemsetAsync(nobsl, 0, sizeof(int32_t) * (size_t)p->nlev * grid->nij1, (cudaStream_t)stream));
  return launch_count(ws, p, grid_view(grid), nobsl, (cudaStream_t)stream);
}

int sbletkf_get_status(sbletkf_workspace *ws, void *stream, int32_t *status) {
  if (!ws || !status) return SBLETKF_ERR_ARG;
  if (cudaSetDevice(ws->device) != cudaSuccess) return SBLETKF_ERR_CUDA;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(ws->h_status, ws->d_status, sizeof(int32_t), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemsetAsync(ws->d_status, 0, sizeof(int32_t), s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    *status = SBLETKF_ERR_CUDA;
    return SBLETKF_ERR_CUDA;
  }
  *status = ws->h_status[0];
  return SBLETKF_OK;
}

int sbletkf_latch_status(sbletkf_workspace *ws, int32_t bits, void *stream) {
  if (!ws) return SBLETKF_ERR_ARG;
  if (cudaSetDevice(ws->device) != cudaSuccess) return SBLETKF_ERR_CUDA;
  k_latch<<<1, 1, 0, (cudaStream_t)stream>>>(ws->d_status, bits);
  return cuda_status(cudaGetLastError());
}

int sbletkf_core_batched(const sbletkf_params *p, int32_t npts, const int64_t *off, const double *hdxf,
                         const double *rdiag, const double *rloc, const double *dep, double *wvec, double *wmat,
                         const double *uniforms, int32_t *resample_src, int32_t *point_status, void *stream) {
  int st = check_params(p);
  if (st) return st;
  if (npts < 0 || (npts > 0 && (!off || !wvec || !wmat))) return SBLETKF_ERR_ARG;
  if (p->iswitch_da != SBLETKF_DA_LETKF && npts > 0 && !uniforms) return SBLETKF_ERR_ARG;
  int *d_status = nullptr;
  if (cudaGetSymbolAddress((void **)&d_status, g_core_status) != cudaSuccess) return SBLETKF_ERR_CUDA;
  return launch_core_batched(p, npts, off, hdxf, rdiag, rloc, dep, wvec, wmat, uniforms, resample_src,
                             point_status, d_status, (cudaStream_t)stream);
}

int sbletkf_backward(sbletkf_workspace *ws, const sbletkf_params *p, const sbletkf_grid *grid, const void *fcst3d,
                     const void *fcst2d, int32_t state_dtype, const void *grad_anal3d, const void *grad_anal2d,
                     double *grad_dep, double *grad_rdiag, double *grad_infl, double *grad_sigma_obs,
                     void *stream) {
  if (!ws || !ws->prepared) return SBLETKF_ERR_ARG;
  int st = check_params(p);
  if (st) return st;
  if (!same_shape(ws, p) || !grid_ok(grid) || grid->nij1 != ws->nij1) return SBLETKF_ERR_ARG;
  if (p->iswitch_da != SBLETKF_DA_LETKF) return SBLETKF_ERR_UNSUPPORTED;
  if (!grad_dep || !grad_rdiag || !grad_infl || !grad_sigma_obs) return SBLETKF_ERR_ARG;
  if (state_dtype != SBLETKF_F32 && state_dtype != SBLETKF_F64) return SBLETKF_ERR_ARG;
  if (cudaSetDevice(ws->device) != cudaSuccess) return SBLETKF_ERR_CUDA;
  return launch_backward(ws, p, grid_view(grid), fcst3d, fcst2d, state_dtype, grad_anal3d, grad_anal2d, grad_dep,
                         grad_rdiag, grad_infl, grad_sigma_obs, (cudaStream_t)stream);
}

int sbletkf_obs_operator(const sbletkf_params *p, const double *glon, const double *glat, const double *gfsm,
                         const double *gdepth, const void *state3d, const void *state2d, int32_t state_dtype,
                         const sbletkf_obs_in *obs, int32_t flags, const sbletkf_obs_out *out, double *stats,
                         void *stream) {
  int st = check_params(p);
  if (st) return st;
  if (!obs || !out || obs->nobs < 0) return SBLETKF_ERR_ARG;
  if (p->nlev < 6) return SBLETKF_ERR_UNSUPPORTED;
  if (state_dtype != SBLETKF_F32 && state_dtype != SBLETKF_F64) return SBLETKF_ERR_ARG;
  if (obs->nobs > 0 && (!obs->elm || !obs->lon || !obs->lat || !obs->lev || !obs->dat || !obs->err || !glon ||
                        !glat || !gfsm || !gdepth || (p->nv3d > 0 && !state3d) || (p->nv2d > 0 && !state2d)))
    return SBLETKF_ERR_ARG;
  return sbl::launch_obs_operator(p, glon, glat, gfsm, gdepth, state3d, state2d, state_dtype, obs, flags, out,
                                  stats, (cudaStream_t)stream);
}

int sbletkf_ensemble_mean_spread(const sbletkf_params *p, int32_t nij1, const void *state3d, const void *state2d,
                                 int32_t state_dtype, void *mean3d, void *sprd3d, void *mean2d, void *sprd2d,
                                 void *stream) {
  if (!p || p->nmem < 1 || p->nmem > 128 || p->nlev < 1 || p->nv3d < 0 || p->nv2d < 0 || nij1 < 1)
    return SBLETKF_ERR_ARG;
  if (state_dtype != SBLETKF_F32 && state_dtype != SBLETKF_F64) return SBLETKF_ERR_ARG;
  if ((p->nv3d > 0 && (!state3d || !mean3d)) || (p->nv2d > 0 && (!state2d || !mean2d))) return SBLETKF_ERR_ARG;
  return sbl::launch_ens_mesp(p, nij1, state3d, state2d, state_dtype, mean3d, sprd3d, mean2d, sprd2d,
                              (cudaStream_t)stream);
}

}  // extern "C"
