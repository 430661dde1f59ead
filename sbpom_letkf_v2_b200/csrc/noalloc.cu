// noalloc.cu -- an analysis entry point that allocates no memory.
//
// sbletkf_analysis needs a workspace from sbletkf_workspace_create, which
// calls cudaMalloc.  Some callers cannot do that where they run the analysis:
// a host model that hands the whole device to its own memory pool at start-up
// and forbids further cudaMalloc (cudaMalloc synchronises the device and fails
// once the pool has reserved the free memory), or code that must not pay an
// allocation inside its time step.  sbletkf_analysis_noalloc serves them for
// small problems: the observation bucketing and the analysis run with all their
// scratch in g_sbletkf_noalloc_scratch, a fixed array of this library that
// every GPU using the entry point holds until the process exits.
//
// Limits: nobs <= SBLETKF_NOALLOC_MAX_OBS, nlon*nlat <= SBLETKF_NOALLOC_MAX_CELLS,
// nmem <= 128.  Larger calls return SBLETKF_ERR_WORKSPACE before any launch.
//
// Set-up.  The first call on a device looks the array's device address up
// with cudaGetSymbolAddress (with that device current) and caches it together
// with the current CUDA context; a call in another context (after
// cudaDeviceReset, say) looks it up again.  Under CUDA's lazy module loading
// (the default) that first lookup is also when the array is allocated, so make
// the first call -- before any stream capture -- before the caller's memory
// pool reserves the device's free memory, or run with CUDA_MODULE_LOADING=EAGER.
//
// Errors.  Observation errors (a cell index outside the grid, non-finite
// values, err <= 0) and analysis errors are latched in a status word inside
// the array; the call's last kernel ORs that word into every point_status
// entry, so point_status is required.
//
// Reuse.  Every call reuses the same array, which keeps the previous call's
// contents: the status word and the per-cell counts are cleared by each call,
// everything else is fully rewritten before it is read.  Calls that overlap on
// the GPU (other streams, other host threads) race on the array and must be
// serialised by the caller.
#include <cuda.h>
#include <mutex>
#include <string.h>

#include "point.cuh"

namespace {

constexpr size_t al256(size_t v) { return (v + 255) & ~size_t(255); }
constexpr size_t kMaxObs = SBLETKF_NOALLOC_MAX_OBS;
constexpr size_t kMaxCells = SBLETKF_NOALLOC_MAX_CELLS;
constexpr size_t kLdh = 128;  // widest hdxf row (nmem <= 128)

constexpr size_t kOffElm = 0;
constexpr size_t kOffLon = kOffElm + al256(4 * kMaxObs);
constexpr size_t kOffLat = kOffLon + al256(8 * kMaxObs);
constexpr size_t kOffLev = kOffLat + al256(8 * kMaxObs);
constexpr size_t kOffRdiag = kOffLev + al256(8 * kMaxObs);
constexpr size_t kOffDep = kOffRdiag + al256(8 * kMaxObs);
constexpr size_t kOffH64 = kOffDep + al256(8 * kMaxObs);
constexpr size_t kOffH32 = kOffH64 + al256(8 * kMaxObs * kLdh);
constexpr size_t kOffPerm = kOffH32 + al256(4 * kMaxObs * kLdh);
constexpr size_t kOffTmp = kOffPerm + al256(4 * kMaxObs);
constexpr size_t kOffStart = kOffTmp + al256(4 * kMaxObs);
constexpr size_t kOffCnt = kOffStart + al256(4 * (kMaxCells + 1));
constexpr size_t kOffStatus = kOffCnt + al256(4 * kMaxCells);
constexpr size_t kScratchBytes = kOffStatus + al256(4 * 4);

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
struct Cached {
  CUcontext ctx;
  void *addr;
};
Cached g_scratch[kMaxDevices] = {};

}  // namespace

// All scratch of sbletkf_analysis_noalloc (about 13.4 MB per device).
static __device__ __align__(256) unsigned char g_sbletkf_noalloc_scratch[kScratchBytes];

namespace {

// The current CUDA context, through the runtime's driver entry point (so the
// library needs no link against libcuda); nullptr if it cannot be had.
CUcontext current_context() {
  using Fn = CUresult (*)(CUcontext *);
  static Fn fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<Fn>(f);
  }();
  CUcontext c = nullptr;
  if (!fn || fn(&c) != CUDA_SUCCESS) return nullptr;
  return c;
}

// Device address of the scratch array on `dev` (the current device), looked
// up once per device and context.  In host code the array's name is only a
// stand-in for the symbol, never a device address, so kernels get the
// looked-up pointer.
int scratch_address(int dev, unsigned char **out) {
  if (dev < 0 || dev >= kMaxDevices) return SBLETKF_ERR_ARG;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  const CUcontext ctx = current_context();
  Cached &c = g_scratch[dev];
  if (!c.addr || !ctx || c.ctx != ctx) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_sbletkf_noalloc_scratch);
    if (e != cudaSuccess || !ptr) return SBLETKF_ERR_CUDA;
    c.addr = ptr;
    c.ctx = current_context();  // the lookup may have created the primary context
  }
  *out = static_cast<unsigned char *>(c.addr);
  return SBLETKF_OK;
}

bool grid_complete(const sbletkf_grid *g) {
  return g && g->nij1 > 0 && g->lon1 && g->lat1 && g->ri1 && g->rj1 && g->dlon1 && g->dlat1 && g->phi1 &&
         g->depth1;
}

// point_status[p] |= *status for every point: hands the observation-level
// errors, which have no point of their own, to the caller.
__global__ void k_or_status(int32_t *__restrict__ pst, long long n, const int32_t *__restrict__ status) {
  const int32_t s = *status;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long long)gridDim.x * blockDim.x)
    pst[q] |= s;
}

}  // namespace

extern "C" int sbletkf_analysis_noalloc(const sbletkf_params *p, const sbletkf_grid *grid, const sbletkf_obs *obs,
                                        const void *fcst3d, const void *fcst2d, void *anal3d, void *anal2d,
                                        int32_t state_dtype, const double *uniforms, int32_t *point_status,
                                        void *stream) {
  int st = sbl::check_params(p);
  if (st) return st;
  if (!obs || obs->nobs < 0 || !grid_complete(grid) || !point_status) return SBLETKF_ERR_ARG;
  if ((size_t)obs->nobs > kMaxObs || (size_t)p->nlon * (size_t)p->nlat > kMaxCells ||
      (size_t)sbl::kp_of_r(sbl::r_for_k(p->nmem)) > kLdh)
    return SBLETKF_ERR_WORKSPACE;
  if (obs->nobs > 0 && (!obs->elm || !obs->idx || !obs->idy || !obs->lon || !obs->lat || !obs->lev || !obs->err ||
                        !obs->dep || !obs->hdxf))
    return SBLETKF_ERR_ARG;
  if (obs->hdxf_dtype != SBLETKF_F32 && obs->hdxf_dtype != SBLETKF_F64) return SBLETKF_ERR_ARG;
  if (state_dtype != SBLETKF_F32 && state_dtype != SBLETKF_F64) return SBLETKF_ERR_ARG;
  if (p->nv3d > 0 && (!fcst3d || !anal3d)) return SBLETKF_ERR_ARG;
  if (p->nv2d > 0 && (!fcst2d || !anal2d)) return SBLETKF_ERR_ARG;
  if (p->iswitch_da != SBLETKF_DA_LETKF && !uniforms && obs->nobs > 0) return SBLETKF_ERR_ARG;
  if (p->precision == SBLETKF_PREC_MIXED) return SBLETKF_ERR_UNSUPPORTED;

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SBLETKF_ERR_CUDA;
  unsigned char *base = nullptr;
  st = scratch_address(dev, &base);
  if (st) return st;

  // A workspace view of the fixed array (plain struct on the stack).
  sbletkf_workspace ws;
  memset(&ws, 0, sizeof(ws));
  ws.device = dev;
  ws.p = *p;
  ws.nij1 = grid->nij1;
  ws.max_nobs = (int32_t)kMaxObs;
  ws.nobs = obs->nobs;
  ws.ncell = p->nlon * p->nlat;
  ws.ldh = sbl::kp_of_r(sbl::r_for_k(p->nmem));
  ws.prepared = 1;
  ws.d_elm = reinterpret_cast<int32_t *>(base + kOffElm);
  ws.d_lon = reinterpret_cast<double *>(base + kOffLon);
  ws.d_lat = reinterpret_cast<double *>(base + kOffLat);
  ws.d_lev = reinterpret_cast<double *>(base + kOffLev);
  ws.d_rdiag = reinterpret_cast<double *>(base + kOffRdiag);
  ws.d_dep = reinterpret_cast<double *>(base + kOffDep);
  ws.d_hdxf64 = reinterpret_cast<double *>(base + kOffH64);
  ws.d_hdxf32 = reinterpret_cast<float *>(base + kOffH32);
  ws.d_perm = reinterpret_cast<int32_t *>(base + kOffPerm);
  ws.d_tmp = reinterpret_cast<int32_t *>(base + kOffTmp);
  ws.d_cellstart = reinterpret_cast<int32_t *>(base + kOffStart);
  ws.d_cellcnt = reinterpret_cast<int32_t *>(base + kOffCnt);
  ws.d_status = reinterpret_cast<int32_t *>(base + kOffStatus);

  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long npts = (long long)p->nlev * grid->nij1;
  cudaError_t e = cudaMemsetAsync(ws.d_status, 0, 4 * sizeof(int32_t), s);
  if (e != cudaSuccess) return SBLETKF_ERR_CUDA;
  st = sbl::launch_prepare_obs(&ws, p, obs, s);
  if (st) return st;
  if (obs->nobs == 0) {  // common_da.f90:57-61: analysis = forecast
    const size_t es = state_dtype == SBLETKF_F64 ? 8 : 4;
    const size_t n3 = (size_t)p->nv3d * p->nmem * p->nlev * grid->nij1;
    const size_t n2 = (size_t)p->nv2d * p->nmem * grid->nij1;
    if (n3) e = cudaMemcpyAsync(anal3d, fcst3d, n3 * es, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess && n2) e = cudaMemcpyAsync(anal2d, fcst2d, n2 * es, cudaMemcpyDeviceToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(point_status, 0, sizeof(int32_t) * (size_t)npts, s);
    if (e != cudaSuccess) return SBLETKF_ERR_CUDA;
  } else {
    sbl::GridView g;
    g.nij1 = grid->nij1;
    g.lon1 = grid->lon1; g.lat1 = grid->lat1; g.ri1 = grid->ri1; g.rj1 = grid->rj1;
    g.dlon1 = grid->dlon1; g.dlat1 = grid->dlat1; g.phi1 = grid->phi1; g.depth1 = grid->depth1;
    st = sbl::launch_analysis(&ws, p, g, fcst3d, fcst2d, anal3d, anal2d, state_dtype, uniforms, nullptr,
                              point_status, s);
    if (st) return st;
  }
  const long long blocks = (npts + 255) / 256;
  k_or_status<<<(unsigned)(blocks < 1184 ? blocks : 1184), 256, 0, s>>>(point_status, npts, ws.d_status);
  return cudaGetLastError() == cudaSuccess ? SBLETKF_OK : SBLETKF_ERR_CUDA;
}
