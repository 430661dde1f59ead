// analysis.cu -- the analysis step: a CTA analyses one grid point at a time.
//
// Replaces the body of the (k,i) loop of da_main (letkf/run/src/common_da.f90:
// 67-116): local observation selection (count_nobsl / obs_local, :133-293) as a
// single streaming pass over the search box in the reference's candidate order,
// the LETKF / LPF / LPFGM transform, the ensemble update with RTPP / RTPS, and
// the T/S round-off (:506-533), which is per point and so fused here.
//
// The transform is applied without forming W or Pa:
//   anal_v = xm_v + dX_v V c  +  (dX_v V) diag(sqrt((k-1)/lambda)) V^T
// with c = Lambda^-1 V^T b, b = Y^T R^-1 rho dep; this equals
// xm + dX (wvec 1^T + W) of Analysis_Ensemble (:407-432) up to rounding.
//
// Points with nobsl < k (at most kDualMax) take the observation-space form of
// the same transform: with Z = diag(sqrt(rloc/rdiag)) Y (n x k) and
// N = alpha I_n + Z Z^T = Q Lambda Q^T (alpha = (k-1)/rho),
//   wvec = Z^T Q Lambda^-1 Q^T d,  d = sqrt(rloc/rdiag) dep
//   W    = sqrt(k-1) [ alpha^-1/2 I + Z^T Q diag(g) Q^T Z ],
//   g_j  = -1 / ( sqrt(alpha lambda_j) (sqrt(lambda_j) + sqrt(alpha)) ),
// exact algebra (push-through identity), so only an n x n eigensolve is needed.
#include "point_tail.cuh"
#include "tc_point.cuh"

namespace sbl {
namespace {

// Analysis of grid point pid by the whole CTA (the body of the (k,i) loop of
// da_main).  With vprev != nullptr (persistent, column-ordered launch) a
// primal eigensolve starts from the eigenvectors of the previous level of
// the same column when `warm` is set, and leaves its own there.
template <int R, typename ST, bool MIXED>
__device__ __forceinline__ void analyze_point(const sbletkf_params &p, const GridView &g, const ObsView &ob,
                                              const ST *__restrict__ f3, const ST *__restrict__ f2,
                                              ST *__restrict__ a3, ST *__restrict__ a2,
                                              const double *__restrict__ uni, int32_t *__restrict__ src_out,
                                              int32_t *__restrict__ pst, int *status, const PointSmem &S,
                                              TcState &tcs, uint64_t *s_mbar, bool tc_on, long long pid,
                                              double *vprev, int &warm) {
  constexpr int KP = kp_of_r(R);
  const int k = p.nmem;
  const int tid = threadIdx.x;
  const int nij1 = g.nij1, nlev = p.nlev;
  const int kl = (int)(pid / nij1), i = (int)(pid % nij1);
  const bool do_pf = p.iswitch_da != SBLETKF_DA_LETKF;
  const bool do_gram = p.iswitch_da != SBLETKF_DA_LPF;
  __shared__ int sh[8];
  __shared__ double shd[4];
  int bits = 0;
  if (tc_on) {
    // after a tensor-core wait has timed out anywhere in the launch, later
    // points return at once (the status word already carries the error)
    __shared__ int s_abort;
    if (tid == 0) s_abort = (*(volatile int *)status & SBLETKF_ERR_TIMEOUT) != 0;
    __syncthreads();
    const int ab = s_abort;
    __syncthreads();
    if (ab) {
      if (tid == 0 && pst) pst[pid] = SBLETKF_ERR_TIMEOUT;
      return;
    }
    tcs.nchunk = 0;
    tcs.nflushed = 0;
  }

  // ---- search box and its grid rows (common_da.f90:158-161, 314-346)
  if (tid == 0) {
    int imin, imax, jmin, jmax;
    search_box(p, g, i, imin, imax, jmin, jmax);
    int nrows = jmax - jmin + 1;
    if (nrows < 0) nrows = 0;
    if (nrows > kRowMax) {
      nrows = kRowMax;
      sh[5] = SBLETKF_ERR_ROWS;
    } else {
      sh[5] = 0;
    }
    sh[0] = imin; sh[1] = imax; sh[2] = jmin; sh[4] = nrows;
    shd[0] = g.depth1[pid];
    shd[1] = g.lon1[i];
    shd[2] = g.lat1[i];
    shd[3] = g.phi1[i];
  }
  __syncthreads();
  bits |= sh[5];
  const int imin = sh[0], imax = sh[1], jmin = sh[2], nrows = sh[4];
  const double rdep = shd[0], plon = shd[1], plat = shd[2], phi = shd[3];
  {
    int lens[4], loc = 0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int r = tid * 4 + t;
      lens[t] = 0;
      if (r < nrows) {
        const int j = jmin + r;
        const int st = ob.cellstart[(long)(j - 1) * p.nlon + (imin - 1)];
        const int en = ob.cellstart[(long)(j - 1) * p.nlon + imax];
        S.rowstart[r] = st;
        lens[t] = en > st ? en - st : 0;
        loc += lens[t];
      }
    }
    int excl;
    const int tot = block_excl_scan(loc, excl, S.iws);
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int r = tid * 4 + t;
      if (r < nrows) {
        S.rowpref[r] = excl;
        excl += lens[t];
      }
    }
    if (tid == 0) S.rowpref[nrows] = tot;
    __syncthreads();
  }
  const int ncand = S.rowpref[nrows];
  // FP32 accumulation in tensor memory is accurate to ~eps32 sqrt(n/16) |G|;
  // points whose search box holds more candidates take the FP64 Gram
  const bool use_tc = tc_on && (double)ncand <= (p.tc_max_cand > 0.0 ? p.tc_max_cand : (double)tc::kMaxCand);

  // ---- streaming local-obs selection + accumulation (obs order preserved).
  // Rows are consumed on the fly once nobsl exceeds the dual limit; below it
  // the list is kept for the observation-space transform.
  Accum<R> A;
  A.zero();
  // tensor-core staging: FP32 rows of the sorted observations, by list index
  const auto rows = [&](float *stg, int f, int cnt) {
    constexpr int KP4 = KP / 4;
    for (int e = tid; e < tc::kKC * KP4; e += kThreads) {
      const int cc = e / KP4, col = e - cc * KP4;
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (cc < cnt) v = reinterpret_cast<const float4 *>(ob.hdxf32 + (long)S.lidx[f + cc] * ob.ldh)[col];
      reinterpret_cast<float4 *>(stg)[e] = v;
    }
  };
  int L = 0, nacc = 0;
  const int ndm = do_gram ? PointSmem::dual_max(k) : -1;
  bool primal = ndm < 0;
  for (int base = 0; base < ncand; base += kThreads) {
    const int c = base + tid;
    int accept = 0, o = 0;
    double rl = 0.0;
    if (c < ncand) {
      int lo = 0, hi = nrows - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (S.rowpref[mid] <= c) lo = mid;
        else hi = mid - 1;
      }
      o = S.rowstart[lo] + (c - S.rowpref[lo]);
      const double dl = dlev_of(ob.elm[o], ob.lev[o], rdep, kl, nlev, p.id_z_obs);
      if (!(p.dist_zerov < dl)) {
        const double dist = distance_2p(ob.lon[o], ob.lat[o], plon, plat, p.pi, p.re);
        if (!(p.dist_zero < dist)) {
          accept = 1;
          rl = loc_weight(dist, dl, p.sigma_obs, p.sigma_obsv);
        }
      }
    }
    int excl;
    const int tot = block_excl_scan(accept, excl, S.iws);
    if (accept) {
      const int q = L + excl;
      const double rd = ob.rdiag[o], dp = ob.dep[o];
      S.lidx[q] = o;
      S.lrloc[q] = rl;
      S.lrdiag[q] = rd;
      S.ldep[q] = dp;
      const double w = rl / rd;
      S.lw[q] = w;
      S.lwd[q] = w * dp;
    }
    L += tot;
    nacc += tot;
    __syncthreads();
    if (!primal && L > ndm) primal = true;
    if (!primal) continue;
    int f = 0;
    if (use_tc) {
      while (L - f >= tc::kKC) {
        tc_chunk<KP>(S, rows, tcs, s_mbar, f, tc::kKC, k, do_pf, A.b, A.ll, bits);
        f += tc::kKC;
      }
    }
    while (!use_tc && L - f >= kChunk) {
      constexpr int KP2 = KP / 2;
      for (int e = tid; e < kChunk * KP2; e += kThreads) {
        const int cc = e / KP2, col = e - cc * KP2;
        reinterpret_cast<double2 *>(S.u)[e] =
            reinterpret_cast<const double2 *>(ob.hdxf64 + (long)S.lidx[f + cc] * ob.ldh)[col];
      }
      __syncthreads();
      accumulate_chunk<R>(S, f, kChunk, k, do_gram, do_pf, A);
      f += kChunk;
    }
    const int rem = L - f;
    if (f > 0 && rem > 0) {
      if (tid < rem) {
        const int s = f + tid;
        S.lidx[tid] = S.lidx[s];
        S.lrloc[tid] = S.lrloc[s];
        S.lrdiag[tid] = S.lrdiag[s];
        S.ldep[tid] = S.ldep[s];
        S.lw[tid] = S.lw[s];
        S.lwd[tid] = S.lwd[s];
      }
      __syncthreads();
    }
    L = rem;
  }
  if (use_tc && primal && L > 0) tc_chunk<KP>(S, rows, tcs, s_mbar, 0, L, k, do_pf, A.b, A.ll, bits);
  if (!use_tc && primal && L > 0) {
    constexpr int KP2 = KP / 2;
    for (int e = tid; e < L * KP2; e += kThreads) {
      const int cc = e / KP2, col = e - cc * KP2;
      reinterpret_cast<double2 *>(S.u)[e] =
          reinterpret_cast<const double2 *>(ob.hdxf64 + (long)S.lidx[cc] * ob.ldh)[col];
    }
    __syncthreads();
    accumulate_chunk<R>(S, 0, L, k, do_gram, do_pf, A);
  }

  const bool dual = !primal && nacc > 0;
  if (!dual && nacc > 0 && do_gram) {  // G + alpha I into S.u, b into S.b
    const double alpha = (double)(k - 1) / (p.iswitch_da == SBLETKF_DA_LETKF ? p.cov_infl_mul : p.cov_infl_gm);
    if (use_tc) tc_finish<KP>(S, tcs, s_mbar, k, alpha, A.b, bits);
    else store_gram<R>(S, k, alpha, A);
  }
  point_tail<R, ST>(p, ob, f3, f2, a3, a2, uni, src_out, pst, status, S, pid, nij1, phi, nacc, dual, A.ll, bits,
                    tc_on, vprev, warm);
}

// One CTA per grid point (queue == nullptr; point p0 + blockIdx.x), or a
// persistent launch of one CTA per SM taking items of up to colchunk grid
// columns, cstride apart, from the atomic counter *queue and analysing their
// levels in snake order,
// warm-starting every primal eigensolve from the previous primal point
// (slab: one k x k FP64 matrix per CTA, the previous eigenvectors).
template <int R, typename ST, bool MIXED>
__global__ void __launch_bounds__(kThreads, 1)
    k_analysis(const sbletkf_params p, const GridView g, const ObsView ob, const ST *__restrict__ f3,
               const ST *__restrict__ f2, ST *__restrict__ a3, ST *__restrict__ a2, const double *__restrict__ uni,
               int32_t *__restrict__ src_out, int32_t *__restrict__ pst, int *status, long long p0, int *queue,
               double *slab, int colchunk, int cstride) {
  constexpr int KP = kp_of_r(R);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PointSmem S;
  const int k = p.nmem;
  S.carve(smem_raw, k, KP);
  const int tid = threadIdx.x;
  const bool do_gram = p.iswitch_da != SBLETKF_DA_LPF;
  __shared__ uint64_t s_mbar[2];
  __shared__ uint32_t s_tmem;
  const bool tc_on = MIXED && do_gram;  // TMEM and barriers held by this CTA
  TcState tcs;
  tcs.uses[0] = tcs.uses[1] = 0;
  tcs.issued[0] = tcs.issued[1] = 0;
  tcs.nchunk = 0;
  tcs.nflushed = 0;
  tcs.tbase = 0;
  tcs.broken = 0;
  // A launch that finds SBLETKF_ERR_TIMEOUT already latched (a tensor-core
  // wait expired earlier) allocates no tensor memory and issues no UMMA: one
  // CTA per point marks its point and returns; the persistent launch still
  // drains its queue, and analyze_point marks every point it takes.
  __shared__ int s_abort;
  if (tid == 0) s_abort = tc_on && (*(volatile int *)status & SBLETKF_ERR_TIMEOUT) != 0;
  __syncthreads();
  const bool aborted = s_abort != 0;
  if (aborted && !queue) {
    if (tid == 0 && pst) pst[p0 + blockIdx.x] = SBLETKF_ERR_TIMEOUT;
    return;
  }
  if (tc_on && !aborted) tc_open<KP>(tcs, s_mbar, &s_tmem);
  // one call site of the point body for both schedules.  Column schedule: a
  // queue item is up to colchunk (1..8) columns cstride apart -- with cstride
  // = nlon, neighbours along a meridian -- walked in snake order (levels down,
  // then up, ...), so every column's first level with a primal eigensolve
  // starts from the same level of the column beside it and every later level
  // from the level above or below.  Items q and q+1 hold adjacent columns of
  // the same latitude rows, so the CTAs running at the same time read and
  // write the same 32-byte sectors of the state at about the same time.
  double *vprev = queue ? slab + (size_t)blockIdx.x * k * k : nullptr;
  __shared__ int s_item;
  int warm = 0, c0 = 0, w = 0, pos = 0, npos = 0;
  bool first = true;
  for (;;) {
    long long pid;
    if (queue) {
      if (pos == npos) {  // next item from the queue
        if (tid == 0) s_item = atomicAdd(queue, 1);
        __syncthreads();
        const long long q = s_item, band = q / cstride;
        const long long cs = band * colchunk * cstride + (q - band * cstride);
        __syncthreads();
        if (cs >= g.nij1) break;  // later items start further on
        const long long left = (g.nij1 - cs + cstride - 1) / cstride;
        c0 = (int)cs;
        w = (int)(left < colchunk ? left : colchunk);
        pos = 0;
        npos = w * p.nlev;
        warm = 0;
      }
      const int j = pos / p.nlev, r = pos - j * p.nlev;
      const int kl = (j & 1) ? r : p.nlev - 1 - r;  // surface-down first, then bottom-up, ...
      ++pos;
      pid = (long long)kl * g.nij1 + c0 + (long long)j * cstride;
    } else {
      if (!first) break;
      first = false;
      pid = p0 + blockIdx.x;
    }
    analyze_point<R, ST, MIXED>(p, g, ob, f3, f2, a3, a2, uni, src_out, pst, status, S, tcs, s_mbar, tc_on, pid,
                                vprev, warm);
  }
  if (tc_on && !aborted) tc_close<KP>(tcs, s_mbar, status);
}

// count_nobsl (common_da.f90:133-205): one warp per point.
__global__ void k_count(const sbletkf_params p, const GridView g, const ObsView ob, int32_t *__restrict__ nobsl,
                        long long npts, int *status) {
  const int lane = threadIdx.x & 31;
  const long long pid = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (pid >= npts) return;
  const int nij1 = g.nij1;
  const int kl = (int)(pid / nij1), i = (int)(pid % nij1);
  int imin, imax, jmin, jmax;
  search_box(p, g, i, imin, imax, jmin, jmax);
  const double rdep = g.depth1[pid], plon = g.lon1[i], plat = g.lat1[i];
  int cnt = 0;
  for (int j = jmin; j <= jmax; ++j) {
    const int st = ob.cellstart[(long)(j - 1) * p.nlon + (imin - 1)];
    const int en = ob.cellstart[(long)(j - 1) * p.nlon + imax];
    for (int o = st + lane; o < en; o += 32) {
      const double dl = dlev_of(ob.elm[o], ob.lev[o], rdep, kl, p.nlev, p.id_z_obs);
      if (p.dist_zerov < dl) continue;
      const double dist = distance_2p(ob.lon[o], ob.lat[o], plon, plat, p.pi, p.re);
      if (p.dist_zero < dist) continue;
      ++cnt;
    }
  }
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if (lane == 0) nobsl[pid] = cnt;
  (void)status;
}

struct Sched {
  int *queue;    // nullptr: one CTA per point
  double *slab;
  int ctas;
  int width;     // columns per queue item
};

template <int R, typename ST, bool MIXED>
int launch_r(const sbletkf_params *p, const GridView &g, const ObsView &ob, const void *f3, const void *f2, void *a3,
             void *a2, const double *uni, int32_t *src, int32_t *pst, int *status, const Sched &sc, cudaStream_t s) {
  const size_t smem = PointSmem::bytes(p->nmem, kp_of_r(R), MIXED);
  auto kern = k_analysis<R, ST, MIXED>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_status(e);
  if (sc.queue) {
    const int colchunk = sc.width;
    const int cstride = p->nlon > 1 ? p->nlon : 1;
    e = cudaMemsetAsync(sc.queue, 0, sizeof(int), s);
    if (e != cudaSuccess) return cuda_status(e);
    kern<<<(unsigned)sc.ctas, kThreads, smem, s>>>(*p, g, ob, (const ST *)f3, (const ST *)f2, (ST *)a3, (ST *)a2,
                                                    uni, src, pst, status, 0, sc.queue, sc.slab, colchunk, cstride);
    return cuda_status(cudaGetLastError());
  }
  const long long P = (long long)p->nlev * g.nij1;
  const long long maxg = 2147483647LL;
  for (long long p0 = 0; p0 < P; p0 += maxg) {
    const long long n = P - p0 < maxg ? P - p0 : maxg;
    kern<<<(unsigned)n, kThreads, smem, s>>>(*p, g, ob, (const ST *)f3, (const ST *)f2, (ST *)a3, (ST *)a2, uni,
                                              src, pst, status, p0, nullptr, nullptr, 1, 1);
  }
  return cuda_status(cudaGetLastError());
}

template <typename ST>
int launch_t(const sbletkf_params *p, const GridView &g, const ObsView &ob, const void *f3, const void *f2, void *a3,
             void *a2, const double *uni, int32_t *src, int32_t *pst, int *status, const Sched &sc, cudaStream_t s) {
  const bool mixed = p->precision == SBLETKF_PREC_MIXED;
  switch (r_for_k(p->nmem)) {
    case 2: return mixed ? launch_r<2, ST, true>(p, g, ob, f3, f2, a3, a2, uni, src, pst, status, sc, s)
                         : launch_r<2, ST, false>(p, g, ob, f3, f2, a3, a2, uni, src, pst, status, sc, s);
    case 4: return mixed ? launch_r<4, ST, true>(p, g, ob, f3, f2, a3, a2, uni, src, pst, status, sc, s)
                         : launch_r<4, ST, false>(p, g, ob, f3, f2, a3, a2, uni, src, pst, status, sc, s);
    case 7: return mixed ? launch_r<7, ST, true>(p, g, ob, f3, f2, a3, a2, uni, src, pst, status, sc, s)
                         : launch_r<7, ST, false>(p, g, ob, f3, f2, a3, a2, uni, src, pst, status, sc, s);
    default: return mixed ? launch_r<8, ST, true>(p, g, ob, f3, f2, a3, a2, uni, src, pst, status, sc, s)
                          : launch_r<8, ST, false>(p, g, ob, f3, f2, a3, a2, uni, src, pst, status, sc, s);
  }
}

}  // namespace

int launch_analysis(sbletkf_workspace *ws, const sbletkf_params *p, const GridView &g, const void *f3,
                    const void *f2, void *a3, void *a2, int dtype, const double *uni, int32_t *src, int32_t *pst,
                    cudaStream_t s) {
  int sched = ws->schedule;
  // Automatic: the pipeline pays where a point's eigensolve outweighs the
  // producer's tensor-core Gram, whose cost per chunk does not shrink with k
  // (UMMA M is 128 rows): 65 <= k <= 112.  Measured: k = 100 503.6k vs 439.4k
  // gridpoints/s for the column queue; k = 64 685k vs 843k; k = 20 1.67M vs
  // 2.2M.  The FP64 Gram is faster in the column queue's 256-thread CTA.
  if (sched == SBLETKF_SCHED_AUTO)
    sched = p->iswitch_da == SBLETKF_DA_LPF                                ? SBLETKF_SCHED_POINT
            : (p->precision == SBLETKF_PREC_MIXED && r_for_k(p->nmem) == 7) ? SBLETKF_SCHED_PIPELINE
                                                                            : SBLETKF_SCHED_COLUMNS;
  if (sched == SBLETKF_SCHED_PIPELINE && ws->d_list_idx && ws->d_queue && ws->d_slab && pipeline_supported(p))
    return launch_analysis_ws(ws, p, g, f3, f2, a3, a2, dtype, uni, src, pst, s);
  const ObsView ob = ws->obs_view();
  Sched sc{nullptr, nullptr, 0, 1};
  if (sched >= SBLETKF_SCHED_COLUMNS && ws->d_queue && ws->d_slab)
    sc = Sched{ws->d_queue, ws->d_slab, ws->nslab, queue_item_width(ws, g.nij1, ws->nslab)};
  if (dtype == SBLETKF_F64) return launch_t<double>(p, g, ob, f3, f2, a3, a2, uni, src, pst, ws->d_status, sc, s);
  return launch_t<float>(p, g, ob, f3, f2, a3, a2, uni, src, pst, ws->d_status, sc, s);
}

int launch_count(sbletkf_workspace *ws, const sbletkf_params *p, const GridView &g, int32_t *nobsl,
                 cudaStream_t s) {
  const ObsView ob = ws->obs_view();
  const long long P = (long long)p->nlev * g.nij1;
  const int wpb = 8;
  k_count<<<(unsigned)((P + wpb - 1) / wpb), wpb * 32, 0, s>>>(*p, g, ob, nobsl, P, ws->d_status);
  return cuda_status(cudaGetLastError());
}

}  // namespace sbl
