// analysis_ws.cu -- the analysis step as a warp-specialised persistent
// kernel (SBLETKF_SCHED_PIPELINE): LETKF and LPFGM, nmem <= 112.
//
// One CTA per SM, 384 threads in two roles that work on consecutive grid
// points of the CTA's column-queue items (the walk of the column schedule:
// items of up to 8 columns nlon apart, levels in snake order):
//
//   producer (warps 8..11, 128 threads), point i+1:
//     search box and candidate scan of count_nobsl / obs_local
//     (common_da.f90:133-348), the accepted observations appended in the
//     reference's candidate order to a per-CTA list in global memory; for a
//     point whose Gram goes to the tensor cores (mixed precision, search box
//     <= tc_max_cand candidates, more than dual_max local obs) the list is
//     streamed at once, 32 observations at a time, into tcgen05 UMMAs:
//     thread m loads member m of each row, scales it by sqrt(rloc/rdiag),
//     splits it into BF16 h/m/l and stores the K-major operand tiles; chunk
//     pairs accumulate in FP32 in tensor memory and are added into a running
//     double-FP32 (TwoSum) sum; b = Y^T diag(w) dep and (LPFGM) the PF
//     log-likelihood are accumulated in FP64 in the same pass;
//   consumer (warps 0..7, 256 threads), point i:
//     takes the Gram out of tensor memory (or, on the FP64 path and for
//     denser points, accumulates it from the list in FP64 registers), then
//     the eigensolve (warm-started from the previous level), transform,
//     update, RTPP / RTPS / round-off and the store (point_tail).
//
// So the selection and the Gram of one point run under the eigensolve of the
// previous one.  Hand-over: two slots (list, b, log-likelihood, point
// record) guarded by full/empty mbarriers, and a tmem_free mbarrier that
// holds the next Gram back until the consumer has read the previous one.
// Every wait across the roles is bounded (kWaitNs); one that expires latches
// SBLETKF_ERR_TIMEOUT, raises the CTA's abort flag and both roles stop.
#include "point_tail.cuh"
#include "tc_point.cuh"

namespace sbl {
namespace {

constexpr int kProd = 128;                              // producer threads
constexpr int kWsThreads = kThreads + kProd;            // 384
constexpr int kWin = 192;                               // producer list window
constexpr int kKCw = 32;                                // observations per UMMA chunk
constexpr int kTileW = tc::kBlockBytes * (kKCw / tc::kKB);  // one split part of a chunk: 8 KB
constexpr int kStageW = 3 * kTileW;                     // h, m, l: 24 KB
constexpr unsigned long long kWaitNs = 4000000000ull;   // cross-role wait limit
constexpr int kRegLaunch = 168, kRegProd = 120, kRegCons = 192;  // registers per thread
static_assert(kRegProd * kProd + kRegCons * kThreads <= kRegLaunch * kWsThreads,
              "the role split must fit in the launch's registers");
static_assert(kRegLaunch * kWsThreads <= 65536, "one CTA per SM");

// point record flags
constexpr int kFPrimal = 1, kFTc = 2, kFNewItem = 4, kFEnd = 8, kFAbort = 16;

__device__ __forceinline__ void pbar() { asm volatile("bar.sync 2, %0;" ::"n"(kProd) : "memory"); }

__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(tc::smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Wait for phase `parity` of a hand-over barrier: false when the CTA's abort
// flag is raised or kWaitNs passes.  One thread.
__device__ __forceinline__ bool ws_wait(uint64_t *bar, uint32_t parity, volatile int *abort) {
  const unsigned long long t0 = gtimer();
  for (unsigned it = 0;; ++it) {
    if (mbar_try(bar, parity)) return true;
    if (*abort) return false;
    if ((it & 63) == 63 && gtimer() - t0 > kWaitNs) return false;
  }
}

// Control block of the two roles (static shared memory).
struct WsCtl {
  uint64_t full[2], empty[2], tmem_free, mma[2];
  uint32_t tmem;
  int abort;
  int item;
  int ok_c, ok_p, brk_p;
  long long pid[2];
  int nacc[2], flags[2], bits[2];
};

// Producer shared memory.
struct ProdSmem {
  int *rowstart, *rowpref, *wlidx, *ws;
  double *wlw, *wlwd, *wlrloc, *wlrdiag, *wldep;
  float *sw;
  double *pb, *pll;          // [2][KP] each: b and log-likelihood per slot
  unsigned char *stage;      // two operand stages, 1024-aligned

  __host__ __device__ static size_t a16(size_t v) { return (v + 15) & ~size_t(15); }
  __host__ __device__ static size_t bytes(int kp) {
    size_t s = a16(sizeof(int) * kRowMax) + a16(sizeof(int) * (kRowMax + 1)) + a16(sizeof(int) * kWin) +
               a16(sizeof(int) * 16);
    s += 5 * a16(sizeof(double) * kWin) + a16(sizeof(float) * kKCw) + 4 * a16(sizeof(double) * kp);
    return s + 1024 + 2 * (size_t)kStageW;
  }
  __device__ void carve(unsigned char *base, int kp) {
    unsigned char *q = base;
    auto take = [&](size_t n) { unsigned char *r = q; q += a16(n); return (void *)r; };
    rowstart = (int *)take(sizeof(int) * kRowMax);
    rowpref = (int *)take(sizeof(int) * (kRowMax + 1));
    wlidx = (int *)take(sizeof(int) * kWin);
    ws = (int *)take(sizeof(int) * 16);
    wlw = (double *)take(sizeof(double) * kWin);
    wlwd = (double *)take(sizeof(double) * kWin);
    wlrloc = (double *)take(sizeof(double) * kWin);
    wlrdiag = (double *)take(sizeof(double) * kWin);
    wldep = (double *)take(sizeof(double) * kWin);
    sw = (float *)take(sizeof(float) * kKCw);
    pb = (double *)take(2 * sizeof(double) * kp);
    pll = (double *)take(2 * sizeof(double) * kp);
    const uintptr_t a = (reinterpret_cast<uintptr_t>(q) + 1023) & ~uintptr_t(1023);
    stage = reinterpret_cast<unsigned char *>(a);
  }
};

template <int KP>
__host__ __device__ constexpr int ws_listcap() { return KP > 64 ? KP : 64; }

template <int KP>
__host__ __device__ size_t ws_consumer_bytes(int k) {
  return PointSmem::bytes(k, KP, false, 0, ws_listcap<KP>());
}

// Producer block scan of one int per thread (128 threads).
__device__ __forceinline__ int pscan(int v, int &excl, int *ws) {
  const int pt = threadIdx.x - kThreads, lane = pt & 31, wid = pt >> 5;
  const int inc = warp_incl_scan(v);
  if (lane == 31) ws[wid] = inc;
  pbar();
  int base = 0, tot = 0;
#pragma unroll
  for (int w = 0; w < kProd / 32; ++w) {
    const int t = ws[w];
    base += w < wid ? t : 0;
    tot += t;
  }
  excl = base + inc - v;
  pbar();
  return tot;
}

// Split 8 FP32 values into BF16 h / m / l rows of the three part tiles.
__device__ __forceinline__ void store_split8w(unsigned char *t, uint32_t off, const float *z) {
  uint32_t h[4], m[4], l[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    __nv_bfloat16 a[2], b[2], c[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const float x = z[2 * i + u];
      a[u] = __float2bfloat16_rn(x);
      const float r1 = x - __bfloat162float(a[u]);
      b[u] = __float2bfloat16_rn(r1);
      c[u] = __float2bfloat16_rn(r1 - __bfloat162float(b[u]));
    }
    h[i] = (uint32_t)__bfloat16_as_ushort(a[0]) | ((uint32_t)__bfloat16_as_ushort(a[1]) << 16);
    m[i] = (uint32_t)__bfloat16_as_ushort(b[0]) | ((uint32_t)__bfloat16_as_ushort(b[1]) << 16);
    l[i] = (uint32_t)__bfloat16_as_ushort(c[0]) | ((uint32_t)__bfloat16_as_ushort(c[1]) << 16);
  }
  *reinterpret_cast<uint4 *>(t + off) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4 *>(t + kTileW + off) = make_uint4(m[0], m[1], m[2], m[3]);
  *reinterpret_cast<uint4 *>(t + 2 * kTileW + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

// Add chunk-pair accumulator a into the running sum (hi, lo) with TwoSum;
// producer warps, warp q = lanes 32q..32q+31, every 16-column group.
template <int KP>
__device__ __forceinline__ void tcp_flush(TcState &st, int a) {
  using namespace tc;
  const int q = (threadIdx.x >> 5) & 3;
  const uint32_t trow = st.tbase + ((uint32_t)(32 * q) << 16);
  const uint32_t cc = (uint32_t)((2 + a) * KP);
  const bool first = st.nflushed == 0;
  float c[16], h[16], l[16];
#pragma unroll 1
  for (int ch = 0; ch < KP / 16; ++ch) {
    tmem_ld16(trow + cc + 16 * ch, c);
    if (first) {
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        h[i] = c[i];
        l[i] = 0.0f;
      }
    } else {
      tmem_ld16(trow + 16 * ch, h);
      tmem_ld16(trow + KP + 16 * ch, l);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float t = __fadd_rn(h[i], c[i]);
        const float bv = __fsub_rn(t, h[i]);
        const float e = __fadd_rn(__fsub_rn(h[i], __fsub_rn(t, bv)), __fsub_rn(c[i], bv));
        h[i] = t;
        l[i] = __fadd_rn(l[i], e);
      }
    }
    tmem_st16(trow + 16 * ch, h);
    tmem_st16(trow + KP + 16 * ch, l);
  }
  tmem_wait_st();
  st.nflushed++;
}

// One chunk of cnt <= 32 window entries from f on the tensor cores, plus b and
// (do_pf) the log-likelihood of member m = producer thread.  Producer warps.
template <int KP>
__device__ __forceinline__ void tcp_chunk(const ProdSmem &P, const ObsView &ob, WsCtl &ctl, TcState &st, int f,
                                          int cnt, int k, bool do_pf, double &bacc, double &llacc, int &bits) {
  using namespace tc;
  const int m = threadIdx.x - kThreads;
  const int s = st.nchunk & 1;
  if (m == 0) {  // the stage's previous UMMAs must be done
    if (!st.broken && st.uses[s] > 0 && !mbar_wait(&ctl.mma[s], (uint32_t)((st.uses[s] - 1) & 1))) {
      bits |= SBLETKF_ERR_TIMEOUT;
      ctl.brk_p = 1;
    } else {
      ctl.brk_p = st.broken;
    }
  }
  if (m < kKCw) P.sw[m] = m < cnt ? (float)sqrt(P.wlw[f + m]) : 0.0f;
  float y[kKCw];
#pragma unroll
  for (int cc = 0; cc < kKCw; ++cc)
    y[cc] = (m < KP && cc < cnt) ? ob.hdxf32[(long)P.wlidx[f + cc] * ob.ldh + m] : 0.0f;
  pbar();
  st.broken = ctl.brk_p;
  if (!st.broken && (st.nchunk & 1) && st.nchunk >= 3) {  // pair (nchunk - 3) / 2 is complete
    fence_after_sync();
    tcp_flush<KP>(st, ((st.nchunk >> 1) + 1) & 1);
    fence_before_sync();
  }
  if (m < k) {
#pragma unroll
    for (int cc = 0; cc < kKCw; ++cc)
      if (cc < cnt) bacc = fma(P.wlwd[f + cc], (double)y[cc], bacc);
    if (do_pf) {  // common_lpfgm.f90:64-69, serial in obs order, no contraction
#pragma unroll
      for (int cc = 0; cc < kKCw; ++cc) {
        if (cc < cnt) {
          const double d = __dsub_rn(P.wldep[f + cc], (double)y[cc]);
          double q = __dmul_rn(__dmul_rn(0.5, d), d);
          q = __ddiv_rn(__dmul_rn(q, P.wlrloc[f + cc]), P.wlrdiag[f + cc]);
          llacc = __dsub_rn(llacc, q);
        }
      }
    }
  }
  unsigned char *stg = P.stage + s * kStageW;
#pragma unroll
  for (int g = 0; g < kKCw / 8; ++g) {
    float z[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) z[i] = P.sw[g * 8 + i] * y[g * 8 + i];
    store_split8w(stg, tile_off(m, g * 8), z);
  }
  fence_async_smem();
  pbar();
  if (m == 0 && !st.broken) {
    fence_after_sync();
    const uint32_t idesc = idesc_bf16(kM, KP);
    const uint32_t a0 = smem_u32(stg);
    const uint32_t d = st.tbase + (uint32_t)((2 + ((st.nchunk >> 1) & 1)) * KP);
#pragma unroll
    for (int kb = 0; kb < kKCw / kKB; ++kb) {
      const uint64_t dh = sdesc(a0 + kb * kBlockBytes), dm = sdesc(a0 + kTileW + kb * kBlockBytes),
                     dl = sdesc(a0 + 2 * kTileW + kb * kBlockBytes);
      const uint32_t acc = (kb > 0 || (st.nchunk & 1)) ? 1u : 0u;  // each pair starts its accumulator afresh
      mma_bf16(d, dh, dh, idesc, acc);  // H^T H
      mma_bf16(d, dh, dm, idesc, 1u);   // H^T M
      mma_bf16(d, dm, dh, idesc, 1u);   // M^T H
      mma_bf16(d, dh, dl, idesc, 1u);   // H^T L
      mma_bf16(d, dl, dh, idesc, 1u);   // L^T H
      mma_bf16(d, dm, dm, idesc, 1u);   // M^T M
    }
    commit_to(&ctl.mma[s]);
  }
  if (!st.broken) st.issued[s] = st.uses[s] + 1;
  st.uses[s]++;
  st.nchunk++;
}

// Wait for the point's last UMMAs and add the pairs not yet flushed into the
// running sum; the Gram is then hi + lo in tensor memory.  Producer warps.
template <int KP>
__device__ __forceinline__ void tcp_finish(WsCtl &ctl, TcState &st, int &bits) {
  using namespace tc;
  if (threadIdx.x == kThreads) {
    int brk = st.broken;
    for (int s = 0; s < 2; ++s)
      if (!brk && st.uses[s] > 0 && !mbar_wait(&ctl.mma[s], (uint32_t)((st.uses[s] - 1) & 1))) {
        bits |= SBLETKF_ERR_TIMEOUT;
        brk = 1;
      }
    ctl.brk_p = brk;
  }
  pbar();
  st.broken = ctl.brk_p;
  fence_after_sync();
  if (!st.broken)
    for (int pr = st.nflushed; pr <= ((st.nchunk - 1) >> 1); ++pr) tcp_flush<KP>(st, pr & 1);
  fence_before_sync();
}

// G + alpha I = hi + lo + alpha I from tensor memory into B (FP64, column-major,
// stride ldb; lower triangle read and mirrored).  Consumer warps.
template <int KP>
__device__ __forceinline__ void tc_extract(const PointSmem &S, uint32_t tbase, int k, double alpha) {
  using namespace tc;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int q = wid & 3, half = wid >> 2, r = 32 * q + lane;
  const uint32_t trow = tbase + ((uint32_t)(32 * q) << 16);
  double *B = S.u;
  float vh[16], vl[16];
  for (int ch = half; ch < KP / 16; ch += 2) {
    tmem_ld16(trow + 16 * ch, vh);
    tmem_ld16(trow + KP + 16 * ch, vl);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const int c = 16 * ch + i;
      if (r < k && c <= r) {
        const double gv = (double)vh[i] + (double)vl[i] + (r == c ? alpha : 0.0);
        B[(long)c * S.ldb + r] = gv;
        B[(long)r * S.ldb + c] = gv;
      }
    }
  }
  fence_before_sync();
}

template <int R, typename ST, bool MIXED>
__global__ void __launch_bounds__(kWsThreads, 1)
    k_analysis_ws(const sbletkf_params p, const GridView g, const ObsView ob, const ST *__restrict__ f3,
                  const ST *__restrict__ f2, ST *__restrict__ a3, ST *__restrict__ a2,
                  const double *__restrict__ uni, int32_t *__restrict__ src_out, int32_t *__restrict__ pst,
                  int *status, int *queue, double *slab, int32_t *list_idx, double *list_rloc, long long list_cap,
                  int colchunk, int cstride) {
  constexpr int KP = kp_of_r(R);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ WsCtl ctl;
  const int k = p.nmem;
  const int tid = threadIdx.x;
  const bool do_pf = p.iswitch_da != SBLETKF_DA_LETKF;
  const int ndm = PointSmem::dual_max(k);
  const int nij1 = g.nij1;
  PointSmem S;
  S.carve(smem_raw, k, KP, 0, ws_listcap<KP>());
  ProdSmem P;
  P.carve(smem_raw + ws_consumer_bytes<KP>(k), KP);
  int32_t *gl_idx[2];
  double *gl_rloc[2];
  for (int s = 0; s < 2; ++s) {
    gl_idx[s] = list_idx + ((long long)blockIdx.x * 2 + s) * list_cap;
    gl_rloc[s] = list_rloc + ((long long)blockIdx.x * 2 + s) * list_cap;
  }

  // A launch that finds SBLETKF_ERR_TIMEOUT latched allocates no tensor
  // memory; its producer marks every point it takes as aborted.
  if (tid == 0) {
    ctl.abort = 0;
    ctl.brk_p = 0;
    ctl.ok_p = 1;
    for (int s = 0; s < 2; ++s) {
      tc::mbar_init(&ctl.full[s], 1);
      tc::mbar_init(&ctl.empty[s], 1);
      tc::mbar_init(&ctl.mma[s], 1);
    }
    tc::mbar_init(&ctl.tmem_free, 1);
    ctl.ok_c = (*(volatile int *)status & SBLETKF_ERR_TIMEOUT) == 0;
  }
  __syncthreads();
  const bool tc_on = MIXED && ctl.ok_c != 0;
  if (tc_on && (tid >> 5) == kThreads / 32) tc::tmem_alloc(&ctl.tmem, tc_cols<KP>());
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = ctl.tmem;
  volatile int *abort = &ctl.abort;

  if (tid >= kThreads) {
    // =========================== producer ===========================
    // registers: kRegProd per producer thread, kRegCons per consumer thread
    // (the launch's 384 x kRegLaunch in all)
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(kRegProd));
    const int pt = tid - kThreads;
    TcState st;
    st.tbase = tbase;
    st.uses[0] = st.uses[1] = 0;
    st.issued[0] = st.issued[1] = 0;
    st.broken = 0;
    st.nchunk = 0;
    st.nflushed = 0;
    const double tc_max = p.tc_max_cand > 0.0 ? p.tc_max_cand : (double)tc::kMaxCand;
    int seq = 0, ntc = 0;
    int c0 = 0, w = 0, pos = 0, npos = 0;
    for (;;) {
      long long pid = -1;
      int flags = 0;
      if (pos == npos) {  // next item from the queue
        if (pt == 0) ctl.item = atomicAdd(queue, 1);
        pbar();
        const long long q = ctl.item, band = q / cstride;
        const long long cs = band * colchunk * cstride + (q - band * cstride);
        pbar();
        if (cs < nij1) {
          const long long left = (nij1 - cs + cstride - 1) / cstride;
          c0 = (int)cs;
          w = (int)(left < colchunk ? left : colchunk);
          pos = 0;
          npos = w * p.nlev;
          flags |= kFNewItem;
        }
      }
      if (pos < npos) {
        const int j = pos / p.nlev, r = pos - j * p.nlev;
        const int kl = (j & 1) ? r : p.nlev - 1 - r;  // surface-down first, then bottom-up, ...
        ++pos;
        pid = (long long)kl * nij1 + c0 + (long long)j * cstride;
      }
      const int s = seq & 1;
      if (seq >= 2) {  // the consumer has finished with this slot's previous point
        if (pt == 0) {
          const bool ok = ws_wait(&ctl.empty[s], (uint32_t)(((seq >> 1) - 1) & 1), abort);
          if (!ok && !*abort) {
            *abort = 1;
            atomicOr(status, SBLETKF_ERR_TIMEOUT);
          }
          P.ws[7] = ok;  // one decision for every producer thread
        }
        pbar();
        if (!P.ws[7]) break;
      }
      if (pid < 0) {  // the queue is exhausted: tell the consumer
        if (pt == 0) {
          ctl.flags[s] = kFEnd;
          mbar_arrive(&ctl.full[s]);
        }
        break;
      }
      int bits = 0, nacc = 0;
      bool primal = false, use_tc = false;
      double bacc = 0.0, llacc = 0.0;
      // mixed path: after a timeout anywhere in the launch, later points are only marked
      if (pt == 0) P.ws[8] = MIXED && ((*(volatile int *)status & SBLETKF_ERR_TIMEOUT) != 0 || !tc_on);
      pbar();
      if (P.ws[8]) {
        flags |= kFAbort;
      } else {
        const int kl = (int)(pid / nij1), i = (int)(pid % nij1);
        // ---- search box and its grid rows (common_da.f90:158-161, 314-346)
        if (pt == 0) {
          int imin, imax, jmin, jmax;
          search_box(p, g, i, imin, imax, jmin, jmax);
          int nrows = jmax - jmin + 1;
          if (nrows < 0) nrows = 0;
          P.ws[9] = 0;
          if (nrows > kRowMax) {
            nrows = kRowMax;
            P.ws[9] = SBLETKF_ERR_ROWS;
          }
          P.ws[10] = imin;
          P.ws[11] = imax;
          P.ws[12] = jmin;
          P.ws[13] = nrows;
        }
        pbar();
        bits |= P.ws[9];
        const int imin = P.ws[10], imax = P.ws[11], jmin = P.ws[12], nrows = P.ws[13];
        const double rdep = g.depth1[pid], plon = g.lon1[i], plat = g.lat1[i];
        {
          constexpr int RPT = kRowMax / kProd;
          int lens[RPT], loc = 0;
#pragma unroll
          for (int t = 0; t < RPT; ++t) {
            const int r = pt * RPT + t;
            lens[t] = 0;
            if (r < nrows) {
              const int j = jmin + r;
              const int st0 = ob.cellstart[(long)(j - 1) * p.nlon + (imin - 1)];
              const int en = ob.cellstart[(long)(j - 1) * p.nlon + imax];
              P.rowstart[r] = st0;
              lens[t] = en > st0 ? en - st0 : 0;
              loc += lens[t];
            }
          }
          int excl;
          const int tot = pscan(loc, excl, P.ws);
#pragma unroll
          for (int t = 0; t < RPT; ++t) {
            const int r = pt * RPT + t;
            if (r < nrows) {
              P.rowpref[r] = excl;
              excl += lens[t];
            }
          }
          if (pt == 0) P.rowpref[nrows] = tot;
          pbar();
        }
        const int ncand = P.rowpref[nrows];
        use_tc = tc_on && (double)ncand <= tc_max;
        // ---- streaming selection in the reference's candidate order
        int Lw = 0;
        bool held = false, stop = false;
        for (int base = 0; base < ncand; base += kProd) {
          const int c = base + pt;
          int accept = 0, o = 0;
          double rl = 0.0;
          if (c < ncand) {
            int lo = 0, hi = nrows - 1;
            while (lo < hi) {
              const int mid = (lo + hi + 1) >> 1;
              if (P.rowpref[mid] <= c) lo = mid;
              else hi = mid - 1;
            }
            o = P.rowstart[lo] + (c - P.rowpref[lo]);
            const double dl = dlev_of(ob.elm[o], ob.lev[o], rdep, kl, p.nlev, p.id_z_obs);
            if (!(p.dist_zerov < dl)) {
              const double dist = distance_2p(ob.lon[o], ob.lat[o], plon, plat, p.pi, p.re);
              if (!(p.dist_zero < dist)) {
                accept = 1;
                rl = loc_weight(dist, dl, p.sigma_obs, p.sigma_obsv);
              }
            }
          }
          int excl;
          const int tot = pscan(accept, excl, P.ws);
          if (accept) {
            const long long gq = (long long)nacc + excl;
            if (!use_tc || gq <= ndm) {  // the consumer reads these back
              gl_idx[s][gq] = o;
              gl_rloc[s][gq] = rl;
            }
            if (use_tc) {
              const int q = Lw + excl;
              const double rd = ob.rdiag[o], dp = ob.dep[o];
              P.wlidx[q] = o;
              P.wlrloc[q] = rl;
              P.wlrdiag[q] = rd;
              P.wldep[q] = dp;
              const double wq = rl / rd;
              P.wlw[q] = wq;
              P.wlwd[q] = wq * dp;
            }
          }
          nacc += tot;
          if (use_tc) Lw += tot;
          pbar();
          if (!primal && nacc > ndm) primal = true;
          if (use_tc && primal) {
            if (!held) {  // the consumer must have read the previous Gram out of tensor memory
              if (ntc > 0) {
                if (pt == 0) {
                  const bool ok = ws_wait(&ctl.tmem_free, (uint32_t)((ntc - 1) & 1), abort);
                  if (!ok && !*abort) {
                    *abort = 1;
                    atomicOr(status, SBLETKF_ERR_TIMEOUT);
                  }
                  P.ws[7] = ok;
                }
                pbar();
                if (!P.ws[7]) {
                  stop = true;
                  break;
                }
                tc::fence_after_sync();
              }
              held = true;
              st.nchunk = 0;
              st.nflushed = 0;
            }
            int f = 0;
            while (Lw - f >= kKCw) {
              tcp_chunk<KP>(P, ob, ctl, st, f, kKCw, k, do_pf, bacc, llacc, bits);
              f += kKCw;
            }
            const int rem = Lw - f;
            if (f > 0 && rem > 0) {  // move the rest to the front of the window
              double a = 0.0, b = 0.0, c2 = 0.0, d2 = 0.0, e = 0.0;
              int ix = 0;
              if (pt < rem) {
                ix = P.wlidx[f + pt];
                a = P.wlrloc[f + pt];
                b = P.wlrdiag[f + pt];
                c2 = P.wldep[f + pt];
                d2 = P.wlw[f + pt];
                e = P.wlwd[f + pt];
              }
              pbar();
              if (pt < rem) {
                P.wlidx[pt] = ix;
                P.wlrloc[pt] = a;
                P.wlrdiag[pt] = b;
                P.wldep[pt] = c2;
                P.wlw[pt] = d2;
                P.wlwd[pt] = e;
              }
            }
            Lw = rem;
            pbar();
          }
        }
        if (stop) break;
        if (use_tc && primal) {
          if (Lw > 0) tcp_chunk<KP>(P, ob, ctl, st, 0, Lw, k, do_pf, bacc, llacc, bits);
          tcp_finish<KP>(ctl, st, bits);
          if (pt < KP) {
            P.pb[s * KP + pt] = pt < k ? bacc : 0.0;
            P.pll[s * KP + pt] = pt < k ? llacc : 0.0;
          }
          ++ntc;
          flags |= kFTc;
        }
        if (primal) flags |= kFPrimal;
      }
      // the producer's bits of the point: OR over its threads (only thread 0
      // latches timeouts, every thread may see ERR_ROWS)
      if (pt == 0) P.ws[14] = 0;
      pbar();
      if (bits) atomicOr(&P.ws[14], bits);
      pbar();
      if (pt == 0) {
        ctl.pid[s] = pid;
        ctl.nacc[s] = nacc;
        ctl.flags[s] = flags;
        ctl.bits[s] = P.ws[14];
        tc::fence_before_sync();
        mbar_arrive(&ctl.full[s]);
      }
      ++seq;
    }
    // drain: a timed-out UMMA wait may have left commits in flight
    if (tc_on && st.broken && pt == 0) {
      int ok = 1;
      for (int s = 0; s < 2; ++s)
        if (st.issued[s] > 0 && !tc::mbar_wait(&ctl.mma[s], (uint32_t)((st.issued[s] - 1) & 1), tc::kDrainLimit))
          ok = 0;
      if (!ok) atomicOr(status, SBLETKF_ERR_TIMEOUT);
      ctl.ok_p = ok;
    } else if (pt == 0) {
      ctl.ok_p = 1;
    }
  } else {
    // =========================== consumer ===========================
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(kRegCons));
    double *vprev = slab + (size_t)blockIdx.x * k * k;
    const double alpha = (double)(k - 1) / (p.iswitch_da == SBLETKF_DA_LETKF ? p.cov_infl_mul : p.cov_infl_gm);
    int warm = 0;
    for (int seq = 0;; ++seq) {
      const int s = seq & 1;
      if (tid == 0) {
        const bool ok = ws_wait(&ctl.full[s], (uint32_t)((seq >> 1) & 1), abort);
        if (!ok && !*abort) {
          *abort = 1;
          atomicOr(status, SBLETKF_ERR_TIMEOUT);
        }
        ctl.ok_c = ok;
      }
      cta_sync();
      if (!ctl.ok_c) break;
      tc::fence_after_sync();
      const int flags = ctl.flags[s];
      if (flags & kFEnd) break;
      const long long pid = ctl.pid[s];
      const int nacc = ctl.nacc[s];
      int bits = ctl.bits[s];
      if (flags & kFNewItem) warm = 0;
      if (flags & kFAbort) {
        if (tid == 0 && pst) pst[pid] = SBLETKF_ERR_TIMEOUT;
      } else {
        const bool primal = (flags & kFPrimal) != 0;
        const bool dual = !primal && nacc > 0;
        double llv = 0.0;
        if (primal) {
          if (flags & kFTc) {
            tc_extract<KP>(S, tbase, k, alpha);
            if (tid < KP) S.b[tid] = P.pb[s * KP + tid];
            if (tid < k) llv = P.pll[s * KP + tid];
            cta_sync();
            if (tid == 0) mbar_arrive(&ctl.tmem_free);
          } else {  // FP64 Gram from the list, 32 observations at a time
            Accum<R> A;
            A.zero();
            for (int f = 0; f < nacc; f += kChunk) {
              const int cnt = min(kChunk, nacc - f);
              if (tid < cnt) {
                const int o = gl_idx[s][f + tid];
                const double rl = gl_rloc[s][f + tid], rd = ob.rdiag[o], dp = ob.dep[o];
                S.lidx[tid] = o;
                S.lrloc[tid] = rl;
                S.lrdiag[tid] = rd;
                S.ldep[tid] = dp;
                const double wq = rl / rd;
                S.lw[tid] = wq;
                S.lwd[tid] = wq * dp;
              }
              cta_sync();
              constexpr int KP2 = KP / 2;
              for (int e = tid; e < cnt * KP2; e += kThreads) {
                const int cc = e / KP2, col = e - cc * KP2;
                reinterpret_cast<double2 *>(S.u)[e] =
                    reinterpret_cast<const double2 *>(ob.hdxf64 + (long)S.lidx[cc] * ob.ldh)[col];
              }
              cta_sync();
              accumulate_chunk<R>(S, 0, cnt, k, true, do_pf, A);
            }
            store_gram<R>(S, k, alpha, A);
            llv = A.ll;
          }
        } else if (dual) {  // the list itself (<= dual_max entries)
          if (tid < nacc) {
            const int o = gl_idx[s][tid];
            const double rl = gl_rloc[s][tid], rd = ob.rdiag[o], dp = ob.dep[o];
            S.lidx[tid] = o;
            S.lrloc[tid] = rl;
            S.lrdiag[tid] = rd;
            S.ldep[tid] = dp;
            const double wq = rl / rd;
            S.lw[tid] = wq;
            S.lwd[tid] = wq * dp;
          }
          cta_sync();
        }
        const int i = (int)(pid % nij1);
        point_tail<R, ST, true>(p, ob, f3, f2, a3, a2, uni, src_out, pst, status, S, pid, nij1, g.phi1[i], nacc, dual,
                          llv, bits, tc_on, vprev, warm);
      }
      cta_sync();
      if (tid == 0) mbar_arrive(&ctl.empty[s]);
    }
  }
  __syncthreads();
  if (tc_on && (tid >> 5) == kThreads / 32 && ctl.ok_p) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tbase, tc_cols<KP>());
  }
}

template <int R, typename ST, bool MIXED>
int launch_ws_r(const sbletkf_params *p, const GridView &g, const ObsView &ob, const void *f3, const void *f2,
                void *a3, void *a2, const double *uni, int32_t *src, int32_t *pst, sbletkf_workspace *ws,
                cudaStream_t s) {
  constexpr int KP = kp_of_r(R);
  const size_t smem = ws_consumer_bytes<KP>(p->nmem) + ProdSmem::bytes(KP);
  auto kern = k_analysis_ws<R, ST, MIXED>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_status(e);
  const int colchunk = queue_item_width(ws, g.nij1, ws->nslab);
  const int cstride = p->nlon > 1 ? p->nlon : 1;
  e = cudaMemsetAsync(ws->d_queue, 0, sizeof(int), s);
  if (e != cudaSuccess) return cuda_status(e);
  kern<<<(unsigned)ws->nslab, kWsThreads, smem, s>>>(*p, g, ob, (const ST *)f3, (const ST *)f2, (ST *)a3, (ST *)a2,
                                                      uni, src, pst, ws->d_status, ws->d_queue, ws->d_slab,
                                                      ws->d_list_idx, ws->d_list_rloc, ws->list_cap, colchunk,
                                                      cstride);
  return cuda_status(cudaGetLastError());
}

template <typename ST>
int launch_ws_t(const sbletkf_params *p, const GridView &g, const ObsView &ob, const void *f3, const void *f2,
                void *a3, void *a2, const double *uni, int32_t *src, int32_t *pst, sbletkf_workspace *ws,
                cudaStream_t s) {
  const bool mixed = p->precision == SBLETKF_PREC_MIXED;
  switch (r_for_k(p->nmem)) {
    case 2: return mixed ? launch_ws_r<2, ST, true>(p, g, ob, f3, f2, a3, a2, uni, src, pst, ws, s)
                         : launch_ws_r<2, ST, false>(p, g, ob, f3, f2, a3, a2, uni, src, pst, ws, s);
    case 4: return mixed ? launch_ws_r<4, ST, true>(p, g, ob, f3, f2, a3, a2, uni, src, pst, ws, s)
                         : launch_ws_r<4, ST, false>(p, g, ob, f3, f2, a3, a2, uni, src, pst, ws, s);
    default: return mixed ? launch_ws_r<7, ST, true>(p, g, ob, f3, f2, a3, a2, uni, src, pst, ws, s)
                          : launch_ws_r<7, ST, false>(p, g, ob, f3, f2, a3, a2, uni, src, pst, ws, s);
  }
}

}  // namespace

bool pipeline_supported(const sbletkf_params *p) {
  return p->iswitch_da != SBLETKF_DA_LPF && r_for_k(p->nmem) <= 7;
}

int launch_analysis_ws(sbletkf_workspace *ws, const sbletkf_params *p, const GridView &g, const void *f3,
                       const void *f2, void *a3, void *a2, int dtype, const double *uni, int32_t *src, int32_t *pst,
                       cudaStream_t s) {
  const ObsView ob = ws->obs_view();
  if (dtype == SBLETKF_F64) return launch_ws_t<double>(p, g, ob, f3, f2, a3, a2, uni, src, pst, ws, s);
  return launch_ws_t<float>(p, g, ob, f3, f2, a3, a2, uni, src, pst, ws, s);
}

}  // namespace sbl
