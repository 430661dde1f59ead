// tc_point.cuh -- the local Gram of one point on the tensor cores (tcgen05):
// the CTA-side pipeline around gram_tc.cuh's operand tiles and UMMAs, shared
// by the analysis kernel (rows gathered from the sorted observations) and the
// ragged-batch core (rows from the caller's Fortran hdxf blocks).
//
// Per 64-observation chunk: stage FP32 rows, scale by sqrt(rloc/rdiag), split
// into BF16 h/m/l tiles, issue six UMMAs per 16-wide K block into a chunk-pair
// FP32 accumulator in tensor memory, and add finished pairs into a running
// double-FP32 (TwoSum) sum; b = Y^T diag(w) dep and the PF log-likelihood
// are accumulated on the side in FP64.  Replaces the Gram of letkf_core
// (common_letkf.f90:93-122).
#pragma once

#include "point.cuh"

namespace sbl {

// State of the tensor-core Gram pipeline of one CTA (uniform across threads).
struct TcState {
  uint32_t tbase;   // TMEM base: sum hi, sum lo, chunk accumulators 0 and 1 (KP columns each)
  int uses[2];      // chunks staged per operand stage (commit index of the next chunk)
  int issued[2];    // commits actually issued per operand stage
  int nchunk;
  int nflushed;     // chunk pairs added into the running sum
  int broken;       // a wait timed out: issue nothing more
};

// Add chunk accumulator a (0, 1) into the running double-FP32 sum with
// Knuth's TwoSum (hi + c = s_ + e exactly; lo += e).  Whole CTA: warp w owns
// TMEM lanes 32 (w % 4) .. +31 and half w / 4 of the 16-column groups.
template <int KP>
__device__ __forceinline__ void tc_flush(TcState &st, int s) {
  using namespace tc;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  (void)lane;
  const int q = wid & 3, half = wid >> 2;
  const uint32_t trow = st.tbase + ((uint32_t)(32 * q) << 16);
  const uint32_t cc = (uint32_t)((2 + s) * KP);
  const bool first = st.nflushed == 0;
  float c[16], h[16], l[16];
  for (int ch = half; ch < KP / 16; ch += 2) {
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

// Stage `cnt` list entries starting at f as BF16 h/m/l operand tiles and issue
// their six UMMAs per K-block.  Chunks 2p and 2p+1 share chunk accumulator
// p % 2 (FP32 over 128 observations); at chunk 2p+3, whose entry wait on
// stage 1 covers chunk 2p+1's UMMAs, pair p is added into the running sum,
// before chunk 2p+4 starts that accumulator afresh.  Also
// accumulates b = sum w dep y (FP64) and, when do_pf, the PF log-likelihood.
// Whole CTA; ends with the tiles handed to the tensor core.
// `rows(stg, f, cnt)` fills the FP32 staging rows stg[kKC][KP] with the
// chunk's observations (rows cc >= cnt and members >= k zero); whole CTA,
// no barrier.
template <int KP, typename RowLoader>
__device__ __forceinline__ void tc_chunk(const PointSmem &S, const RowLoader &rows, TcState &st, uint64_t *mbar,
                                         int f, int cnt, int k, bool do_pf, double &bacc, double &llacc,
                                         int &bits) {
  using namespace tc;
  const int tid = threadIdx.x;
  const int s = st.nchunk & 1;
  float *stg = reinterpret_cast<float *>(S.u);  // [kKC][KP] FP32 rows
  unsigned char *tiles = reinterpret_cast<unsigned char *>(S.u) + PointSmem::tc_tiles_off(KP);
  unsigned char *stage = tiles + s * kStageBytes;
  float *sw = reinterpret_cast<float *>(S.cw);
  __shared__ int s_broken;
  if (tid == 0) {  // the stage's previous UMMAs must be done
    if (!st.broken && st.uses[s] > 0 && !mbar_wait(&mbar[s], (uint32_t)((st.uses[s] - 1) & 1))) {
      bits |= SBLETKF_ERR_TIMEOUT;
      s_broken = 1;
    } else {
      s_broken = st.broken;
    }
  }
  rows(stg, f, cnt);
  if (tid < kKC) sw[tid] = tid < cnt ? (float)sqrt(S.lw[f + tid]) : 0.0f;
  cta_sync();
  st.broken = s_broken;
  if (!st.broken && (st.nchunk & 1) && st.nchunk >= 3) {  // pair (nchunk - 3) / 2 is complete: add it
    fence_after_sync();
    tc_flush<KP>(st, ((st.nchunk >> 1) + 1) & 1);
    fence_before_sync();
  }
  if (tid < KP)
    for (int cc = 0; cc < cnt; ++cc) bacc = fma(S.lwd[f + cc], (double)stg[cc * KP + tid], bacc);
  if (do_pf && tid < k) {
    for (int cc = 0; cc < cnt; ++cc) {
      double d = __dsub_rn(S.ldep[f + cc], (double)stg[cc * KP + tid]);
      double q = __dmul_rn(__dmul_rn(0.5, d), d);
      q = __ddiv_rn(__dmul_rn(q, S.lrloc[f + cc]), S.lrdiag[f + cc]);
      llacc = __dsub_rn(llacc, q);
    }
  }
  for (int e = tid; e < kM * (kKC / 8); e += kThreads) {
    const int m = e & (kM - 1), g = e >> 7;
    float z[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int o = g * 8 + i;
      z[i] = m < KP ? sw[o] * stg[o * KP + m] : 0.0f;
    }
    store_split8(stage, tile_off(m, g * 8), z);
  }
  fence_async_smem();
  cta_sync();
  if (tid == 0 && !st.broken) {
    fence_after_sync();
    const uint32_t idesc = idesc_bf16(kM, KP);
    const uint32_t a0 = smem_u32(stage);
#pragma unroll
    for (int kb = 0; kb < kKC / kKB; ++kb) {
      const uint64_t dh = sdesc(a0 + kb * kBlockBytes), dm = sdesc(a0 + kTileBytes + kb * kBlockBytes),
                     dl = sdesc(a0 + 2 * kTileBytes + kb * kBlockBytes);
      const uint32_t acc = (kb > 0 || (st.nchunk & 1)) ? 1u : 0u;  // each pair starts a fresh accumulator
      const uint32_t d = st.tbase + (uint32_t)((2 + ((st.nchunk >> 1) & 1)) * KP);
      mma_bf16(d, dh, dh, idesc, acc);  // H^T H
      mma_bf16(d, dh, dm, idesc, 1u);   // H^T M
      mma_bf16(d, dm, dh, idesc, 1u);   // M^T H
      mma_bf16(d, dh, dl, idesc, 1u);   // H^T L
      mma_bf16(d, dl, dh, idesc, 1u);   // L^T H
      mma_bf16(d, dm, dm, idesc, 1u);   // M^T M
    }
    commit_to(&mbar[s]);
  }
  if (!st.broken) st.issued[s] = st.uses[s] + 1;
  st.uses[s]++;
  st.nchunk++;
}

// Wait for every issued UMMA, add the pairs not yet flushed (at most two) into
// the running sum, then
// G + alpha I = hi + lo + alpha I into B (FP64, column-major, stride ldb; the
// lower triangle read and mirrored, so B is exactly symmetric) and b into S.b.
template <int KP>
__device__ __forceinline__ void tc_finish(const PointSmem &S, TcState &st, uint64_t *mbar, int k, double alpha,
                                          double bacc, int &bits) {
  using namespace tc;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  __shared__ int s_brk;
  if (tid == 0) {
    int brk = st.broken;
    for (int s = 0; s < 2; ++s)
      if (!brk && st.uses[s] > 0 && !mbar_wait(&mbar[s], (uint32_t)((st.uses[s] - 1) & 1))) {
        bits |= SBLETKF_ERR_TIMEOUT;
        brk = 1;
      }
    s_brk = brk;
  }
  cta_sync();
  st.broken = s_brk;
  fence_after_sync();
  if (!st.broken)
    for (int pr = st.nflushed; pr <= ((st.nchunk - 1) >> 1); ++pr) tc_flush<KP>(st, pr & 1);
  double *B = S.u;
  const int q = wid & 3, half = wid >> 2, r = 32 * q + lane;
  const uint32_t trow = st.tbase + ((uint32_t)(32 * q) << 16);
  float vh[16], vl[16];
  for (int ch = half; ch < KP / 16; ch += 2) {  // row r, columns c <= r
    tmem_ld16(trow + 16 * ch, vh);
    tmem_ld16(trow + KP + 16 * ch, vl);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const int c = 16 * ch + i;
      if (r < k && c <= r) {
        const double g = (double)vh[i] + (double)vl[i] + (r == c ? alpha : 0.0);
        B[(long)c * S.ldb + r] = g;
        B[(long)r * S.ldb + c] = g;
      }
    }
  }
  if (tid < k) S.b[tid] = bacc;
  fence_before_sync();
  cta_sync();
}

// Tensor-memory columns of one CTA: sum hi, sum lo and two chunk-pair
// accumulators of KP columns each, rounded up to an allocatable size.
template <int KP>
__host__ __device__ constexpr uint32_t tc_cols() {
  return (4 * KP <= 128) ? 128u : (4 * KP <= 256) ? 256u : 512u;
}

// Allocate the CTA's tensor memory (warp 0) and initialise the two stage
// mbarriers; whole CTA.
template <int KP>
__device__ __forceinline__ void tc_open(TcState &st, uint64_t *mbar, uint32_t *s_tmem) {
  st.uses[0] = st.uses[1] = 0;
  st.issued[0] = st.issued[1] = 0;
  st.nchunk = 0;
  st.nflushed = 0;
  st.broken = 0;
  if ((threadIdx.x >> 5) == 0) tc::tmem_alloc(s_tmem, tc_cols<KP>());
  if (threadIdx.x == 0) {
    tc::mbar_init(&mbar[0], 1);
    tc::mbar_init(&mbar[1], 1);
  }
  tc::fence_before_sync();
  cta_sync();
  tc::fence_after_sync();
  st.tbase = *s_tmem;
}

// Free the CTA's tensor memory; whole CTA.  Without a timeout every UMMA was
// waited for in tc_finish.  After a timed-out wait, committed UMMAs may still
// be writing tensor memory: thread 0 waits (bounded again) for each stage's
// last commit first.  If that wait expires too the tensor memory is not
// freed: *status gets SBLETKF_ERR_TIMEOUT, later CTAs see it and allocate
// none, and the caller should treat the device as needing a reset.
template <int KP>
__device__ __forceinline__ void tc_close(TcState &st, uint64_t *mbar, int *status) {
  __shared__ int s_free;
  if (threadIdx.x == 0) {
    int ok = 1;
    if (st.broken)
      for (int s = 0; s < 2; ++s)
        if (st.issued[s] > 0 && !tc::mbar_wait(&mbar[s], (uint32_t)((st.issued[s] - 1) & 1), tc::kDrainLimit))
          ok = 0;
    if (!ok) atomicOr(status, SBLETKF_ERR_TIMEOUT);
    s_free = ok;
  }
  tc::fence_before_sync();
  cta_sync();
  if (s_free && (threadIdx.x >> 5) == 0) {
    tc::fence_after_sync();
    tc::tmem_dealloc(st.tbase, tc_cols<KP>());
  }
}

}  // namespace sbl
