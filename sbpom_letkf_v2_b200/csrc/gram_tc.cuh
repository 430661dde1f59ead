// gram_tc.cuh -- the local Gram Y^T diag(rloc/rdiag) Y on the 5th-generation
// tensor cores (tcgen05, sm_100a), split-precision BF16.
//
// With z_o = sqrt(rloc_o/rdiag_o) y_o the Gram is G = Z^T Z.  Each FP32 row is
// split three ways, z = h + m + l with h = bf16(z), m = bf16(z - h),
// l = bf16(z - h - m) (24 significant bits, all of FP32), and
//   G ~= H^T H + H^T M + M^T H + H^T L + L^T H + M^T M,
// six UMMAs per K-block into an FP32 chunk accumulator in tensor memory; the
// dropped terms (M^T L, L^T M, L^T L) are below 2^-24 of G.  Transposed pairs
// are separate UMMAs (A and B swapped), so the accumulator needs no transpose.
// Each pair of chunks (2 x 64 observations) has its own accumulator, which
// the CTA adds into a running double-FP32 sum (hi + lo, error-free TwoSum)
// also held in tensor memory, so FP32 rounding stays at the scale of one
// chunk pair rather than growing with nobsl.  Tensor-memory columns: sum hi
// [0,KP), sum lo [KP,2KP), chunk-pair accumulators [2KP,3KP) and [3KP,4KP).
// (common_letkf.f90:93-122 computes the same Gram with sgemm/dgemm.)
//
// Operand tile: rows = members (M = 128, zero-padded), K = observations, in the
// K-major canonical layout without swizzle: 8x8 "core matrices" of 8 rows x 16
// bytes; element (row r, k) of a 16-wide K block lives at
//   (r/8)*256 + ((k%16)/8)*128 + (r%8)*16 + (k%8)*2     (LBO = 128, SBO = 256),
// one K block of 128 rows = 4096 bytes.  Z^T (A, M x K) and Z (B, K x N) are the
// same tile, so one descriptor serves both operands.
#pragma once

#include <cuda_bf16.h>

#include "internal.cuh"

namespace sbl {
namespace tc {

constexpr int kM = 128;            // UMMA M (members, zero padded)
constexpr int kKC = 64;            // observations per staged chunk (4 K-blocks)
constexpr int kKB = 16;            // UMMA K for kind::f16
constexpr int kBlockBytes = kM * kKB * 2;             // one 16-wide K block, 4096 B
constexpr int kTileBytes = kBlockBytes * (kKC / kKB);  // one chunk of one split part: 16 KB
constexpr int kSplit = 3;                              // h, m, l
constexpr int kStageBytes = kSplit * kTileBytes;
constexpr unsigned kWaitLimit = 1u << 20;              // bounded mbarrier polls
constexpr unsigned kDrainLimit = 1u << 26;             // polls of the drain before TMEM is freed
// Largest search-box candidate count whose Gram goes to the tensor cores: the
// FP32 accumulator's rounding grows like eps32 sqrt(n/16) |G|, which must stay
// well below alpha = (k-1)/rho for the eigensolve; denser points use FP64.
constexpr int kMaxCand = 12288;

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// tcgen05 shared-memory matrix descriptor (no swizzle, K-major).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr & 0x3FFFFu) >> 4);            // start address  [0,14)
  d |= (uint64_t)((128u >> 4) & 0x3FFFu) << 16;       // LBO = 128 B    [16,30)
  d |= (uint64_t)((256u >> 4) & 0x3FFFu) << 32;       // SBO = 256 B    [32,46)
  d |= (uint64_t)1 << 46;                             // descriptor version 1 [46,48)
  return d;                                           // base 0, layout SWIZZLE_NONE
}

// Instruction descriptor, kind::f16: D F32, A/B BF16, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t *dst_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols));
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void mma_bf16(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
      "l"(a), "l"(b), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void commit_to(uint64_t *mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

// Wait for phase `parity` of an mbarrier; false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, unsigned limit = kWaitLimit) {
  const uint32_t a = smem_u32(mbar);
  for (unsigned it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Store 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float *v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          taddr),
      "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])), "r"(__float_as_uint(v[3])),
      "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])), "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])),
      "r"(__float_as_uint(v[8])), "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])),
      "r"(__float_as_uint(v[11])), "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])),
      "r"(__float_as_uint(v[14])), "r"(__float_as_uint(v[15]))
      : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Byte offset of (row, k) inside one chunk tile (k in [0, kKC)).
__device__ __forceinline__ uint32_t tile_off(int row, int k) {
  return (uint32_t)((k >> 4) * kBlockBytes + (row >> 3) * 256 + ((k >> 3) & 1) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Split 8 FP32 values into BF16 h / m / l and store them as 16-byte rows of
// the three tiles (tile j at t + j * kTileBytes).
__device__ __forceinline__ void store_split8(unsigned char *t, uint32_t off, const float *z) {
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
  *reinterpret_cast<uint4 *>(t + kTileBytes + off) = make_uint4(m[0], m[1], m[2], m[3]);
  *reinterpret_cast<uint4 *>(t + 2 * kTileBytes + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

}  // namespace tc
}  // namespace sbl
