// core_batched.cu -- letkf_core / lpfgm_core over a ragged batch of local
// problems, writing wvec and the explicit transform W (unit-parity entry).
//
//   letkf_core        letkf/run/src/common_letkf.f90:61-210
//   letkf_core_noobs  letkf/run/src/common_letkf.f90:37-57
//   lpfgm_core        letkf/run/src/common_lpfgm.f90:444-494 (LPF and LPFGM)
//   lpfgm_core_noobs  letkf/run/src/common_lpfgm.f90:422-440
// Point q's inputs are the Fortran arrays hdxf(nobsl,nmem), rdiag, rloc, dep
// starting at row off[q].  W is written column-major, W(i,j) at j*k+i.
// With SBLETKF_PREC_MIXED the Gram runs on the tensor cores exactly as in the
// analysis kernel (tc_point.cuh, FP32 rows of hdxf), so W states the mixed
// path's error against letkf_core.
#include "tc_point.cuh"

namespace sbl {
namespace {

template <int R, bool MIXED>
__global__ void __launch_bounds__(kThreads, 1)
    k_core(const sbletkf_params p, const int64_t *__restrict__ off, const double *__restrict__ hdxf,
           const double *__restrict__ rdiag, const double *__restrict__ rloc, const double *__restrict__ dep,
           double *__restrict__ wvec, double *__restrict__ wmat, const double *__restrict__ uni,
           int32_t *__restrict__ src_out, int32_t *__restrict__ pst, int *status) {
  constexpr int KP = kp_of_r(R);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PointSmem S;
  const int k = p.nmem;
  S.carve(smem_raw, k, KP);
  const int tid = threadIdx.x;
  const long long q = blockIdx.x;
  const long long o0 = off[q];
  const int n = (int)(off[q + 1] - o0);
  const double *hq = hdxf + o0 * k;
  double *W = wmat + q * (long long)k * k;
  double *wv = wvec + q * (long long)k;
  const bool do_pf = p.iswitch_da != SBLETKF_DA_LETKF;
  const bool do_gram = p.iswitch_da != SBLETKF_DA_LPF;
  int bits = 0;

  Accum<R> A;
  A.zero();
  const auto fill_list = [&](int f, int cnt) {
    if (tid < cnt) {
      const long long r = o0 + f + tid;
      const double rl = rloc[r], rd = rdiag[r], dp = dep[r];
      S.lrloc[tid] = rl;
      S.lrdiag[tid] = rd;
      S.ldep[tid] = dp;
      S.lw[tid] = rl / rd;
      S.lwd[tid] = (rl / rd) * dp;
    }
  };
  __shared__ uint64_t s_mbar[2];
  __shared__ uint32_t s_tmem;
  TcState tcs;
  const bool tc_on = MIXED && do_gram;
  if (tc_on) {
    tc_open<KP>(tcs, s_mbar, &s_tmem);
    // FP32 rows of the chunk at observation f0: stg[cc][m] = hdxf(f0+cc, m)
    // (Fortran order in hq); the chunk's list entries sit at [0, cnt)
    int f0 = 0;
    const auto rows = [&](float *stg, int, int cnt) {
      for (int e = tid; e < tc::kKC * KP; e += kThreads) {
        const int m = e / tc::kKC, cc = e - m * tc::kKC;
        stg[cc * KP + m] = (m < k && cc < cnt) ? (float)hq[(long long)m * n + f0 + cc] : 0.0f;
      }
    };
    for (; f0 < n; f0 += tc::kKC) {
      const int cnt = min(tc::kKC, n - f0);
      fill_list(f0, cnt);
      __syncthreads();
      tc_chunk<KP>(S, rows, tcs, s_mbar, 0, cnt, k, do_pf, A.b, A.ll, bits);
    }
  } else {
    for (int f = 0; f < n; f += kChunk) {
      const int cnt = min(kChunk, n - f);
      fill_list(f, cnt);
      for (int e = tid; e < cnt * KP; e += kThreads) {
        const int m = e / cnt, cc = e - m * cnt;
        S.u[cc * KP + m] = m < k ? hq[(long long)m * n + f + cc] : 0.0;
      }
      __syncthreads();
      accumulate_chunk<R>(S, 0, cnt, k, do_gram, do_pf, A);
    }
  }

  if (n == 0) {
    const double d = (p.iswitch_da == SBLETKF_DA_LETKF) ? sqrt(p.cov_infl_mul) : 1.0;
    for (int e = tid; e < k * k; e += kThreads) W[e] = (e / k == e % k) ? d : 0.0;
    for (int e = tid; e < k; e += kThreads) wv[e] = 0.0;
  } else {
    if (do_gram) {
      const double alpha = (double)(k - 1) / (p.iswitch_da == SBLETKF_DA_LETKF ? p.cov_infl_mul : p.cov_infl_gm);
      if (tc_on) tc_finish<KP>(S, tcs, s_mbar, k, alpha, A.b, bits);
      else store_gram<R>(S, k, alpha, A);
      const double tol = jacobi_tol_of(p, k);
      bits |= jacobi_eig<KP / 4>(S.u, k, S.ldb, tol, jacobi_stop_of(p), p.max_sweeps, S.lam, S.iws + 40, S.lidx, S.cw);
      vt_times(S.u, k, S.ldb, S.b, S.c);
      __syncthreads();
      if (tid < k) S.c[tid] /= S.lam[tid];
      __syncthreads();
      const double *B = S.u;
      if (tid < k) {  // w = V c  (wvec for LETKF, w_gm for LPFGM)
        double s = 0.0;
        for (int j = 0; j < k; ++j) s = fma(B[(long)j * S.ldb + tid], S.c[j], s);
        S.t[tid] = s;
      }
      __syncthreads();
      const bool letkf = p.iswitch_da == SBLETKF_DA_LETKF;
      const double agm = (double)(k - 1) / p.cov_infl_gm;
      // LETKF: W = V diag(sqrt((k-1)/lambda)) V^T ; LPFGM: W_GM = w 1^T + alpha Pa
      for (int e = tid; e < k * k; e += kThreads) {
        const int jj = e / k, ii = e - jj * k;
        double s = 0.0;
        for (int j = 0; j < k; ++j) {
          const double f = letkf ? sqrt((double)(k - 1) / S.lam[j]) : 1.0 / S.lam[j];
          s = fma(B[(long)j * S.ldb + ii] * B[(long)j * S.ldb + jj], f, s);
        }
        W[e] = letkf ? s : S.t[ii] + agm * s;
      }
      if (letkf && tid < k) wv[tid] = S.t[tid];
      __syncthreads();
    }
    if (do_pf) {
      if (tid < k) S.ll[tid] = A.ll;
      __syncthreads();
      pf_weights(S, k);
      int16_t *srcb = reinterpret_cast<int16_t *>(S.u);
      const int wid = tid >> 5, lane = tid & 31;
      int *whist = reinterpret_cast<int *>(srcb + kDrawBatch * k) + wid * k;
      int16_t *wup =
          reinterpret_cast<int16_t *>(reinterpret_cast<int *>(srcb + kDrawBatch * k) + (kThreads / 32) * k) + wid * k;
      uint16_t *cnt = reinterpret_cast<uint16_t *>(S.x);  // [member j][particle i]
      for (int e = tid; e < k * k; e += kThreads) cnt[e] = 0;
      for (int d0 = 0; d0 < p.nmonte; d0 += kDrawBatch) {
        const int nb = min(kDrawBatch, p.nmonte - d0);
        __syncthreads();
        for (int t = wid; t < nb; t += kThreads / 32) {  // a warp per draw
          const int d = d0 + t;
          const double *u = (p.rm == SBLETKF_RM_SR) ? uni + q * p.nmonte + d : uni + (q * p.nmonte + d) * k;
          int16_t *sr = srcb + t * k;
          resample_draw(p, S.cw, k, u, whist, wup, sr);
          if (src_out) {
            int32_t *so = src_out + (q * p.nmonte + d) * k;
            for (int j = lane; j < k; j += 32) so[j] = sr[j];
          }
        }
        __syncthreads();
        for (int j = tid; j < k; j += kThreads)
          for (int t = 0; t < nb; ++t) cnt[j * k + srcb[t * k + j]]++;
      }
      __syncthreads();
      const double a = 1.0 / (double)p.nmonte;
      if (p.iswitch_da == SBLETKF_DA_LPF) {
        // W(i,j) = RSmat sum / nmonte accumulated draw by draw (:258-261)
        for (int e = tid; e < k * k; e += kThreads) {
          const int j = e / k, ii = e - j * k;
          double s = 0.0;
          for (int c = 0; c < cnt[j * k + ii]; ++c) s += a;
          W[e] = s;
        }
      } else {
        // W = W_GM W_LPF, row by row (W_GM is in W)
        double *row = S.lam;  // free after W_GM; S.x..S.w hold the counts
        for (int r = 0; r < k; ++r) {
          __syncthreads();
          for (int ii = tid; ii < k; ii += kThreads) row[ii] = W[(long long)ii * k + r];
          __syncthreads();
          for (int j = tid; j < k; j += kThreads) {
            double s = 0.0;
            for (int ii = 0; ii < k; ++ii) {
              double wl = 0.0;
              for (int c = 0; c < cnt[j * k + ii]; ++c) wl += a;
              s = fma(row[ii], wl, s);
            }
            W[(long long)j * k + r] = s;
          }
        }
      }
      for (int e = tid; e < k; e += kThreads) wv[e] = 0.0;
    }
  }
  if (tc_on) tc_close<KP>(tcs, s_mbar, status);
  __shared__ int s_bits;
  if (tid == 0) s_bits = 0;
  __syncthreads();
  if (bits) atomicOr(&s_bits, bits);
  __syncthreads();
  if (tid == 0) {
    if (pst) pst[q] = s_bits;
    if (s_bits) atomicOr(status, s_bits);
  }
}

template <int R>
int launch_core_r(const sbletkf_params *p, int32_t npts, const int64_t *off, const double *hdxf,
                  const double *rdiag, const double *rloc, const double *dep, double *wvec, double *wmat,
                  const double *uni, int32_t *src, int32_t *pst, int *d_status, cudaStream_t s) {
  const bool mixed = p->precision == SBLETKF_PREC_MIXED;
  const size_t smem = PointSmem::bytes(p->nmem, kp_of_r(R), mixed);
  auto kern = mixed ? k_core<R, true> : k_core<R, false>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_status(e);
  kern<<<npts, kThreads, smem, s>>>(*p, off, hdxf, rdiag, rloc, dep, wvec, wmat, uni, src, pst, d_status);
  return cuda_status(cudaGetLastError());
}

}  // namespace

int launch_core_batched(const sbletkf_params *p, int32_t npts, const int64_t *off, const double *hdxf,
                        const double *rdiag, const double *rloc, const double *dep, double *wvec, double *wmat,
                        const double *uni, int32_t *src, int32_t *pst, int *d_status, cudaStream_t s) {
  if (npts == 0) return SBLETKF_OK;
  switch (r_for_k(p->nmem)) {
    case 2: return launch_core_r<2>(p, npts, off, hdxf, rdiag, rloc, dep, wvec, wmat, uni, src, pst, d_status, s);
    case 4: return launch_core_r<4>(p, npts, off, hdxf, rdiag, rloc, dep, wvec, wmat, uni, src, pst, d_status, s);
    case 7: return launch_core_r<7>(p, npts, off, hdxf, rdiag, rloc, dep, wvec, wmat, uni, src, pst, d_status, s);
    default: return launch_core_r<8>(p, npts, off, hdxf, rdiag, rloc, dep, wvec, wmat, uni, src, pst, d_status, s);
  }
}

}  // namespace sbl
