// point.cuh -- per-grid-point building blocks shared by the analysis, core
// and backward kernels.  One CTA of kThreads threads owns one local problem.
//
//   accumulate_chunk   Gram  G += Y^T diag(rloc/rdiag) Y and b += Y^T diag(rloc/rdiag) dep
//                      (common_letkf.f90:93-122) in FP64 registers, and the PF
//                      log-likelihood (common_lpfgm.f90:64-69) in obs order
//   jacobi_eig         eigenpairs of the SPD k x k matrix A = G + (k-1)/rho I
//                      (replaces mtx_eigen / DSYEV, common.f90:992-1050):
//                      one-sided (Hestenes) cyclic Jacobi on A in shared memory,
//                      round-robin parallel ordering.  B <- A V converges to
//                      columns lambda_j v_j, so lambda_j = |b_j|, v_j = b_j/lambda_j.
//   pf_weights         max-subtracted exp, normalise, cumulative sum (serial)
//   resample_draw      SR/MR draw, inum search and diagonal-priority assignment
//                      (common_lpfgm.f90:89-197)
#pragma once

#include "internal.cuh"

namespace sbl {

// R x R register tile per thread over a 16 x 16 thread grid: k <= 16*R.
__host__ __device__ constexpr int kp_of_r(int r) { return 16 * r; }
inline int r_for_k(int k) { return k <= 32 ? 2 : k <= 64 ? 4 : k <= 112 ? 7 : 8; }

constexpr int kDrawBatch = 64;  // PF draws resolved per pass

// Shared-memory carve of one per-point CTA (all sizes in bytes, 16-aligned).
struct PointSmem {
  int *rowstart, *rowpref, *lidx, *iws;
  double *lw, *lwd, *lrloc, *lrdiag, *ldep;
  double *b, *lam, *c, *ll, *cw, *misc;
  double *x, *t, *an, *w;
  double *u;       // union: chunk rows | eigenvector matrix | PF draw buffers
  int ldb;

  __host__ __device__ static size_t a16(size_t v) { return (v + 15) & ~size_t(15); }

  // Largest nobsl that takes the observation-space (dual) transform.
  __host__ __device__ static int dual_max(int k) { return k - 1 < kDualMax ? k - 1 : kDualMax; }
  // Union size: max(chunk rows, k x ldb matrix, dual Z and N, draw buffers).
  __host__ __device__ static size_t union_bytes(int k, int kp) {
    const size_t nd = (size_t)dual_max(k);
    size_t chunk = sizeof(double) * kChunk * kp;
    size_t mat = sizeof(double) * (size_t)k * (kp + 1);
    size_t dual = sizeof(double) * (nd * (kp + 1) + nd * (nd + 1));
    size_t pf = (size_t)kDrawBatch * k * (sizeof(int16_t) + 1) + 16;
    size_t m = chunk > mat ? chunk : mat;
    m = m > dual ? m : dual;
    return a16(m > pf ? m : pf);
  }
  __host__ __device__ static size_t fixed_bytes(int kp) {
    size_t s = 0;
    s += a16(sizeof(int) * kRowMax) + a16(sizeof(int) * (kRowMax + 1)) + a16(sizeof(int) * kListCap) +
         a16(sizeof(int) * 64);
    s += 5 * a16(sizeof(double) * kListCap);
    s += 5 * a16(sizeof(double) * kp) + a16(sizeof(double) * 64);
    s += 4 * a16(sizeof(double) * kNvMax * kp);
    return s;
  }
  __host__ __device__ static size_t bytes(int k, int kp) { return fixed_bytes(kp) + union_bytes(k, kp); }

  __device__ void carve(void *base, int k, int kp) {
    char *q = (char *)base;
    auto take = [&](size_t n) { char *r = q; q += a16(n); return (void *)r; };
    rowstart = (int *)take(sizeof(int) * kRowMax);
    rowpref = (int *)take(sizeof(int) * (kRowMax + 1));
    lidx = (int *)take(sizeof(int) * kListCap);
    iws = (int *)take(sizeof(int) * 64);
    lw = (double *)take(sizeof(double) * kListCap);
    lwd = (double *)take(sizeof(double) * kListCap);
    lrloc = (double *)take(sizeof(double) * kListCap);
    lrdiag = (double *)take(sizeof(double) * kListCap);
    ldep = (double *)take(sizeof(double) * kListCap);
    b = (double *)take(sizeof(double) * kp);
    lam = (double *)take(sizeof(double) * kp);
    c = (double *)take(sizeof(double) * kp);
    ll = (double *)take(sizeof(double) * kp);
    cw = (double *)take(sizeof(double) * kp);
    misc = (double *)take(sizeof(double) * 64);
    x = (double *)take(sizeof(double) * kNvMax * kp);
    t = (double *)take(sizeof(double) * kNvMax * kp);
    an = (double *)take(sizeof(double) * kNvMax * kp);
    w = (double *)take(sizeof(double) * kNvMax * kp);
    u = (double *)q;
    ldb = kp + 1;  // odd stride: row and column walks are bank-conflict free
  }
};

// Per-thread accumulators of the streaming phase.
template <int R>
struct Accum {
  double g[R][R];
  double b;
  double ll;
  __device__ void zero() {
#pragma unroll
    for (int a = 0; a < R; ++a)
#pragma unroll
      for (int c = 0; c < R; ++c) g[a][c] = 0.0;
    b = 0.0;
    ll = 0.0;
  }
};

// Consume `cnt` staged rows (chunk buffer S.u, row stride KP) whose list
// entries start at f.  Must be called by the whole CTA; ends with a barrier.
template <int R>
__device__ __forceinline__ void accumulate_chunk(const PointSmem &S, int f, int cnt, int k, bool do_gram,
                                                 bool do_pf, Accum<R> &A) {
  constexpr int KP = kp_of_r(R);
  const int tid = threadIdx.x, tr = tid >> 4, tc = tid & 15;
  if (do_gram) {
    for (int cc = 0; cc < cnt; ++cc) {
      const double *yr = S.u + cc * KP;
      const double w = S.lw[f + cc];
      double av[R], bv[R];
#pragma unroll
      for (int a = 0; a < R; ++a) av[a] = yr[tr + 16 * a] * w;
#pragma unroll
      for (int c = 0; c < R; ++c) bv[c] = yr[tc + 16 * c];
#pragma unroll
      for (int a = 0; a < R; ++a)
#pragma unroll
        for (int c = 0; c < R; ++c) A.g[a][c] = fma(av[a], bv[c], A.g[a][c]);
      if (tid < KP) A.b = fma(S.lwd[f + cc], yr[tid], A.b);
    }
  }
  if (do_pf && tid < k) {
    // log_like(j) = log_like(j) - 0.5*(dep-hdxf)*(dep-hdxf)*rloc/rdiag, serial in
    // obs order, no contraction (common_lpfgm.f90:64-69)
    double ll = A.ll;
    for (int cc = 0; cc < cnt; ++cc) {
      double d = __dsub_rn(S.ldep[f + cc], S.u[cc * KP + tid]);
      double q = __dmul_rn(__dmul_rn(0.5, d), d);
      q = __ddiv_rn(__dmul_rn(q, S.lrloc[f + cc]), S.lrdiag[f + cc]);
      ll = __dsub_rn(ll, q);
    }
    A.ll = ll;
  }
  __syncthreads();
}

// Write G + alpha I (k x k, column-major, stride ldb) into B = S.u and b into S.b.
template <int R>
__device__ __forceinline__ void store_gram(const PointSmem &S, int k, double alpha, const Accum<R> &A) {
  constexpr int KP = kp_of_r(R);
  const int tid = threadIdx.x, tr = tid >> 4, tc = tid & 15;
  double *B = S.u;
#pragma unroll
  for (int a = 0; a < R; ++a)
#pragma unroll
    for (int c = 0; c < R; ++c) {
      const int r = tr + 16 * a, cl = tc + 16 * c;
      if (r < k && cl < k) B[(long)cl * S.ldb + r] = A.g[a][c] + (r == cl ? alpha : 0.0);
    }
  if (tid < k) S.b[tid] = A.b;
  (void)KP;
  __syncthreads();
}

// One-sided cyclic Jacobi on the SPD matrix in B (n x n, column-major,
// stride ldb, n <= 128).  Round-robin ordering: in each of the n2-1 rounds the
// n2/2 column pairs are disjoint and are processed concurrently, one 8-lane
// group per pair (4 pairs per warp).  A pair (p,q) is rotated when
// |b_p.b_q| > tol |b_p||b_q|; the sweep loop ends after a sweep without
// rotations.  On return B holds the eigenvectors as columns and lam[] the
// eigenvalues (column norms).  Returns status bits (uniform over the CTA).
static __device__ __noinline__ int jacobi_eig(double *B, int n, int ldb, double tol, int maxsw, double *lam,
                                              int *flag) {
  constexpr int G = 8, E = 16;  // lanes per pair, elements per lane (n <= G*E)
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int grp = lane / G, gl = lane % G, lead = grp * G;
  const int n2 = (n + 1) & ~1, m = n2 - 1, npair = n2 / 2;
  int bits = 0, sweep = 0;
  if (threadIdx.x == 0) flag[1] = 0;
  for (; sweep < maxsw; ++sweep) {
    if (threadIdx.x == 0) *flag = 0;
    __syncthreads();
    for (int rd = 0; rd < m; ++rd) {
      for (int base = wid * (32 / G); base < npair; base += nw * (32 / G)) {
        const int pi = base + grp;
        int a = 0, b = 0;
        if (pi == 0) {
          a = m;
          b = rd;
        } else {
          a = (rd + pi) % m;
          b = (rd - pi + m) % m;
        }
        const bool act = pi < npair && a < n && b < n;
        double *ca = B + (long)(act ? a : 0) * ldb, *cb = B + (long)(act ? b : 0) * ldb;
        double va[E], vb[E], al = 0.0, be = 0.0, ga = 0.0;
#pragma unroll
        for (int t = 0; t < E; ++t) {
          const int r = gl + G * t;
          const bool in = act && r < n;
          va[t] = in ? ca[r] : 0.0;
          vb[t] = in ? cb[r] : 0.0;
          al = fma(va[t], va[t], al);
          be = fma(vb[t], vb[t], be);
          ga = fma(va[t], vb[t], ga);
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) {
          al += __shfl_xor_sync(0xffffffffu, al, o);
          be += __shfl_xor_sync(0xffffffffu, be, o);
          ga += __shfl_xor_sync(0xffffffffu, ga, o);
        }
        // one value per group, so every lane of a pair applies the same rotation
        al = __shfl_sync(0xffffffffu, al, lead);
        be = __shfl_sync(0xffffffffu, be, lead);
        ga = __shfl_sync(0xffffffffu, ga, lead);
        if (act && fabs(ga) > tol * sqrt(al * be)) {
          const double zeta = (be - al) / (2.0 * ga);
          const double tt = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
          const double cs = 1.0 / sqrt(1.0 + tt * tt), sn = cs * tt;
#pragma unroll
          for (int t = 0; t < E; ++t) {
            const int r = gl + G * t;
            if (r < n) {
              ca[r] = cs * va[t] - sn * vb[t];
              cb[r] = sn * va[t] + cs * vb[t];
            }
          }
          if (gl == 0) *flag = 1;
        }
      }
      __syncthreads();
    }
    const int rot = *flag;
    __syncthreads();
    if (!rot) break;
  }
  if (sweep >= maxsw) bits |= SBLETKF_ERR_EIG_NOCONV;
  for (int j = wid; j < n; j += nw) {
    double *cj = B + (long)j * ldb;
    double s = 0.0;
    for (int r = lane; r < n; r += 32) s = fma(cj[r], cj[r], s);
    s = __shfl_sync(0xffffffffu, warp_sum(s), 0);
    const double l = sqrt(s);
    if (lane == 0) lam[j] = l;
    const double inv = 1.0 / l;
    for (int r = lane; r < n; r += 32) cj[r] *= inv;
  }
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += blockDim.x)
    if (!(lam[j] > 0.0) || !isfinite(lam[j])) atomicOr(flag + 1, SBLETKF_ERR_NONFINITE);
  __syncthreads();
  bits |= flag[1];
  return bits;
}

// Normalised weights and their serial cumulative sum into S.cw
// (common_lpfgm.f90:71-75, 252-255).  ll[] holds log-likelihoods.
__device__ __forceinline__ void pf_weights(const PointSmem &S, int k) {
  if (threadIdx.x == 0) {
    double mx = S.ll[0];
    for (int j = 1; j < k; ++j) mx = S.ll[j] > mx ? S.ll[j] : mx;
    S.misc[40] = mx;
  }
  __syncthreads();
  if (threadIdx.x < k) S.ll[threadIdx.x] = exp(__dsub_rn(S.ll[threadIdx.x], S.misc[40]));
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int j = 0; j < k; ++j) s = __dadd_rn(s, S.ll[j]);
    double acc = 0.0;
    for (int j = 0; j < k; ++j) {
      const double wj = __ddiv_rn(S.ll[j], s);
      acc = j == 0 ? wj : __dadd_rn(acc, wj);
      S.cw[j] = acc;
    }
  }
  __syncthreads();
}

// First i with r <= cw[i] (i < k-1), else k-1 (common_lpfgm.f90:142-149).
__device__ __forceinline__ int pf_select(const double *cw, int k, double r) {
  int lo = 0, hi = k - 1;  // answer in [lo, hi]
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (r <= cw[mid]) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// One resampling draw (common_lpfgm.f90:89-197) by one thread.
// hist: k bytes of scratch.  src[j] = particle (0-based) taken by member j.
// The selected particles depend on the uniforms only through the histogram of
// inum (inum is monotone in the sorted uniforms), so SR and MR share the
// assignment below; MR needs no sort.
__device__ __forceinline__ void resample_draw(const sbletkf_params &p, const double *cw, int k, const double *u,
                                              uint8_t *hist, int16_t *src) {
  for (int i = 0; i < k; ++i) hist[i] = 0;
  if (p.rm == SBLETKF_RM_SR) {
    const double r1 = __ddiv_rn(__dsub_rn(__dadd_rn(u[0], 1.0), 1.0), (double)k);
    const double base = p.sr_textbook ? u[0] : r1;
    int i = 0;
    for (int j = 0; j < k; ++j) {
      const double r = j == 0 ? r1 : __ddiv_rn(__dsub_rn(__dadd_rn(base, (double)(j + 1)), 1.0), (double)k);
      while (i < k - 1 && !(r <= cw[i])) ++i;  // r ascending -> merge scan
      hist[i]++;
    }
  } else {
    for (int j = 0; j < k; ++j) hist[pf_select(cw, k, u[j])]++;
  }
  if (p.dp) {
    // diagonal priority: every selected particle keeps its own column; the
    // extra copies, in increasing particle order, fill the unused columns
    // left to right (:152-181)
    int f = 0;
    for (int i = 0; i < k; ++i)
      if (hist[i]) src[i] = (int16_t)i;
    for (int i = 0; i < k; ++i)
      for (int c = 1; c < hist[i]; ++c) {
        while (f < k - 1 && hist[f]) ++f;
        src[f++] = (int16_t)i;
      }
  } else {
    int j = 0;
    for (int i = 0; i < k; ++i)
      for (int c = 0; c < hist[i]; ++c) src[j++] = (int16_t)i;
  }
}

// Mean / spread (k-1) / perturbation of S.x rows v < nvt, warp v per row
// (common_da.f90:354-401).  Mean into misc[v], spread into misc[8+v].
__device__ __forceinline__ void mean_spread_pert(const PointSmem &S, int kp, int k, int nvt) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int v = wid; v < nvt; v += blockDim.x >> 5) {
    double *xv = S.x + v * kp;
    double s = 0.0;
    for (int m = lane; m < k; m += 32) s += xv[m];
    const double mean = __shfl_sync(0xffffffffu, warp_sum(s), 0) / (double)k;
    double q = 0.0;
    for (int m = lane; m < k; m += 32) {
      const double d = xv[m] - mean;
      q = fma(d, d, q);
      xv[m] = d;
    }
    const double sp = sqrt(__shfl_sync(0xffffffffu, warp_sum(q), 0) / (double)(k - 1));
    if (lane == 0) {
      S.misc[v] = mean;
      S.misc[8 + v] = sp;
    }
  }
  __syncthreads();
}

// RTPP / RTPS on the analysis in S.an (rows v < nvt) with forecast
// perturbations in S.x, then the T/S round-off (common_da.f90:99-113,
// 438-533).  Warp v per row; results stay in S.an.
__device__ __forceinline__ void relax_and_clamp(const sbletkf_params &p, const PointSmem &S, int kp, int k, int nvt,
                                                int kl, double phi) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int v = wid; v < nvt; v += blockDim.x >> 5) {
    double *av = S.an + v * kp;
    const double *dxf = S.x + v * kp;
    double s = 0.0;
    for (int m = lane; m < k; m += 32) s += av[m];
    const double am = __shfl_sync(0xffffffffu, warp_sum(s), 0) / (double)k;
    double q = 0.0;
    for (int m = lane; m < k; m += 32) {
      const double d = av[m] - am;
      q = fma(d, d, q);
    }
    const double as = sqrt(__shfl_sync(0xffffffffu, warp_sum(q), 0) / (double)(k - 1));
    const double fs = S.misc[8 + v];
    const bool rtpp = 0.0 < p.alpha_rtpp, rtps = 0.0 < p.alpha_rtps;
    double fac = 0.0;
    if (rtps) fac = (as == 0.0) ? 0.0 : p.alpha_rtps * fs / as + (1.0 - p.alpha_rtps);
    const bool clampT = p.roff && v < p.nv3d && v == p.iv3d_t && kl >= 1 && phi != 1.0;
    const bool clampS = p.roff && v < p.nv3d && v == p.iv3d_s && kl >= 1 && phi != 1.0;
    for (int m = lane; m < k; m += 32) {
      const double dxa = av[m] - am;
      double a = av[m];
      if (rtpp) a = am + p.alpha_rtpp * dxf[m] + (1.0 - p.alpha_rtpp) * dxa;
      if (rtps) a = am + dxa * fac;
      if (clampT) a = fmin(fmax(a, p.tmin), p.tmax);
      if (clampS) a = fmin(fmax(a, p.smin), p.smax);
      av[m] = a;
    }
  }
  __syncthreads();
}

}  // namespace sbl
