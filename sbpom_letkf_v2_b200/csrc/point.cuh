// point.cuh -- per-grid-point building blocks shared by the analysis, core
// and backward kernels.  One CTA of kThreads threads owns one local problem.
//
//   accumulate_chunk   Gram  G += Y^T diag(rloc/rdiag) Y and b += Y^T diag(rloc/rdiag) dep
//                      (common_letkf.f90:93-122) in FP64 registers, and the PF
//                      log-likelihood (common_lpfgm.f90:64-69) in obs order
//   jacobi_eig         eigenpairs of the SPD k x k matrix A = G + (k-1)/rho I
//                      (replaces mtx_eigen / DSYEV, common.f90:992-1050):
//                      pivoted Cholesky, then one-sided (Hestenes) cyclic
//                      Jacobi on the factor's columns, odd-even ordering
//   jacobi_eig_warm    the same from a nearby matrix's eigenvectors V:
//                      one-sided Jacobi on A V, lambda_j = |column j|
//   pf_weights         max-subtracted exp, normalise, cumulative sum (serial)
//   resample_draw      SR/MR draw, inum search and diagonal-priority assignment (one warp)
//                      (common_lpfgm.f90:89-197)
#pragma once

#include "gram_tc.cuh"
#include "internal.cuh"

namespace sbl {

// Relative rotation size that ends the Jacobi eigensolve (see
// jacobi_sweeps_oe) unless sbletkf_params.jacobi_stop sets another.  The
// mixed path's Gram carries ~1e-6 relative error, so its eigensolve stops
// earlier: the sweep whose rotations stay below 1e-5 leaves residuals of
// ~1e-10 (Jacobi converges quadratically), far below the Gram's error, and
// a warm-started solve takes 3 sweeps instead of 4.
constexpr double kJacobiStop = 1e-10;
constexpr double kJacobiStopMixed = 1e-5;
__host__ __device__ inline double jacobi_stop_of(const sbletkf_params &p) {
  return p.jacobi_stop > 0.0 ? p.jacobi_stop : p.precision == SBLETKF_PREC_MIXED ? kJacobiStopMixed : kJacobiStop;
}
// Smallest relative rotation the sweeps apply, unless sbletkf_params.jacobi_tol
// sets another: k eps on the FP64 path; 1e-8 on the mixed path, where the
// rotations below it (left as residual, ~3e-8) are well under the Gram's own
// ~1e-6 error and only cost the last sweep time.
constexpr double kJacobiTolMixed = 1e-8;
__host__ __device__ inline double jacobi_tol_of(const sbletkf_params &p, int k) {
  return p.jacobi_tol > 0.0 ? p.jacobi_tol
         : p.precision == SBLETKF_PREC_MIXED ? kJacobiTolMixed
                                             : (double)k * 2.220446049250313e-16;
}

// R x R register tile per thread over a 16 x 16 thread grid: k <= 16*R.
__host__ __device__ constexpr int kp_of_r(int r) { return 16 * r; }
inline int r_for_k(int k) { return k <= 32 ? 2 : k <= 64 ? 4 : k <= 112 ? 7 : 8; }

constexpr int kDrawBatch = 64;  // PF draws resolved per pass

// Shared memory of the PF draws: kDrawBatch draws' src rows (int16), then per
// warp a k-int histogram and k int16 unused-column ranks.
__host__ __device__ constexpr size_t pf_draw_bytes(int k) {
  return (size_t)kDrawBatch * k * sizeof(int16_t) + (size_t)(kThreads / 32) * k * (sizeof(int) + sizeof(int16_t));
}
// Leading dimension of an n x n eigensolver matrix: 4 (mod 16) doubles.
__host__ __device__ inline int eig_ld(int n) { return (n + 15) / 16 * 16 + 4; }

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
  // Offset of the tensor-core operand stages inside the union (mixed path):
  // after the FP32 staging rows, 1024-aligned.
  __host__ __device__ static size_t tc_tiles_off(int kp) {
    return ((size_t)tc::kKC * kp * sizeof(float) + 1023) & ~size_t(1023);
  }
  // Union size: max(chunk rows, k x ldb matrix, dual Z and N, draw buffers,
  // and for the mixed path FP32 staging + two operand stages).
  __host__ __device__ static size_t union_bytes(int k, int kp, bool mixed = false) {
    const size_t tcb = mixed ? tc_tiles_off(kp) + 2 * (size_t)tc::kStageBytes + 1024 : 0;
    const size_t nd = (size_t)dual_max(k);
    size_t chunk = sizeof(double) * kChunk * kp;
    const size_t kk = (size_t)k;
    size_t mat = sizeof(double) * kk * eig_ld(kp);
    size_t dual = sizeof(double) * (nd * (kp + 1) + nd * eig_ld((int)nd));
    size_t pf = pf_draw_bytes(k) + 16;
    size_t m = chunk > mat ? chunk : mat;
    m = m > dual ? m : dual;
    m = m > tcb ? m : tcb;
    return a16(m > pf ? m : pf);
  }
  // nrows: grid rows of a search box kept (0: none, the rows live
  // elsewhere); listcap: local-obs list entries (>= dual_max and >= kp,
  // since the eigensolve borrows lidx as its permutation).
  __host__ __device__ static size_t fixed_bytes(int kp, int nrows = kRowMax, int listcap = kListCap) {
    size_t s = 0;
    s += (nrows > 0 ? a16(sizeof(int) * nrows) + a16(sizeof(int) * (nrows + 1)) : 0) +
         a16(sizeof(int) * listcap) + a16(sizeof(int) * 64);
    s += 5 * a16(sizeof(double) * listcap);
    s += 5 * a16(sizeof(double) * kp) + a16(sizeof(double) * 64);
    s += 4 * a16(sizeof(double) * kNvMax * kp);
    return s;
  }
  __host__ __device__ static size_t bytes(int k, int kp, bool mixed = false, int nrows = kRowMax,
                                          int listcap = kListCap) {
    return fixed_bytes(kp, nrows, listcap) + union_bytes(k, kp, mixed) + (mixed ? 1024 : 0);
  }

  __device__ void carve(void *base, int k, int kp, int nrows = kRowMax, int listcap = kListCap) {
    char *q = (char *)base;
    auto take = [&](size_t n) { char *r = q; q += a16(n); return (void *)r; };
    rowstart = nrows > 0 ? (int *)take(sizeof(int) * nrows) : nullptr;
    rowpref = nrows > 0 ? (int *)take(sizeof(int) * (nrows + 1)) : nullptr;
    lidx = (int *)take(sizeof(int) * listcap);
    iws = (int *)take(sizeof(int) * 64);
    lw = (double *)take(sizeof(double) * listcap);
    lwd = (double *)take(sizeof(double) * listcap);
    lrloc = (double *)take(sizeof(double) * listcap);
    lrdiag = (double *)take(sizeof(double) * listcap);
    ldep = (double *)take(sizeof(double) * listcap);
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
    ldb = eig_ld(kp);  // 4 (mod 16): bank-conflict-free Jacobi column groups
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
  if (do_pf) {
    // log_like(j) = log_like(j) - 0.5*(dep-hdxf)*(dep-hdxf)*rloc/rdiag, serial in
    // obs order, no contraction (common_lpfgm.f90:64-69).  The terms are
    // independent: the whole CTA computes them (in place of the rows, which the
    // Gram above has finished with), then each member's thread subtracts its
    // column of terms in observation order -- the same operations and order.
    if (do_gram) cta_sync();
    double *q = S.u;
#pragma unroll 4
    for (int e = tid; e < cnt * KP; e += kThreads) {
      const int cc = e / KP, m = e - cc * KP;
      if (m < k) {
        const double d = __dsub_rn(S.ldep[f + cc], q[e]);
        double t = __dmul_rn(__dmul_rn(0.5, d), d);
        q[e] = __ddiv_rn(__dmul_rn(t, S.lrloc[f + cc]), S.lrdiag[f + cc]);
      }
    }
    cta_sync();
    if (tid < k) {
      double ll = A.ll;
      for (int cc = 0; cc < cnt; ++cc) ll = __dsub_rn(ll, q[cc * KP + tid]);
      A.ll = ll;
    }
  }
  cta_sync();
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
  cta_sync();
}

// ---------------------------------------------------------------------------
// Symmetric eigensolver of the SPD matrix A (n x n, column-major, stride ldb)
// held in shared memory.  Replaces mtx_eigen / DSYEV (common.f90:992-1050);
// A >= alpha I > 0, so the reference's negative-eigenvalue branch never fires.
//
//  1. Cholesky with diagonal pivoting, P A P^T = L L^T, in place.
//  2. One-sided cyclic Jacobi on the columns of L: L W -> columns that are
//     mutually orthogonal.  Since L = V' S U^T (SVD), the converged columns are
//     s_j v'_j: normalised, they are the eigenvectors of P A P^T, and
//     lambda_j = s_j^2 = |column j|^2.  Un-permuting the rows gives A's.
//     This is the preconditioned one-sided Jacobi SVD (Drmac & Veselic 2008):
//     the sweep count follows A's spectrum (one-sided Jacobi on A itself acts
//     on A^2, whose squared gaps near the alpha cluster need many more
//     sweeps), and the pivoted factor's columns start nearly orthogonal.
//
// Jacobi detail: odd-even ordering (jacobi_sweeps_oe below) with 4-lane
// groups, each holding a column pair in registers and passing one column per
// step to a neighbour through shared memory.  Column norms are carried
// (recomputed each sweep), so only b_p.b_q is a dot product.  A pair is
// rotated when (b_p.b_q)^2 > tol^2 |b_p|^2 |b_q|^2; the angle t is computed
// in FP32 while c = 1/sqrt(1+t^2), s = c t are FP64, so every rotation is
// orthogonal to FP64 rounding and the angle only has to shrink b_p.b_q (the
// residual of a rotation is ~1e-7 of what it removes).  The loop ends after
// a sweep whose largest relative b_p.b_q was <= `stop` (1e-10 by default).
// Ending earlier, after the sweep whose rotations were all below 1e-7 instead
// of after the next one, which mostly only confirms convergence, saved 5 % of
// the workload-1 cycle but left the analysis 1e-9..1e-8 from the oracle.
// ---------------------------------------------------------------------------

// In-place pivoted Cholesky of the full symmetric matrix in B: on return B's
// lower triangle holds L (P A P^T = L L^T), the strict upper triangle is zero
// and perm[i] is the original index of row i.  vec: n doubles of scratch.
static __device__ __noinline__ int chol_pivot(double *B, int n, int ldb, int *perm, double *vec, int *flag) {
  const int tid = threadIdx.x, nt = kThreads, tx = tid & 15, ty = tid >> 4, nty = nt >> 4;
  const int lane = tid & 31, wid = tid >> 5;
  for (int i = tid; i < n; i += nt) perm[i] = i;
  if (tid == 0) flag[1] = 0;
  cta_sync();
  for (int j = 0; j < n; ++j) {
    if (wid == 0) {  // pivot: largest remaining diagonal (first on ties)
      double best = -1.0;
      int bi = j;
      for (int i = j + lane; i < n; i += 32) {
        const double d = B[(long)i * ldb + i];
        if (d > best) {
          best = d;
          bi = i;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (lane == 0) flag[2] = bi;
    }
    cta_sync();
    const int pv = flag[2];
    if (pv != j) {  // symmetric swap of rows / columns j and pv
      for (int c = tid; c < n; c += nt) {
        double *bc = B + (long)c * ldb;
        const double t = bc[j];
        bc[j] = bc[pv];
        bc[pv] = t;
      }
      cta_sync();
      for (int r = tid; r < n; r += nt) {
        const double t = B[(long)j * ldb + r];
        B[(long)j * ldb + r] = B[(long)pv * ldb + r];
        B[(long)pv * ldb + r] = t;
      }
      if (tid == 0) {
        const int t = perm[j];
        perm[j] = perm[pv];
        perm[pv] = t;
      }
      cta_sync();
    }
    double d = B[(long)j * ldb + j];
    const bool bad = !(d > 0.0) || !isfinite(d);
    if (bad) d = 1.0;
    const double r = sqrt(d), inv = 1.0 / r;
    double *bj = B + (long)j * ldb;
    for (int i = j + 1 + tid; i < n; i += nt) vec[i] = bj[i] * inv;
    cta_sync();
    if (tid == 0) {
      bj[j] = r;
      if (bad) flag[1] |= SBLETKF_ERR_NONFINITE;
    }
    for (int i = j + 1 + tid; i < n; i += nt) bj[i] = vec[i];
    for (int c = j + 1 + ty; c < n; c += nty) {  // full symmetric trailing update
      const double vc = vec[c];
      double *bc = B + (long)c * ldb;
      for (int i = j + 1 + tx; i < n; i += 16) bc[i] = fma(-vec[i], vc, bc[i]);
    }
    cta_sync();
  }
  for (int c = ty; c < n; c += nty)
    for (int i = tx; i < c; i += 16) B[(long)c * ldb + i] = 0.0;
  cta_sync();
  return flag[1];
}

// One-sided Jacobi sweeps with the odd-even ordering, columns held in
// registers: 4-lane group g holds the columns at positions (2g, 2g+1) in odd
// steps and (2g+1, 2g+2) in even steps (E rows per lane each).  After a
// rotation the pair's columns trade positions, so after an odd step a group
// passes one column (and its squared norm) to its left neighbour and after an
// even step one to its right.  The columns travel through slots in B (the
// matrix is in registers meanwhile): left-going slot g = column g of B,
// right-going slot g = column ng+g, norms in nrm[] likewise; position 0 in
// even steps stays parked in left slot 0.  Over n2 steps every pair of
// columns meets once, as in a round-robin sweep, but each step moves one
// column per pair through shared memory instead of loading and storing both,
// with one barrier.  On exit B holds the columns in some order (the zero
// padding column of odd n is dropped), which is all the eigenpair extraction
// needs.  nrm: >= n doubles of scratch; flag: >= 4 shared ints.
template <int E>
static __device__ __forceinline__ int jacobi_sweeps_oe(double *B, int n, int ldb, double tol, double stop, int maxsw,
                                                       double *nrm, int *flag) {
  constexpr int G = 4;
  // group g (column pair) = threads 4g..4g+3.  Consecutive groups of a warp
  // use slots ldb apart, conflict-free with ldb = 4 (mod 16); spreading the
  // groups over the warps (g = 8 s + w) would balance the SM sub-partitions
  // but put a warp's slots 8 ldb apart, all on the same banks (measured 37 %
  // slower).
  const int tid = threadIdx.x, gl = tid % G, grp = tid / G;
  const int n2 = (n + 1) & ~1, ng = n2 / 2;   // 2*ng - 1 <= n slots fit in B
  const bool inb = grp < ng;
  double *SL = B, *SR = B + (long)ng * ldb, *NL = nrm, *NR = nrm + ng;
  double x[E], y[E], nx = 0.0, ny = 0.0;
  {  // load positions (2g, 2g+1) = columns 2g, 2g+1 (position n of odd n: zeros)
    const int ca = 2 * grp, cb = 2 * grp + 1;
#pragma unroll
    for (int t = 0; t < E; ++t) {
      const int r = gl + G * t;
      x[t] = (inb && ca < n && r < n) ? B[(long)ca * ldb + r] : 0.0;
      y[t] = (inb && cb < n && r < n) ? B[(long)cb * ldb + r] : 0.0;
    }
  }
  cta_sync();
  const double tol2 = tol * tol, big2 = stop * stop;
  int sweep = 0;
  for (; sweep < maxsw; ++sweep) {
    {  // exact squared norms at the start of a sweep; the xor butterfly
       // leaves the same (commutatively added) sum in all four lanes
      double a = 0.0, b = 0.0;
#pragma unroll
      for (int t = 0; t < E; ++t) {
        a = fma(x[t], x[t], a);
        b = fma(y[t], y[t], b);
      }
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
      }
      nx = a;
      ny = b;
    }
    if (tid == 0) *flag = 0;
    cta_sync();
    int big = 0;
    for (int step = 0; step < n2; ++step) {
      const bool odd = (step & 1) == 0;
      const bool act = inb && (odd || grp < ng - 1);
      double g0 = 0.0, g1 = 0.0;  // two independent chains
#pragma unroll
      for (int t = 0; t < E; ++t) {
        if (t & 1) g1 = fma(x[t], y[t], g1);
        else g0 = fma(x[t], y[t], g0);
      }
      double ga = g0 + g1;
      // xor butterfly: every lane of the group ends with the same sum
#pragma unroll
      for (int o = G / 2; o > 0; o >>= 1) ga += __shfl_xor_sync(0xffffffffu, ga, o);
      const double g2 = ga * ga, ab = nx * ny;
      if (act && g2 > tol2 * ab) {
        // the angle only has to shrink b_p.b_q: FP32 with approximate division
        const float zf = __fdividef((float)(ny - nx) * 0.5f, (float)ga);
        // sqrt(1 + z^2): q rsqrt(q) (MUFU) up to |z| = 4096, beyond which it
        // rounds to |z| in FP32 (capping |z| instead would over-rotate pairs
        // of very different norms)
        const float az = fabsf(zf), qa = fminf(az, 4096.0f), q = fmaf(qa, qa, 1.0f);
        const float tf = __fdividef(copysignf(1.0f, zf), az + (az > 4096.0f ? az : q * rsqrtf(q)));
        const double tt = (double)tf;
        const double cs = rsqrt(fma(tt, tt, 1.0)), sn = cs * tt;
#pragma unroll
        for (int t = 0; t < E; ++t) {
          const double a = x[t], b = y[t];
          x[t] = cs * a - sn * b;
          y[t] = sn * a + cs * b;
        }
        const double c2 = cs * cs, s2 = sn * sn, csg = 2.0 * cs * sn * ga;
        const double nx2 = c2 * nx - csg + s2 * ny;
        ny = s2 * nx + csg + c2 * ny;
        nx = nx2;
        if (g2 > big2 * ab) big = 1;
      }
      // the pair's columns trade positions: x is now at the second, y at the first
      if (odd) {  // y to the left neighbour (group 0's stays parked), new y from the right
        if (inb) {
#pragma unroll
          for (int t = 0; t < E; ++t) {
            const int r = gl + G * t;
            if (r < n) SL[(long)grp * ldb + r] = y[t];
          }
          if (gl == 0) NL[grp] = ny;
        }
        cta_sync();
        if (inb && grp + 1 < ng) {
#pragma unroll
          for (int t = 0; t < E; ++t) {
            const int r = gl + G * t;
            y[t] = r < n ? SL[(long)(grp + 1) * ldb + r] : 0.0;
          }
          ny = NL[grp + 1];
        }
      } else {    // x to the right neighbour, new x from the left (group 0: the parked column)
        if (inb && grp == ng - 1) {  // idle last pair: its single column moves to y
#pragma unroll
          for (int t = 0; t < E; ++t) y[t] = x[t];
          ny = nx;
        }
        if (inb && grp < ng - 1) {
#pragma unroll
          for (int t = 0; t < E; ++t) {
            const int r = gl + G * t;
            if (r < n) SR[(long)grp * ldb + r] = x[t];
          }
          if (gl == 0) NR[grp] = nx;
        }
        cta_sync();
        if (inb) {
          const double *src = grp > 0 ? SR + (long)(grp - 1) * ldb : SL;
#pragma unroll
          for (int t = 0; t < E; ++t) {
            const int r = gl + G * t;
            x[t] = r < n ? src[r] : 0.0;
          }
          nx = grp > 0 ? NR[grp - 1] : NL[0];
        }
      }
      // no second barrier: the next step writes the other slot area, and a
      // slot is rewritten only after the following step's barrier
    }
    if (big) *flag = 1;
    cta_sync();
    const int rot = *flag;
    cta_sync();
    if (!rot) break;
  }
  if (tid == 0) flag[3] = sweep;  // sweeps run (diagnostics)
  // write the columns back; for odd n one position holds the zero padding
  // column (squared norm exactly 0: it never rotates), whose place takes the
  // column at position n
  if (tid == 0) flag[2] = -1;
  cta_sync();
  if ((n & 1) && inb && gl == 0) {
    if (!(nx > 0.0)) flag[2] = 2 * grp;
    if (!(ny > 0.0)) flag[2] = 2 * grp + 1;
  }
  cta_sync();
  const int zpos = flag[2];
  if (inb) {
#pragma unroll
    for (int sl = 0; sl < 2; ++sl) {
      int pos = 2 * grp + sl;
      if ((n & 1) && pos == zpos) continue;      // the padding column
      if (pos >= n) pos = zpos;                  // the column at position n
      if (pos < 0 || pos >= n) continue;
#pragma unroll
      for (int t = 0; t < E; ++t) {
        const int r = gl + G * t;
        if (r < n) B[(long)pos * ldb + r] = sl ? y[t] : x[t];
      }
    }
  }
  cta_sync();
  return sweep >= maxsw ? SBLETKF_ERR_EIG_NOCONV : 0;
}

// Eigenpairs of the SPD matrix in B: eigenvectors replace B's columns and
// lam[] receives the eigenvalues.  vec: n doubles, perm: n ints of scratch;
// flag: >= 4 shared ints (flag[3] = sweeps run).  Returns status bits.
template <int EMAX>
static __device__ __forceinline__ int jacobi_eig(double *B, int n, int ldb, double tol, double stop, int maxsw,
                                                 double *lam, int *flag, int *perm, double *vec) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = kThreads >> 5;
  int bits = chol_pivot(B, n, ldb, perm, vec, flag);
  if (n <= 32 || EMAX <= 8) bits |= jacobi_sweeps_oe<8>(B, n, ldb, tol, stop, maxsw, vec, flag);
  else if (n <= 64 || EMAX <= 16) bits |= jacobi_sweeps_oe<(EMAX < 16 ? EMAX : 16)>(B, n, ldb, tol, stop, maxsw, vec, flag);
  else if (n <= 100 || EMAX <= 25) bits |= jacobi_sweeps_oe<(EMAX < 25 ? EMAX : 25)>(B, n, ldb, tol, stop, maxsw, vec, flag);
  else if (n <= 112 || EMAX <= 28) bits |= jacobi_sweeps_oe<(EMAX < 28 ? EMAX : 28)>(B, n, ldb, tol, stop, maxsw, vec, flag);
  else bits |= jacobi_sweeps_oe<EMAX>(B, n, ldb, tol, stop, maxsw, vec, flag);
  // lambda_j = |column j|^2; eigenvector = column / |column|, rows un-permuted
  for (int j = wid; j < n; j += nw) {
    double *cj = B + (long)j * ldb;
    double v[4], s = 0.0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int r = lane + 32 * t;
      v[t] = r < n ? cj[r] : 0.0;
      s = fma(v[t], v[t], s);
    }
    s = __shfl_sync(0xffffffffu, warp_sum(s), 0);
    if (lane == 0) lam[j] = s;
    const double inv = 1.0 / sqrt(s);
    __syncwarp();
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int r = lane + 32 * t;
      if (r < n) cj[perm[r]] = v[t] * inv;
    }
  }
  if (threadIdx.x == 0) flag[1] = 0;
  cta_sync();
  for (int j = threadIdx.x; j < n; j += kThreads)
    if (!(lam[j] > 0.0) || !isfinite(lam[j])) atomicOr(flag + 1, SBLETKF_ERR_NONFINITE);
  cta_sync();
  bits |= flag[1];
  return bits;
}

// X = A V for the warm start, written over A in B.  Thread (rt, ct) keeps
// rows rt + i nrt (i < 4, nrt = ceil(n/4)) of columns CT ct .. CT ct + CT-1
// in registers, reading A from shared memory (consecutive threads,
// consecutive rows) and V's columns from global memory (a warp's threads
// share one or two column tiles, so those loads are broadcasts).  One
// barrier, then the tiles replace A.  Needs ceil(n/4) ceil(n/CT) <= kThreads.
template <int CT>
static __device__ __forceinline__ void warm_product(double *B, int n, int ldb, const double *V) {
  const int nrt = (n + 3) >> 2, rt = threadIdx.x % nrt, c0 = CT * (threadIdx.x / nrt);
  const bool act = c0 < n;
  double acc[4][CT];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < CT; ++j) acc[i][j] = 0.0;
  if (act) {
    const double *vc = V + (long)c0 * n;
#pragma unroll 2
    for (int q = 0; q < n; ++q) {
      const double *aq = B + (long)q * ldb + rt;
      double a[4], v[CT];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = rt + i * nrt < n ? aq[i * nrt] : 0.0;
#pragma unroll
      for (int j = 0; j < CT; ++j) v[j] = c0 + j < n ? vc[(long)j * n + q] : 0.0;
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < CT; ++j) acc[i][j] = fma(a[i], v[j], acc[i][j]);
    }
  }
  cta_sync();
  if (act) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = rt + i * nrt;
      if (r >= n) continue;
#pragma unroll
      for (int j = 0; j < CT; ++j)
        if (c0 + j < n) B[(long)(c0 + j) * ldb + r] = acc[i][j];
    }
  }
  cta_sync();
}

// Eigenpairs of the SPD matrix in B from a starting orthogonal matrix V
// (n x n in global memory, column j at V + j*n; the eigenvectors of a nearby
// matrix): one-sided Jacobi on the columns of X = A V (formed in place of
// A).  Since X X^T = A^2, the converged columns are lambda_j u_j:
// lambda_j = |column j|, u_j = column / lambda_j.  When A is close to the
// matrix V came from, X starts nearly orthogonal and needs a few sweeps
// instead of the cold solve's pivoted Cholesky and ~10 sweeps.
template <int EMAX>
static __device__ __forceinline__ int jacobi_eig_warm(double *B, int n, int ldb, double tol, double stop, int maxsw,
                                                      double *lam, int *flag, double *vec, const double *V) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = kThreads >> 5;
  // column tile of warm_product: ceil(n/4) ceil(n/CT) <= 256 for n <= 4 EMAX
  if (n <= 64 || EMAX <= 16) warm_product<4>(B, n, ldb, V);
  else if (n <= 80 || EMAX <= 20) warm_product<8>(B, n, ldb, V);
  else if (n <= 100 || EMAX <= 25) warm_product<10>(B, n, ldb, V);
  else if (n <= 112 || EMAX <= 28) warm_product<13>(B, n, ldb, V);
  else warm_product<16>(B, n, ldb, V);
  int bits = 0;
  if (n <= 32 || EMAX <= 8) bits |= jacobi_sweeps_oe<8>(B, n, ldb, tol, stop, maxsw, vec, flag);
  else if (n <= 64 || EMAX <= 16) bits |= jacobi_sweeps_oe<(EMAX < 16 ? EMAX : 16)>(B, n, ldb, tol, stop, maxsw, vec, flag);
  else if (n <= 100 || EMAX <= 25) bits |= jacobi_sweeps_oe<(EMAX < 25 ? EMAX : 25)>(B, n, ldb, tol, stop, maxsw, vec, flag);
  else if (n <= 112 || EMAX <= 28) bits |= jacobi_sweeps_oe<(EMAX < 28 ? EMAX : 28)>(B, n, ldb, tol, stop, maxsw, vec, flag);
  else bits |= jacobi_sweeps_oe<EMAX>(B, n, ldb, tol, stop, maxsw, vec, flag);
  for (int j = wid; j < n; j += nw) {
    double *cj = B + (long)j * ldb;
    double v[4], s = 0.0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int r = lane + 32 * t;
      v[t] = r < n ? cj[r] : 0.0;
      s = fma(v[t], v[t], s);
    }
    s = __shfl_sync(0xffffffffu, warp_sum(s), 0);
    const double l = sqrt(s);
    if (lane == 0) lam[j] = l;
    const double inv = 1.0 / l;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int r = lane + 32 * t;
      if (r < n) cj[r] = v[t] * inv;
    }
  }
  if (threadIdx.x == 0) flag[1] = 0;
  cta_sync();
  for (int j = threadIdx.x; j < n; j += kThreads)
    if (!(lam[j] > 0.0) || !isfinite(lam[j])) atomicOr(flag + 1, SBLETKF_ERR_NONFINITE);
  cta_sync();
  bits |= flag[1];
  return bits;
}

// jacobi_eig as a call of its own (see jacobi_eig_warm_call).
template <int EMAX>
static __device__ __noinline__ int jacobi_eig_call(double *B, int n, int ldb, double tol, double stop, int maxsw,
                                                   double *lam, int *flag, int *perm, double *vec) {
  return jacobi_eig<EMAX>(B, n, ldb, tol, stop, maxsw, lam, flag, perm, vec);
}

// jacobi_eig_warm as a call of its own: the sweeps then get a register
// allocation of their own instead of sharing it with the caller's live state
// (the pipelined kernel's consumer runs at 192 registers per thread).
template <int EMAX>
static __device__ __noinline__ int jacobi_eig_warm_call(double *B, int n, int ldb, double tol, double stop, int maxsw,
                                                        double *lam, int *flag, double *vec, const double *V) {
  return jacobi_eig_warm<EMAX>(B, n, ldb, tol, stop, maxsw, lam, flag, vec, V);
}

// out[v*ldo + j] = sum_m X[v*ldx + m] V[m][j] for v < nv, j < n: warp per
// column j, lanes over rows m (contiguous in a column of V).
static __device__ __forceinline__ void x_times_v(const double *X, int ldx, int nv, const double *V, int n, int ldb,
                                                 double *out, int ldo) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = kThreads >> 5;
  for (int j = wid; j < n; j += nw) {
    const double *vj = V + (long)j * ldb;
    double acc[kNvMax];
#pragma unroll
    for (int v = 0; v < kNvMax; ++v) acc[v] = 0.0;
    for (int r = lane; r < n; r += 32) {
      const double vr = vj[r];
#pragma unroll
      for (int v = 0; v < kNvMax; ++v)
        if (v < nv) acc[v] = fma(X[v * ldx + r], vr, acc[v]);
    }
#pragma unroll
    for (int v = 0; v < kNvMax; ++v) {
      if (v < nv) {
        const double t = __shfl_sync(0xffffffffu, warp_sum(acc[v]), 0);
        if (lane == 0) out[v * ldo + j] = t;
      }
    }
  }
}

// out[j] = sum_m V[m][j] x[m] (j < n), warp per column, lanes over rows.
static __device__ __forceinline__ void vt_times(const double *V, int n, int ldb, const double *x, double *out) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = kThreads >> 5;
  for (int j = wid; j < n; j += nw) {
    const double *vj = V + (long)j * ldb;
    double s = 0.0;
    for (int r = lane; r < n; r += 32) s = fma(vj[r], x[r], s);
    s = __shfl_sync(0xffffffffu, warp_sum(s), 0);
    if (lane == 0) out[j] = s;
  }
}

// Normalised weights and their serial cumulative sum into S.cw
// (common_lpfgm.f90:71-75, 252-255).  ll[] holds log-likelihoods.
__device__ __forceinline__ void pf_weights(const PointSmem &S, int k) {
  if (threadIdx.x == 0) {
    double mx = S.ll[0];
    for (int j = 1; j < k; ++j) mx = S.ll[j] > mx ? S.ll[j] : mx;
    S.misc[40] = mx;
  }
  cta_sync();
  if (threadIdx.x < k) S.ll[threadIdx.x] = exp(__dsub_rn(S.ll[threadIdx.x], S.misc[40]));
  cta_sync();
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
  cta_sync();
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

// One resampling draw (common_lpfgm.f90:89-197) by one warp, k <= 128.
// hist: k ints, upos: k int16 of this warp's scratch.  src[j] = particle
// (0-based) taken by member j.  The selected particles depend on the uniforms
// only through the histogram of inum (inum is monotone in the sorted
// uniforms), so SR and MR share the assignment below; MR needs no sort.  SR:
// the reference's r_j (same operations) ascend, so its merge scan finds for
// each j the first i with r_j <= cw(i) (capped at k-1) -- what pf_select
// returns -- and lanes search independently.  Diagonal priority: every
// selected particle keeps its own column; the extra copies, in increasing
// particle order, take the unused columns in increasing order (:152-181),
// i.e. extra copy number e goes to unused column number e, both ranked by
// warp prefix sums.
__device__ __forceinline__ void resample_draw(const sbletkf_params &p, const double *cw, int k, const double *u,
                                              int *hist, int16_t *upos, int16_t *src) {
  constexpr int PL = 4;  // particles per lane: i = PL lane .. PL lane + 3
  const int lane = threadIdx.x & 31;
  for (int i = lane; i < k; i += 32) hist[i] = 0;
  __syncwarp();
  if (p.rm == SBLETKF_RM_SR) {
    const double r1 = __ddiv_rn(__dsub_rn(__dadd_rn(u[0], 1.0), 1.0), (double)k);
    const double base = p.sr_textbook ? u[0] : r1;
    for (int j = lane; j < k; j += 32) {
      const double r = j == 0 ? r1 : __ddiv_rn(__dsub_rn(__dadd_rn(base, (double)(j + 1)), 1.0), (double)k);
      atomicAdd(&hist[pf_select(cw, k, r)], 1);
    }
  } else {
    for (int j = lane; j < k; j += 32) atomicAdd(&hist[pf_select(cw, k, u[j])], 1);
  }
  __syncwarp();
  int cnt[PL], nun = 0, nex = 0, nall = 0;
#pragma unroll
  for (int t = 0; t < PL; ++t) {
    const int i = PL * lane + t;
    cnt[t] = i < k ? hist[i] : 0;
    nun += (i < k && cnt[t] == 0) ? 1 : 0;
    nex += cnt[t] > 1 ? cnt[t] - 1 : 0;
    nall += cnt[t];
  }
  if (p.dp) {
    int ru = warp_incl_scan(nun) - nun;  // rank of this lane's first unused column
#pragma unroll
    for (int t = 0; t < PL; ++t) {
      const int i = PL * lane + t;
      if (i < k && cnt[t] == 0) upos[ru++] = (int16_t)i;
      if (cnt[t] > 0) src[i] = (int16_t)i;
    }
    __syncwarp();
    int re = warp_incl_scan(nex) - nex;  // rank of this lane's first extra copy
#pragma unroll
    for (int t = 0; t < PL; ++t)
      for (int c = 1; c < cnt[t]; ++c) src[upos[re++]] = (int16_t)(PL * lane + t);
  } else {
    int q = warp_incl_scan(nall) - nall;
#pragma unroll
    for (int t = 0; t < PL; ++t)
      for (int c = 0; c < cnt[t]; ++c) src[q++] = (int16_t)(PL * lane + t);
  }
  __syncwarp();
}

// Mean / spread (k-1) / perturbation of S.x rows v < nvt, warp v per row
// (common_da.f90:354-401).  Mean into misc[v], spread into misc[8+v].
__device__ __forceinline__ void mean_spread_pert(const PointSmem &S, int kp, int k, int nvt) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int v = wid; v < nvt; v += kThreads >> 5) {
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
  cta_sync();
}

// RTPP / RTPS on the analysis in S.an (rows v < nvt) with forecast
// perturbations in S.x, then the T/S round-off (common_da.f90:99-113,
// 438-533).  Warp v per row; results stay in S.an.
__device__ __forceinline__ void relax_and_clamp(const sbletkf_params &p, const PointSmem &S, int kp, int k, int nvt,
                                                int kl, double phi) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int v = wid; v < nvt; v += kThreads >> 5) {
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
  cta_sync();
}

}  // namespace sbl
