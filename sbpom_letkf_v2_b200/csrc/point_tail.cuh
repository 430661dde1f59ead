// point_tail.cuh -- the second half of one grid point's analysis, shared by
// the analysis kernels: the transform (observation-space form for the dual
// points, eigensolve of G + alpha I for the others, letkf_core /
// lpfgm_core, common_letkf.f90:61-210, common_lpfgm.f90:444-494), the
// ensemble update (Analysis_Ensemble, common_da.f90:407-432), the PF draws
// and gather, RTPP / RTPS / round-off (:438-533) and the store.
#pragma once

#include "point.cuh"

namespace sbl {

// Whole CTA (kThreads threads).  On entry, for a primal point (nacc > 0, not
// dual, Gram computed): S.u holds G + alpha I (column-major, stride S.ldb)
// and S.b holds b = Y^T diag(rloc/rdiag) dep; for a dual point S.lidx,
// S.lw, S.ldep, S.lrloc, S.lrdiag hold its nacc local observations.  llv:
// this thread's PF log-likelihood accumulated so far (member tid < k).
// vprev / warm: the warm-start state of the column schedule (vprev
// nullptr: cold eigensolves).  tc_on: the tensor cores ran this launch
// (a timed-out wait in bits is latched into *status at once).
template <int R, typename ST, bool EIG_CALL = false>
__device__ __forceinline__ void point_tail(const sbletkf_params &p, const ObsView &ob, const ST *__restrict__ f3,
                                           const ST *__restrict__ f2, ST *__restrict__ a3, ST *__restrict__ a2,
                                           const double *__restrict__ uni, int32_t *__restrict__ src_out,
                                           int32_t *__restrict__ pst, int *status, const PointSmem &S,
                                           long long pid, int nij1, double phi, int nacc, bool dual, double llv,
                                           int bits, bool tc_on, double *vprev, int &warm) {
  constexpr int KP = kp_of_r(R);
  const int k = p.nmem;
  const int tid = threadIdx.x;
  const int nlev = p.nlev;
  const int kl = (int)(pid / nij1), i = (int)(pid % nij1);
  const bool do_pf = p.iswitch_da != SBLETKF_DA_LETKF;
  const bool do_gram = p.iswitch_da != SBLETKF_DA_LPF;
  const int ndm = do_gram ? PointSmem::dual_max(k) : -1;
  const bool surf = (kl == nlev - 1);
  const int nvt = p.nv3d + (surf ? p.nv2d : 0);
  const int n = nacc;
  const int ldz = KP + 1, ldn = eig_ld(n);
  double *Z = S.u, *Nb = S.u + (long)ndm * ldz;
  const double alpha_d = (double)(k - 1) / (p.iswitch_da == SBLETKF_DA_LETKF ? p.cov_infl_mul : p.cov_infl_gm);
  if (dual) {
    // rows of the n local obs, then (LPFGM) the PF log-likelihood in obs order
    for (int e = tid; e < n * KP; e += kThreads) {
      const int o = e / KP, m = e - o * KP;
      Z[o * ldz + m] = ob.hdxf64[(long)S.lidx[o] * ob.ldh + m];
    }
    cta_sync();
    if (do_pf && tid < k) {
      double ll = llv;
      for (int o = 0; o < n; ++o) {
        double d = __dsub_rn(S.ldep[o], Z[o * ldz + tid]);
        double q = __dmul_rn(__dmul_rn(0.5, d), d);
        q = __ddiv_rn(__dmul_rn(q, S.lrloc[o]), S.lrdiag[o]);
        ll = __dsub_rn(ll, q);
      }
      llv = ll;
    }
    cta_sync();
    for (int e = tid; e < n * KP; e += kThreads) {
      const int o = e / KP, m = e - o * KP;
      Z[o * ldz + m] *= sqrt(S.lw[o]);
    }
    if (tid < n) S.b[tid] = sqrt(S.lw[tid]) * S.ldep[tid];
    cta_sync();
    for (int e = tid; e < n * n; e += kThreads) {  // N = alpha I + Z Z^T
      const int r = e % n, c = e / n;
      if (r <= c) {
        double s = 0.0;
        for (int m = 0; m < k; ++m) s = fma(Z[r * ldz + m], Z[c * ldz + m], s);
        if (r == c) s += alpha_d;
        Nb[(long)c * ldn + r] = s;
        Nb[(long)r * ldn + c] = s;
      }
    }
    cta_sync();
    const double tol = jacobi_tol_of(p, k);
    constexpr int ED = KP / 4 < 16 ? KP / 4 : 16;
    bits |= EIG_CALL ? jacobi_eig_call<ED>(Nb, n, ldn, tol, jacobi_stop_of(p), p.max_sweeps, S.lam, S.iws + 40, S.lidx, S.cw)
                     : jacobi_eig<ED>(Nb, n, ldn, tol, jacobi_stop_of(p), p.max_sweeps, S.lam, S.iws + 40, S.lidx, S.cw);
    vt_times(Nb, n, ldn, S.b, S.c);  // c = Lambda^-1 Q^T d
    cta_sync();
    if (tid < n) S.c[tid] /= S.lam[tid];
  }
  if (!dual && nacc > 0 && do_gram) {
    const double tol = jacobi_tol_of(p, k);
    if (vprev && warm)  // start from the previous level's eigenvectors
      bits |= EIG_CALL ? jacobi_eig_warm_call<KP / 4>(S.u, k, S.ldb, tol, jacobi_stop_of(p), p.max_sweeps, S.lam,
                                                      S.iws + 40, S.cw, vprev)
                       : jacobi_eig_warm<KP / 4>(S.u, k, S.ldb, tol, jacobi_stop_of(p), p.max_sweeps, S.lam, S.iws + 40,
                                                 S.cw, vprev);
    else
      bits |= EIG_CALL ? jacobi_eig_call<KP / 4>(S.u, k, S.ldb, tol, jacobi_stop_of(p), p.max_sweeps, S.lam, S.iws + 40,
                                                 S.lidx, S.cw)
                       : jacobi_eig<KP / 4>(S.u, k, S.ldb, tol, jacobi_stop_of(p), p.max_sweeps, S.lam, S.iws + 40,
                                            S.lidx, S.cw);
    if (vprev) {  // keep this level's eigenvectors for the next one
      for (int e = tid; e < k * k; e += kThreads) vprev[e] = S.u[(long)(e / k) * S.ldb + (e % k)];
      warm = 1;
    }
    vt_times(S.u, k, S.ldb, S.b, S.c);  // c = Lambda^-1 V^T b
    cta_sync();
    if (tid < k) S.c[tid] /= S.lam[tid];
  }
  if (do_pf && tid < k) S.ll[tid] = llv;

  // ---- forecast block: x, mean, spread, perturbation
  for (int e = tid; e < nvt * k; e += kThreads) {
    const int v = e / k, m = e - v * k;
    double xv;
    if (v < p.nv3d) xv = (double)f3[(((long)v * k + m) * nlev + kl) * nij1 + i];
    else xv = (double)f2[((long)(v - p.nv3d) * k + m) * nij1 + i];
    S.x[v * KP + m] = xv;
  }
  cta_sync();
  mean_spread_pert(S, KP, k, nvt);

  const double *B = S.u;
  if (dual) {
    const bool letkf = p.iswitch_da == SBLETKF_DA_LETKF;
    for (int e = tid; e < nvt * n; e += kThreads) {  // P = dX Z^T
      const int v = e / n, o = e - v * n;
      const double *xv = S.x + v * KP, *zo = Z + o * ldz;
      double s = 0.0;
      for (int m = 0; m < k; ++m) s = fma(xv[m], zo[m], s);
      S.t[v * KP + o] = s;
    }
    cta_sync();
    for (int e = tid; e < nvt * n; e += kThreads) {  // Pq = P Q
      const int v = e / n, j = e - v * n;
      const double *qj = Nb + (long)j * ldn, *pv = S.t + v * KP;
      double s = 0.0;
      for (int o = 0; o < n; ++o) s = fma(pv[o], qj[o], s);
      S.w[v * KP + j] = s;
    }
    cta_sync();
    {
      const int lane = tid & 31, wid = tid >> 5;
      for (int v = wid; v < nvt; v += kThreads / 32) {  // dX wvec = Pq Lambda^-1 Q^T d
        double s = 0.0;
        for (int j = lane; j < n; j += 32) s = fma(S.w[v * KP + j], S.c[j], s);
        s = __shfl_sync(0xffffffffu, warp_sum(s), 0);
        if (lane == 0) S.misc[16 + v] = s;
      }
    }
    cta_sync();
    const double sa = sqrt(alpha_d);
    for (int e = tid; e < nvt * n; e += kThreads) {
      const int v = e / n, j = e - v * n;
      const double lj = S.lam[j];
      S.w[v * KP + j] *= letkf ? -1.0 / (sqrt(alpha_d * lj) * (sqrt(lj) + sa)) : 1.0 / lj;
    }
    cta_sync();
    for (int e = tid; e < nvt * n; e += kThreads) {  // Sq = (Pq g) Q^T
      const int v = e / n, o = e - v * n;
      const double *wv = S.w + v * KP;
      double s = 0.0;
      for (int j = 0; j < n; ++j) s = fma(wv[j], Nb[(long)j * ldn + o], s);
      S.t[v * KP + o] = s;
    }
    cta_sync();
    // LETKF: anal = xm + dX wvec + sqrt(k-1) (alpha^-1/2 dX + Sq Z)
    // LPFGM: U = dX W_GM = (dX w) 1^T + dX - (dX Z^T Q Lambda^-1 Q^T) Z
    const double sk = sqrt((double)(k - 1)), isa = 1.0 / sa;
    for (int e = tid; e < nvt * k; e += kThreads) {
      const int v = e / k, m = e - v * k;
      const double *tv = S.t + v * KP;
      double s = 0.0;
      for (int o = 0; o < n; ++o) s = fma(tv[o], Z[o * ldz + m], s);
      const double dx = S.x[v * KP + m];
      if (letkf) S.an[v * KP + m] = S.misc[v] + S.misc[16 + v] + sk * (isa * dx + s);
      else S.w[v * KP + m] = S.misc[16 + v] + dx - s;
    }
    cta_sync();
  } else if (nacc > 0 && do_gram) {
    x_times_v(S.x, KP, nvt, B, k, S.ldb, S.t, KP);  // T = dX V
    cta_sync();
    {  // mean increment dX wvec = T c (LETKF), or dX w_gm (LPFGM)
      const int lane = tid & 31, wid = tid >> 5;
      for (int v = wid; v < nvt; v += kThreads / 32) {
        double s = 0.0;
        for (int j = lane; j < k; j += 32) s = fma(S.t[v * KP + j], S.c[j], s);
        s = __shfl_sync(0xffffffffu, warp_sum(s), 0);
        if (lane == 0) S.misc[16 + v] = s;
      }
    }
    cta_sync();
    const bool letkf = p.iswitch_da == SBLETKF_DA_LETKF;
    for (int e = tid; e < nvt * k; e += kThreads) {
      const int v = e / k, j = e - v * k;
      const double lj = S.lam[j];
      S.t[v * KP + j] *= letkf ? sqrt((double)(k - 1) / lj) : 1.0 / lj;
    }
    cta_sync();
    // LETKF: anal = xm + dX wvec + T2 V^T
    // LPFGM: U = dX W_GM = (dX w) 1^T + alpha dX Pa  (W_GM = w 1^T + alpha Pa,
    //        equal to I + Pa (R^-1 Y)^T (dep 1^T - Y) of gm_core, common_lpfgm.f90:384-397)
    const double agm = (double)(k - 1) / p.cov_infl_gm;
    double *dst = letkf ? S.an : S.w;
    for (int e = tid; e < nvt * k; e += kThreads) {
      const int v = e / k, m = e - v * k;
      const double *tv = S.t + v * KP;
      double s = 0.0;
      for (int j = 0; j < k; ++j) s = fma(tv[j], B[(long)j * S.ldb + m], s);
      dst[v * KP + m] = letkf ? S.misc[v] + S.misc[16 + v] + s : S.misc[16 + v] + agm * s;
    }
    cta_sync();
  } else if (!do_pf || nacc == 0) {
    // letkf_core_noobs: W = sqrt(rho) I ; lpfgm_core_noobs: W = I
    const double d = (p.iswitch_da == SBLETKF_DA_LETKF) ? sqrt(p.cov_infl_mul) : 1.0;
    for (int e = tid; e < nvt * k; e += kThreads) {
      const int v = e / k, m = e - v * k;
      S.an[v * KP + m] = S.misc[v] + S.x[v * KP + m] * d;
    }
    cta_sync();
  }

  if (do_pf && nacc > 0) {
    // LPF weights and nmonte resamplings; anal_j = xm + mean_d U[src_d(j)]
    pf_weights(S, k);
    const double *U = (p.iswitch_da == SBLETKF_DA_LPF) ? S.x : S.w;
    int16_t *srcb = reinterpret_cast<int16_t *>(S.u);
    const int wid = tid >> 5, lane = tid & 31;
    int *whist = reinterpret_cast<int *>(srcb + kDrawBatch * k) + wid * k;
    int16_t *wup = reinterpret_cast<int16_t *>(reinterpret_cast<int *>(srcb + kDrawBatch * k) + (kThreads / 32) * k) +
                   wid * k;
    for (int e = tid; e < nvt * k; e += kThreads) S.an[(e / k) * KP + e % k] = 0.0;
    for (int d0 = 0; d0 < p.nmonte; d0 += kDrawBatch) {
      const int nb = min(kDrawBatch, p.nmonte - d0);
      cta_sync();
      for (int t = wid; t < nb; t += kThreads / 32) {  // a warp per draw
        const int d = d0 + t;
        const double *u = (p.rm == SBLETKF_RM_SR) ? uni + pid * p.nmonte + d : uni + (pid * p.nmonte + d) * k;
        int16_t *sr = srcb + t * k;
        resample_draw(p, S.cw, k, u, whist, wup, sr);
        if (src_out) {
          int32_t *so = src_out + (pid * p.nmonte + d) * k;
          for (int j = lane; j < k; j += 32) so[j] = sr[j];
        }
      }
      cta_sync();
      for (int e = tid; e < nvt * k; e += kThreads) {
        const int v = e / k, j = e - v * k;
        double s = S.an[v * KP + j];
        for (int t = 0; t < nb; ++t) s += U[v * KP + srcb[t * k + j]];
        S.an[v * KP + j] = s;
      }
    }
    cta_sync();
    const double inv = 1.0 / (double)p.nmonte;
    for (int e = tid; e < nvt * k; e += kThreads) {
      const int v = e / k, j = e - v * k;
      S.an[v * KP + j] = S.misc[v] + S.an[v * KP + j] * inv;
    }
    cta_sync();
  }

  // ---- RTPP / RTPS / round-off, then store
  relax_and_clamp(p, S, KP, k, nvt, kl, phi);
  for (int e = tid; e < nvt * k; e += kThreads) {
    const int v = e / k, m = e - v * k;
    const double a = S.an[v * KP + m];
    if (v < p.nv3d) a3[(((long)v * k + m) * nlev + kl) * nij1 + i] = (ST)a;
    else a2[((long)(v - p.nv3d) * k + m) * nij1 + i] = (ST)a;
  }
  if (tc_on && (bits & SBLETKF_ERR_TIMEOUT)) atomicOr(status, SBLETKF_ERR_TIMEOUT);
  __shared__ int s_bits;
  if (tid == 0) s_bits = 0;
  cta_sync();
  if (bits) atomicOr(&s_bits, bits);
  cta_sync();
  bits = s_bits;
  if (tid == 0) {
    if (pst) pst[pid] = bits;
    if (bits) atomicOr(status, bits);
  }
}

}  // namespace sbl
