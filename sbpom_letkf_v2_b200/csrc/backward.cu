// backward.cu -- vector-Jacobian product of the LETKF analysis (FP64).
//
// Given dJ/d anal for every member and variable, accumulate dJ/d dep and
// dJ/d rdiag per observation and dJ/d rho (cov_infl_mul), dJ/d sigma_obs
// (dist_zero held fixed, so the local observation sets do not move).  One CTA
// per grid point recomputes the point's forward problem
// (letkf/run/src/common_da.f90:67-116, common_letkf.f90:61-210):
//
//   w_o  = rloc_o / rdiag_o,  rloc_o = exp(-(d_o/sigma)^2/2 - (dlev_o/sigma_v)^2/2)
//   A    = alpha I + Y^T diag(w) Y = V Lambda V^T,  alpha = (k-1)/rho
//   b    = Y^T diag(w) dep,  wvec = A^-1 b,  W = sqrt(k-1) A^-1/2
//   anal = xm + dX (wvec 1^T + W), then RTPP / RTPS and the T/S clamp.
//
// Reverse mode, with Gb = dJ/d anal after undoing RTPP / RTPS / clamp:
//   g_wvec = dX^T Gb 1,  G_W = dX^T Gb,  G_Pa = g_wvec b^T,  u = dJ/db = A^-1 g_wvec
//   dJ/dA  = V M V^T,  M = Phi_f o (V^T G_W V) + Phi_h o (V^T G_Pa V)
// (Daleckii-Krein), where for f(l) = sqrt(k-1) l^-1/2 and h(l) = 1/l the
// divided differences have cancellation-free closed forms, valid on the
// diagonal and for repeated eigenvalues alike:
//   Phi_f(i,j) = -sqrt(k-1) / (s_i s_j (s_i + s_j)),  s = sqrt(lambda)
//   Phi_h(i,j) = -1 / (lambda_i lambda_j).
// V^T G_W V = P Q^T with P = V^T dX^T, Q = V^T Gb^T (rank <= nv), and the
// Phi_h term is rank one: V (Phi_h o p q^T) V^T = -u wvec^T.  Per local obs,
// with z = V^T y_o:
//   dJ/dw_o  = z^T M1 z - (y.u)(y.wvec) + dep_o (y.u),   M1 = Phi_f o (P Q^T)
//   dJ/ddep_o = w_o (y.u),  y.u = z.(Lambda^-1 V^T g_wvec),  y.wvec = z.c
//   dJ/drdiag_o = -dJ/dw_o rloc_o / rdiag_o^2
//   dJ/dsigma  += dJ/dw_o / rdiag_o * rloc_o d_o^2 / sigma^3
//   dJ/drho    += -tr(M) (k-1)/rho^2      (points with obs)
//               = sum(Gb o dX) / (2 sqrt(rho))  (points without: W = sqrt(rho) I)
// Every point with obs takes this k x k (primal) form; the forward's
// observation-space form for small nobsl is the same function.
#include "point.cuh"

namespace sbl {
namespace {

constexpr int kLB = kThreads + kChunk;  // list: one scan step + leftover (< kChunk)
constexpr int kZC = 32;                 // observations per pass-2 chunk
constexpr int kZG = 8;                  // observations per thread in Z = Y V

__host__ __device__ inline size_t a16b(size_t v) { return (v + 15) & ~size_t(15); }

struct BwdSmem {
  int *rowstart, *rowpref, *lidx, *iws;
  double *lw, *lwd, *lrloc, *lrdiag, *ldep, *ldist;
  double *b, *lam, *c, *pt, *vec, *misc;
  double *x, *gr, *an, *t, *q;  // [nvm][KP]
  double *V;                    // k x ldv eigenvectors (column j = v_j)
  double *U2;                   // pass-1 rows [kChunk][KP], then M1 (k x ldv)
  double *Y2, *Z2;              // pass-2 rows and their V^T y, [kZC][KP]
  int ldv;

  __host__ __device__ static int ld_of(int k) { return eig_ld(k); }
  __host__ __device__ static size_t bytes(int k, int kp, int nvm) {
    const size_t ldv = (size_t)ld_of(k);
    size_t s = a16b(sizeof(int) * kRowMax) + a16b(sizeof(int) * (kRowMax + 1)) + a16b(sizeof(int) * kLB) +
               a16b(sizeof(int) * 64);
    s += 6 * a16b(sizeof(double) * kLB);
    s += 5 * a16b(sizeof(double) * kp) + a16b(sizeof(double) * 64);
    s += 5 * a16b(sizeof(double) * nvm * kp);
    const size_t mat = sizeof(double) * (size_t)k * ldv, rows = sizeof(double) * (size_t)kChunk * kp;
    s += a16b(mat) + a16b(mat > rows ? mat : rows);
    s += 2 * a16b(sizeof(double) * (size_t)kZC * kp);
    return s;
  }
  __device__ void carve(void *base, int k, int kp, int nvm) {
    char *p = (char *)base;
    auto take = [&](size_t n) { char *r = p; p += a16b(n); return (void *)r; };
    ldv = ld_of(k);
    rowstart = (int *)take(sizeof(int) * kRowMax);
    rowpref = (int *)take(sizeof(int) * (kRowMax + 1));
    lidx = (int *)take(sizeof(int) * kLB);
    iws = (int *)take(sizeof(int) * 64);
    lw = (double *)take(sizeof(double) * kLB);
    lwd = (double *)take(sizeof(double) * kLB);
    lrloc = (double *)take(sizeof(double) * kLB);
    lrdiag = (double *)take(sizeof(double) * kLB);
    ldep = (double *)take(sizeof(double) * kLB);
    ldist = (double *)take(sizeof(double) * kLB);
    b = (double *)take(sizeof(double) * kp);
    lam = (double *)take(sizeof(double) * kp);
    c = (double *)take(sizeof(double) * kp);
    pt = (double *)take(sizeof(double) * kp);
    vec = (double *)take(sizeof(double) * kp);
    misc = (double *)take(sizeof(double) * 64);
    x = (double *)take(sizeof(double) * nvm * kp);
    gr = (double *)take(sizeof(double) * nvm * kp);
    an = (double *)take(sizeof(double) * nvm * kp);
    t = (double *)take(sizeof(double) * nvm * kp);
    q = (double *)take(sizeof(double) * nvm * kp);
    const size_t mat = sizeof(double) * (size_t)k * ldv, rows = sizeof(double) * (size_t)kChunk * kp;
    V = (double *)take(mat);
    U2 = (double *)take(mat > rows ? mat : rows);
    Y2 = (double *)take(sizeof(double) * (size_t)kZC * kp);
    Z2 = (double *)take(sizeof(double) * (size_t)kZC * kp);
  }
};

// Streaming local-observation selection in the reference's candidate order
// (count_nobsl / obs_local, common_da.f90:133-293), as in the analysis kernel.
// Accepted entries go to the list; consume(f, cnt) is called (whole CTA) for
// every kChunk entries and once for the remainder.  Returns nobsl.
template <class F>
__device__ __forceinline__ int scan_local(const sbletkf_params &p, const ObsView &ob, const BwdSmem &S, int nrows,
                                          int kl, double rdep, double plon, double plat, F &&consume) {
  const int tid = threadIdx.x;
  const int ncand = S.rowpref[nrows];
  int L = 0, nacc = 0;
  for (int base = 0; base < ncand; base += kThreads) {
    const int cnd = base + tid;
    int accept = 0, o = 0;
    double rl = 0.0, dist = 0.0;
    if (cnd < ncand) {
      int lo = 0, hi = nrows - 1;
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (S.rowpref[mid] <= cnd) lo = mid;
        else hi = mid - 1;
      }
      o = S.rowstart[lo] + (cnd - S.rowpref[lo]);
      const double dl = dlev_of(ob.elm[o], ob.lev[o], rdep, kl, p.nlev, p.id_z_obs);
      if (!(p.dist_zerov < dl)) {
        dist = distance_2p(ob.lon[o], ob.lat[o], plon, plat, p.pi, p.re);
        if (!(p.dist_zero < dist)) {
          accept = 1;
          rl = loc_weight(dist, dl, p.sigma_obs, p.sigma_obsv);
        }
      }
    }
    int excl;
    const int tot = block_excl_scan(accept, excl, S.iws);
    if (accept) {
      const int e = L + excl;
      const double rd = ob.rdiag[o], dp = ob.dep[o];
      S.lidx[e] = o;
      S.lrloc[e] = rl;
      S.lrdiag[e] = rd;
      S.ldep[e] = dp;
      S.ldist[e] = dist;
      const double w = rl / rd;
      S.lw[e] = w;
      S.lwd[e] = w * dp;
    }
    L += tot;
    nacc += tot;
    __syncthreads();
    int f = 0;
    while (L - f >= kChunk) {
      consume(f, kChunk);
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
        S.ldist[tid] = S.ldist[s];
        S.lw[tid] = S.lw[s];
        S.lwd[tid] = S.lwd[s];
      }
      __syncthreads();
    }
    L = rem;
  }
  if (L > 0) consume(0, L);
  return nacc;
}

// Copy `cnt` FP64 hdxf rows of list entries f.. into dst (row stride KP).
template <int KP>
__device__ __forceinline__ void load_rows(const ObsView &ob, const int *lidx, int f, int cnt, double *dst) {
  constexpr int KP2 = KP / 2;
  for (int e = threadIdx.x; e < cnt * KP2; e += kThreads) {
    const int cc = e / KP2, col = e - cc * KP2;
    reinterpret_cast<double2 *>(dst)[e] = reinterpret_cast<const double2 *>(ob.hdxf64 + (long)lidx[f + cc] * ob.ldh)[col];
  }
  __syncthreads();
}

template <int R, typename ST>
__global__ void __launch_bounds__(kThreads, 1)
    k_backward(const sbletkf_params p, const GridView g, const ObsView ob, const ST *__restrict__ f3,
               const ST *__restrict__ f2, const ST *__restrict__ ga3, const ST *__restrict__ ga2,
               double *__restrict__ gdep, double *__restrict__ grdiag, double *__restrict__ ginfl,
               double *__restrict__ gsig, int *status, long long p0) {
  constexpr int KP = kp_of_r(R);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int k = p.nmem, nvm = p.nv3d + p.nv2d;
  BwdSmem S;
  S.carve(smem_raw, k, KP, nvm);
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = kThreads / 32;
  const long long pid = p0 + blockIdx.x;
  const int nij1 = g.nij1, nlev = p.nlev;
  const int kl = (int)(pid / nij1), i = (int)(pid % nij1);
  __shared__ int sh[8];
  __shared__ double shd[4];
  __shared__ double sred[2][kThreads / 32];
  int bits = 0;

  // ---- search box rows (common_da.f90:158-161, 314-346)
  if (tid == 0) {
    int imin, imax, jmin, jmax;
    search_box(p, g, i, imin, imax, jmin, jmax);
    int nrows = jmax - jmin + 1;
    if (nrows < 0) nrows = 0;
    sh[5] = 0;
    if (nrows > kRowMax) {
      nrows = kRowMax;
      sh[5] = SBLETKF_ERR_ROWS;
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

  // ---- pass 1: Gram and b in FP64 registers
  PointSmem P1;  // view for the shared Gram helpers
  P1.u = S.U2;
  P1.lw = S.lw;
  P1.lwd = S.lwd;
  P1.ldep = S.ldep;
  P1.lrloc = S.lrloc;
  P1.lrdiag = S.lrdiag;
  P1.b = S.b;
  P1.ldb = S.ldv;
  Accum<R> A;
  A.zero();
  const int nacc = scan_local(p, ob, S, nrows, kl, rdep, plon, plat, [&](int f, int cnt) {
    load_rows<KP>(ob, S.lidx, f, cnt, S.U2);
    accumulate_chunk<R>(P1, f, cnt, k, true, false, A);
  });

  // ---- forecast block and dJ/d anal
  const bool surf = (kl == nlev - 1);
  const int nvt = p.nv3d + (surf ? p.nv2d : 0);
  for (int e = tid; e < nvt * k; e += kThreads) {
    const int v = e / k, m = e - v * k;
    double xv, gv;
    if (v < p.nv3d) {
      const long o = (((long)v * k + m) * nlev + kl) * nij1 + i;
      xv = (double)f3[o];
      gv = (double)ga3[o];
    } else {
      const long o = ((long)(v - p.nv3d) * k + m) * nij1 + i;
      xv = (double)f2[o];
      gv = (double)ga2[o];
    }
    S.x[v * KP + m] = xv;
    S.gr[v * KP + m] = gv;
  }
  __syncthreads();
  {
    PointSmem Px;
    Px.x = S.x;
    Px.misc = S.misc;
    mean_spread_pert(Px, KP, k, nvt);  // mean misc[v], spread misc[8+v], S.x <- dX
  }

  const double rho = p.cov_infl_mul, alpha = (double)(k - 1) / rho, sk = sqrt((double)(k - 1));
  if (nacc > 0) {
    P1.u = S.V;
    store_gram<R>(P1, k, alpha, A);  // A -> S.V, b -> S.b
    // the backward pass computes in FP64 whatever the forward precision:
    // FP64 defaults of the rotation threshold and stopping rule
    sbletkf_params p64 = p;
    p64.precision = SBLETKF_PREC_FP64;
    const double tol = jacobi_tol_of(p64, k);
    bits |= jacobi_eig<KP / 4>(S.V, k, S.ldv, tol, jacobi_stop_of(p64), p.max_sweeps, S.lam, S.iws + 40, S.lidx, S.vec);
    vt_times(S.V, k, S.ldv, S.b, S.c);
    __syncthreads();
    if (tid < k) S.c[tid] /= S.lam[tid];                    // c = Lambda^-1 V^T b
    x_times_v(S.x, KP, nvt, S.V, k, S.ldv, S.t, KP);       // T = dX V (= P^T)
    __syncthreads();
    for (int v = wid; v < nvt; v += nw) {                   // dX wvec = T c
      double s = 0.0;
      for (int j = lane; j < k; j += 32) s = fma(S.t[v * KP + j], S.c[j], s);
      s = __shfl_sync(0xffffffffu, warp_sum(s), 0);
      if (lane == 0) S.misc[16 + v] = s;
    }
    __syncthreads();
    for (int e = tid; e < nvt * k; e += kThreads) {         // anal before RTPP / RTPS
      const int v = e / k, m = e - v * k;
      double s = 0.0;
      for (int j = 0; j < k; ++j) s = fma(S.t[v * KP + j] * sqrt((double)(k - 1) / S.lam[j]), S.V[(long)j * S.ldv + m], s);
      S.an[v * KP + m] = S.misc[v] + S.misc[16 + v] + s;
    }
  } else {
    const double d = sqrt(rho);                               // letkf_core_noobs
    for (int e = tid; e < nvt * k; e += kThreads) {
      const int v = e / k, m = e - v * k;
      S.an[v * KP + m] = S.misc[v] + S.x[v * KP + m] * d;
    }
  }
  __syncthreads();

  // ---- undo the T/S clamp, RTPS or RTPP (common_da.f90:99-113, 506-533):
  //      S.gr <- dJ/d anal before relaxation
  for (int v = wid; v < nvt; v += nw) {
    const double *av = S.an + v * KP, *dxf = S.x + v * KP;
    double *gv = S.gr + v * KP;
    double s = 0.0;
    for (int m = lane; m < k; m += 32) s += av[m];
    const double am = __shfl_sync(0xffffffffu, warp_sum(s), 0) / (double)k;
    double qq = 0.0;
    for (int m = lane; m < k; m += 32) {
      const double d = av[m] - am;
      qq = fma(d, d, qq);
    }
    const double as = sqrt(__shfl_sync(0xffffffffu, warp_sum(qq), 0) / (double)(k - 1));
    const double fs = S.misc[8 + v];
    const bool rtpp = 0.0 < p.alpha_rtpp, rtps = 0.0 < p.alpha_rtps;
    double fac = 0.0;
    if (rtps) fac = (as == 0.0) ? 0.0 : p.alpha_rtps * fs / as + (1.0 - p.alpha_rtps);
    const bool clampT = p.roff && v < p.nv3d && v == p.iv3d_t && kl >= 1 && phi != 1.0;
    const bool clampS = p.roff && v < p.nv3d && v == p.iv3d_s && kl >= 1 && phi != 1.0;
    double sg = 0.0, sgd = 0.0;
    for (int m = lane; m < k; m += 32) {
      const double dxa = av[m] - am;
      double a = av[m];
      if (rtpp) a = am + p.alpha_rtpp * dxf[m] + (1.0 - p.alpha_rtpp) * dxa;
      if (rtps) a = am + dxa * fac;
      double gm = gv[m];
      if (clampT && (a < p.tmin || a > p.tmax)) gm = 0.0;
      if (clampS && (a < p.smin || a > p.smax)) gm = 0.0;
      gv[m] = gm;
      sg += gm;
      sgd = fma(gm, dxa, sgd);
    }
    sg = __shfl_sync(0xffffffffu, warp_sum(sg), 0);
    sgd = __shfl_sync(0xffffffffu, warp_sum(sgd), 0);
    const double gmean = sg / (double)k;
    if (rtps) {
      if (as == 0.0) {
        for (int m = lane; m < k; m += 32) gv[m] = gmean;
      } else {
        // a = am + dxa fac(as): d/d dxa_m = G_m fac + (sum G dxa) dfac/das das/d dxa_m
        const double coef = -p.alpha_rtps * fs / (as * as) * sgd / ((double)(k - 1) * as);
        double sd = 0.0;
        for (int m = lane; m < k; m += 32) sd += gv[m] * fac + coef * (av[m] - am);
        const double dmean = __shfl_sync(0xffffffffu, warp_sum(sd), 0) / (double)k;
        for (int m = lane; m < k; m += 32) gv[m] = gmean + gv[m] * fac + coef * (av[m] - am) - dmean;
      }
    } else if (rtpp) {
      const double r = 1.0 - p.alpha_rtpp;
      for (int m = lane; m < k; m += 32) gv[m] = gmean + r * (gv[m] - gmean);
    }
  }
  __syncthreads();

  double grho = 0.0, gsg = 0.0;  // this thread's share of the scalar gradients
  if (nacc == 0) {
    for (int e = tid; e < nvt * k; e += kThreads) {
      const int v = e / k, m = e - v * k;
      grho = fma(S.gr[v * KP + m], S.x[v * KP + m], grho);
    }
    grho *= 0.5 / sqrt(rho);
  } else {
    // Q = Gb V, gs_v = sum_m Gb[v][m], pt = V^T g_wvec = sum_v T[v] gs_v
    x_times_v(S.gr, KP, nvt, S.V, k, S.ldv, S.q, KP);
    for (int v = wid; v < nvt; v += nw) {
      double s = 0.0;
      for (int m = lane; m < k; m += 32) s += S.gr[v * KP + m];
      s = __shfl_sync(0xffffffffu, warp_sum(s), 0);
      if (lane == 0) S.misc[24 + v] = s;
    }
    __syncthreads();
    if (tid < k) {
      double s = 0.0;
      for (int v = 0; v < nvt; ++v) s = fma(S.t[v * KP + tid], S.misc[24 + v], s);
      S.pt[tid] = s / S.lam[tid];                           // Lambda^-1 V^T g_wvec
      S.vec[tid] = sqrt(S.lam[tid]);
    }
    __syncthreads();
    // M1(i,j) = Phi_f(i,j) sum_v T[v][i] Q[v][j]  (column-major, stride ldv)
    double tr = 0.0;
    for (int e = tid; e < k * k; e += kThreads) {
      const int ii = e % k, jj = e / k;
      double s = 0.0;
      for (int v = 0; v < nvt; ++v) s = fma(S.t[v * KP + ii], S.q[v * KP + jj], s);
      const double si = S.vec[ii], sj = S.vec[jj];
      const double m1 = -sk * s / (si * sj * (si + sj));
      S.U2[(long)jj * S.ldv + ii] = m1;
      if (ii == jj) tr += m1 - S.pt[ii] * S.c[ii];          // + Phi_h(i,i) pt_i qt_i
    }
    grho = -tr * (double)(k - 1) / (rho * rho);
    __syncthreads();

    // ---- pass 2: per local observation
    const double sig = p.sigma_obs, isig3 = 1.0 / (sig * sig * sig);
    scan_local(p, ob, S, nrows, kl, rdep, plon, plat, [&](int f, int cnt) {
      for (int c0 = 0; c0 < cnt; c0 += kZC) {
        const int nc = cnt - c0 < kZC ? cnt - c0 : kZC;
        load_rows<KP>(ob, S.lidx, f + c0, nc, S.Y2);
        // Z2[o][j] = sum_m Y2[o][m] V[m][j]
        for (int e = tid; e < (kZC / kZG) * KP; e += kThreads) {
          const int j = e % KP, grp = e / KP;
          if (j < k && grp * kZG < nc) {
            double acc[kZG];
#pragma unroll
            for (int o = 0; o < kZG; ++o) acc[o] = 0.0;
            const double *vj = S.V + (long)j * S.ldv;
            const double *yb = S.Y2 + grp * kZG * KP;
            for (int m = 0; m < k; ++m) {
              const double vm = vj[m];
#pragma unroll
              for (int o = 0; o < kZG; ++o) acc[o] = fma(yb[o * KP + m], vm, acc[o]);
            }
#pragma unroll
            for (int o = 0; o < kZG; ++o)
              if (grp * kZG + o < nc) S.Z2[(grp * kZG + o) * KP + j] = acc[o];
          }
        }
        __syncthreads();
        for (int o = wid; o < nc; o += nw) {
          const double *z = S.Z2 + o * KP;
          double qd = 0.0, yu = 0.0, yw = 0.0;
          for (int ii = lane; ii < k; ii += 32) {
            double ti = 0.0;
            for (int jj = 0; jj < k; ++jj) ti = fma(S.U2[(long)jj * S.ldv + ii], z[jj], ti);
            qd = fma(z[ii], ti, qd);
            yu = fma(z[ii], S.pt[ii], yu);
            yw = fma(z[ii], S.c[ii], yw);
          }
          qd = warp_sum(qd);
          yu = warp_sum(yu);
          yw = warp_sum(yw);
          if (lane == 0) {
            const int e = f + c0 + o;
            const double w = S.lw[e], dp = S.ldep[e], rl = S.lrloc[e], rd = S.lrdiag[e], ds = S.ldist[e];
            const double gw = qd - yu * yw + dp * yu;
            const int oc = ob.perm[S.lidx[e]];
            atomicAdd(gdep + oc, w * yu);
            atomicAdd(grdiag + oc, -gw * rl / (rd * rd));
            gsg = fma(gw / rd * rl, ds * ds * isig3, gsg);
          }
        }
        __syncthreads();
      }
    });
  }

  // ---- scalar gradients: block sum, one atomic per point
  grho = warp_sum(grho);
  gsg = warp_sum(gsg);
  if (lane == 0) {
    sred[0][wid] = grho;
    sred[1][wid] = gsg;
  }
  __shared__ int s_bits;
  if (tid == 0) s_bits = 0;
  __syncthreads();
  if (bits) atomicOr(&s_bits, bits);
  __syncthreads();
  if (tid == 0) {
    double a = 0.0, b2 = 0.0;
    for (int w = 0; w < nw; ++w) {
      a += sred[0][w];
      b2 += sred[1][w];
    }
    if (a != 0.0) atomicAdd(ginfl, a);
    if (b2 != 0.0) atomicAdd(gsig, b2);
    if (s_bits) atomicOr(status, s_bits);
  }
}

template <int R, typename ST>
int launch_b(const sbletkf_params *p, const GridView &g, const ObsView &ob, const void *f3, const void *f2,
             const void *ga3, const void *ga2, double *gdep, double *grdiag, double *ginfl, double *gsig,
             int *status, cudaStream_t s) {
  const size_t smem = BwdSmem::bytes(p->nmem, kp_of_r(R), p->nv3d + p->nv2d);
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SBLETKF_ERR_CUDA;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return SBLETKF_ERR_CUDA;
  if (smem + 1024 > (size_t)optin) return SBLETKF_ERR_UNSUPPORTED;
  auto kern = k_backward<R, ST>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_status(e);
  const long long P = (long long)p->nlev * g.nij1;
  const long long maxg = 2147483647LL;
  for (long long p0 = 0; p0 < P; p0 += maxg) {
    const long long n = P - p0 < maxg ? P - p0 : maxg;
    kern<<<(unsigned)n, kThreads, smem, s>>>(*p, g, ob, (const ST *)f3, (const ST *)f2, (const ST *)ga3,
                                              (const ST *)ga2, gdep, grdiag, ginfl, gsig, status, p0);
  }
  return cuda_status(cudaGetLastError());
}

template <typename ST>
int launch_bt(const sbletkf_params *p, const GridView &g, const ObsView &ob, const void *f3, const void *f2,
              const void *ga3, const void *ga2, double *gdep, double *grdiag, double *ginfl, double *gsig,
              int *status, cudaStream_t s) {
  switch (r_for_k(p->nmem)) {
    case 2: return launch_b<2, ST>(p, g, ob, f3, f2, ga3, ga2, gdep, grdiag, ginfl, gsig, status, s);
    case 4: return launch_b<4, ST>(p, g, ob, f3, f2, ga3, ga2, gdep, grdiag, ginfl, gsig, status, s);
    case 7: return launch_b<7, ST>(p, g, ob, f3, f2, ga3, ga2, gdep, grdiag, ginfl, gsig, status, s);
    default: return SBLETKF_ERR_UNSUPPORTED;  // k > 112: two k x k FP64 matrices exceed shared memory
  }
}

}  // namespace

int launch_backward(sbletkf_workspace *ws, const sbletkf_params *p, const GridView &g, const void *f3,
                    const void *f2, int dtype, const void *ga3, const void *ga2, double *gdep, double *grdiag,
                    double *ginfl, double *gsig, cudaStream_t s) {
  if (ws->nobs == 0) return SBLETKF_OK;  // anal = fcst (common_da.f90:57-61): every gradient is zero
  const ObsView ob = ws->obs_view();
  if (dtype == SBLETKF_F64)
    return launch_bt<double>(p, g, ob, f3, f2, ga3, ga2, gdep, grdiag, ginfl, gsig, ws->d_status, s);
  return launch_bt<float>(p, g, ob, f3, f2, ga3, ga2, gdep, grdiag, ginfl, gsig, ws->d_status, s);
}

}  // namespace sbl
