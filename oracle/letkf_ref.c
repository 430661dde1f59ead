/*
 * letkf_ref.c -- C/OpenMP restatement of the sbPOM-LETKF analysis step.
 *
 * TEST INFRASTRUCTURE ONLY: loaded by tests/ (as a second oracle), by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline / reference leg.
 * The product library never links or calls it.
 *
 * It restates the reference's Fortran structure (paths relative to the
 * reference project, src/ = letkf/run/src/):
 *   da_main            src/common_da.f90:22-124   (OpenMP dynamic over (k,i))
 *   count_nobsl        src/common_da.f90:133-205  (first candidate scan)
 *   obs_local          src/common_da.f90:209-293  (second candidate scan)
 *   obs_local_sub      src/common_da.f90:297-348
 *   letkf_core(_noobs) src/common_letkf.f90:37-210 (GEMM sequence)
 *   lpf/gm/lpfgm_core  src/common_lpfgm.f90:38-494
 *   mtx_eigen          src/common.f90:992-1050    (LAPACK dsyev 'V','U')
 *   distance_2p        src/common.f90:79-101
 *   update, RTPP, RTPS, round_off  src/common_da.f90:354-533
 * Compiled twice: RSIZE=8 (r_size = binary64, the parity target) and RSIZE=4
 * (r_size = binary32, the reference's default build, common_setting.f90:20).
 * BLAS/LAPACK (the reference links Fujitsu SSL2) are reached through function
 * pointers set by ref_set_lapack(); the loader passes OpenBLAS's dgemm/sgemm/
 * dsyev from scipy's cython_blas / cython_lapack capsules.
 * One deliberate difference: the per-call ALLOCATE(nobs_use(nobs)) scratch of
 * count_nobsl / obs_local is a per-thread buffer allocated once.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/sbletkf.h"

#ifndef RSIZE
#define RSIZE 8
#endif

#if RSIZE == 8
typedef double real;
#define SUFFIX(x) x##64
#else
typedef float real;
#define SUFFIX(x) x##32
#endif

typedef void (*dgemm_fn)(char *, char *, int *, int *, int *, double *, double *, int *,
                         double *, int *, double *, double *, int *);
typedef void (*sgemm_fn)(char *, char *, int *, int *, int *, float *, float *, int *,
                         float *, int *, float *, float *, int *);
typedef void (*dsyev_fn)(char *, char *, int *, double *, int *, double *, double *, int *, int *);

static dgemm_fn p_dgemm;
static sgemm_fn p_sgemm;
static dsyev_fn p_dsyev;

void SUFFIX(ref_set_lapack)(void *dsyev, void *dgemm, void *sgemm) {
  p_dsyev = (dsyev_fn)dsyev;
  p_dgemm = (dgemm_fn)dgemm;
  p_sgemm = (sgemm_fn)sgemm;
}

static void gemm(char ta, char tb, int m, int n, int k, real *a, int lda, real *b, int ldb, real *c, int ldc) {
#if RSIZE == 8
  double one = 1.0, zero = 0.0;
  p_dgemm(&ta, &tb, &m, &n, &k, &one, a, &lda, b, &ldb, &zero, c, &ldc);
#else
  float one = 1.0f, zero = 0.0f;
  p_sgemm(&ta, &tb, &m, &n, &k, &one, a, &lda, b, &ldb, &zero, c, &ldc);
#endif
}

/* Fortran NINT: halves away from zero */
static long fnint(double x) { return lround(x); }

/* src/common.f90:79-101 */
static real distance_2p(real lona, real lata, real lonb, real latb, real pi, real re) {
  double cosd = sin(pi * lata / 180.0) * sin(pi * latb / 180.0) +
                cos(pi * lata / 180.0) * cos(pi * latb / 180.0) * cos(pi * (lonb - lona) / 180.0);
  real c = (real)cosd;
  if (c > 1.0) c = 1.0;
  if (c < -1.0) c = -1.0;
  return re * (real)acos((double)c);
}

typedef struct {
  const sbletkf_params *p;
  int nij1;
  const double *lon1, *lat1, *ri1, *rj1, *dlon1, *dlat1, *phi1, *depth1;
  int nobs;
  const int64_t *cellstart; /* [nlon*nlat+1] sorted-position starts */
  const int32_t *elm;
  const real *lon, *lat, *lev, *err, *dep;
  const real *hdxf; /* [nobs][nmem] sorted, row per obs */
} ctx_t;

/* obs_local_sub: candidates of rows jmin..jmax, cells imin..imax (common_da.f90:297-348) */
static int obs_local_sub(const ctx_t *c, int imin, int imax, int jmin, int jmax, int *use) {
  int no = 0, nlon = c->p->nlon;
  for (int j = jmin; j <= jmax; ++j) {
    int64_t ib = c->cellstart[(int64_t)(j - 1) * nlon + (imin - 1)];
    int64_t ie = c->cellstart[(int64_t)(j - 1) * nlon + imax];
    for (int64_t ip = ib; ip < ie; ++ip) use[no++] = (int)ip;
  }
  return no;
}

static void search_box(const ctx_t *c, int i, int *imin, int *imax, int *jmin, int *jmax) {
  const sbletkf_params *p = c->p;
  real dz = (real)p->dist_zero;
  real a = (real)c->ri1[i] - dz / (real)c->dlon1[i];
  real b = (real)c->ri1[i] + dz / (real)c->dlon1[i];
  real d = (real)c->rj1[i] - dz / (real)c->dlat1[i];
  real e = (real)c->rj1[i] + dz / (real)c->dlat1[i];
  long v;
  v = fnint(a); *imin = v > 1 ? (int)v : 1;
  v = fnint(b); *imax = v < p->nlon ? (int)v : p->nlon;
  v = fnint(d); *jmin = v > 1 ? (int)v : 1;
  v = fnint(e); *jmax = v < p->nlat ? (int)v : p->nlat;
}

static real dlev_of(const ctx_t *c, int o, int k, real rdep) {
  const sbletkf_params *p = c->p;
  if (c->elm[o] == p->id_z_obs && k < p->nlev - 1) return (real)fabs((double)rdep);
  if (c->elm[o] != p->id_z_obs) return (real)fabs((double)(c->lev[o] - rdep));
  return 0;
}

/* count_nobsl (common_da.f90:133-205) */
static int count_nobsl(const ctx_t *c, int i, int k, real rdep, int *use) {
  int imin, imax, jmin, jmax;
  search_box(c, i, &imin, &imax, &jmin, &jmax);
  int no = obs_local_sub(c, imin, imax, jmin, jmax, use);
  int nobsl = 0;
  real dzv = (real)c->p->dist_zerov, dz = (real)c->p->dist_zero;
  for (int io = 0; io < no; ++io) {
    int o = use[io];
    real dlev = dlev_of(c, o, k, rdep);
    if (dzv < dlev) continue;
    real dist = distance_2p(c->lon[o], c->lat[o], (real)c->lon1[i], (real)c->lat1[i], (real)c->p->pi, (real)c->p->re);
    if (dz < dist) continue;
    ++nobsl;
  }
  return nobsl;
}

/* obs_local (common_da.f90:209-293); hdxf is the Fortran hdxf(nobsl,nmem) */
static void obs_local(const ctx_t *c, int i, int k, int nobsl, real rdep, int *use, real *hdxf, real *rdiag,
                      real *rloc, real *dep) {
  const sbletkf_params *p = c->p;
  int imin, imax, jmin, jmax, nmem = p->nmem;
  search_box(c, i, &imin, &imax, &jmin, &jmax);
  int no = obs_local_sub(c, imin, imax, jmin, jmax, use);
  int iobsl = 0;
  real dzv = (real)p->dist_zerov, dz = (real)p->dist_zero;
  for (int io = 0; io < no; ++io) {
    int o = use[io];
    real dlev = dlev_of(c, o, k, rdep);
    if (dzv < dlev) continue;
    real dist = distance_2p(c->lon[o], c->lat[o], (real)c->lon1[i], (real)c->lat1[i], (real)p->pi, (real)p->re);
    if (dz < dist) continue;
    if (iobsl >= nobsl) break;
    for (int m = 0; m < nmem; ++m) hdxf[(int64_t)m * nobsl + iobsl] = c->hdxf[(int64_t)o * nmem + m];
    dep[iobsl] = c->dep[o];
    rdiag[iobsl] = (real)((double)c->err[o] * (double)c->err[o]);
    double so = p->sigma_obs, sv = p->sigma_obsv;
    if (sv <= 0.0)
      rloc[iobsl] = (real)exp(-0.5 * ((double)dist / so) * ((double)dist / so));
    else
      rloc[iobsl] = (real)exp(-0.5 * (((double)dist / so) * ((double)dist / so) + ((double)dlev / sv) * ((double)dlev / sv)));
    ++iobsl;
  }
}

typedef struct {
  real *rlinv, *work1, *work2, *work3, *wmat, *wvec, *wtmp, *wgm;
  double *evec, *eval, *dwork, *wgt, *cwgt, *rand, *rs;
  int *inum, *used;
} core_buf_t;

/* mtx_eigen (common.f90:992-1050): returns 0 ok, else status bits */
static int mtx_eigen(int n, const real *a, double *eval, double *evec, double *work) {
  int lwork = 3 * n - 1, info = 0;
  char jobz = 'V', uplo = 'U';
  double *ev8 = work + lwork; /* n */
  for (int64_t t = 0; t < (int64_t)n * n; ++t) evec[t] = (double)a[t];
  p_dsyev(&jobz, &uplo, &n, evec, &n, ev8, work, &lwork, &info);
  if (info != 0) return SBLETKF_ERR_EIG_NOCONV;
  if (ev8[n - 1] < 0) return SBLETKF_ERR_EIG_NEG;
  for (int i = 0; i < n; ++i)
    if (ev8[i] < 0.0) {
      ev8[i] = 0.0;
      for (int r = 0; r < n; ++r) evec[(int64_t)i * n + r] = 0.0;
    }
  /* reverse to descending order */
  for (int i = 0; i < n / 2; ++i) {
    int j = n - 1 - i;
    double t = ev8[i]; ev8[i] = ev8[j]; ev8[j] = t;
    for (int r = 0; r < n; ++r) {
      double u = evec[(int64_t)i * n + r];
      evec[(int64_t)i * n + r] = evec[(int64_t)j * n + r];
      evec[(int64_t)j * n + r] = u;
    }
  }
  for (int i = 0; i < n; ++i) eval[i] = ev8[i];
  return 0;
}

/* Shared front half of letkf_core / gm_core: Pa (work3) and work2 = Pa Rlinv^T.
 * common_letkf.f90:93-172 with infl = cov_infl_mul or cov_infl_gm. */
static int letkf_front(int nmem, int nobsl, const real *hdxf, const real *rdiag, const real *rloc, double infl,
                       core_buf_t *b) {
  for (int j = 0; j < nmem; ++j)
    for (int i = 0; i < nobsl; ++i)
      b->rlinv[(int64_t)j * nobsl + i] = hdxf[(int64_t)j * nobsl + i] * rloc[i] / rdiag[i];
  gemm('t', 'n', nmem, nmem, nobsl, b->rlinv, nobsl, (real *)hdxf, nobsl, b->work1, nmem);
  for (int i = 0; i < nmem; ++i) b->work1[(int64_t)i * nmem + i] += (real)(nmem - 1) / (real)infl;
  int st = mtx_eigen(nmem, b->work1, b->eval, b->evec, b->dwork);
  if (st) return st;
  for (int j = 0; j < nmem; ++j)
    for (int i = 0; i < nmem; ++i) b->work1[(int64_t)j * nmem + i] = (real)(b->evec[(int64_t)j * nmem + i] / b->eval[j]);
  real *evr = b->wgm; /* REAL(evec, r_size) */
  for (int64_t t = 0; t < (int64_t)nmem * nmem; ++t) evr[t] = (real)b->evec[t];
  gemm('n', 't', nmem, nmem, nmem, b->work1, nmem, evr, nmem, b->work3, nmem);
  gemm('n', 't', nmem, nobsl, nmem, b->work3, nmem, b->rlinv, nobsl, b->work2, nmem);
  return 0;
}

/* letkf_core (common_letkf.f90:61-210) */
static int letkf_core(const sbletkf_params *p, int nobsl, const real *hdxf, const real *rdiag, const real *rloc,
                      const real *dep, core_buf_t *b) {
  int nmem = p->nmem;
  int st = letkf_front(nmem, nobsl, hdxf, rdiag, rloc, p->cov_infl_mul, b);
  if (st) return st;
  for (int i = 0; i < nmem; ++i) {
    real w = b->work2[i] * dep[0];
    for (int j = 1; j < nobsl; ++j) w = w + b->work2[(int64_t)j * nmem + i] * dep[j];
    b->wvec[i] = w;
  }
  for (int j = 0; j < nmem; ++j)
    for (int i = 0; i < nmem; ++i)
      b->work1[(int64_t)j * nmem + i] = (real)(b->evec[(int64_t)j * nmem + i] * sqrt((double)(real)(nmem - 1) / b->eval[j]));
  real *evr = b->wgm;
  for (int64_t t = 0; t < (int64_t)nmem * nmem; ++t) evr[t] = (real)b->evec[t];
  gemm('n', 't', nmem, nmem, nmem, b->work1, nmem, evr, nmem, b->wmat, nmem);
  return 0;
}

static void noobs(const sbletkf_params *p, core_buf_t *b, double diag) {
  int nmem = p->nmem;
  memset(b->wmat, 0, sizeof(real) * (size_t)nmem * nmem);
  for (int i = 0; i < nmem; ++i) b->wmat[(int64_t)i * nmem + i] = (real)diag;
  memset(b->wvec, 0, sizeof(real) * (size_t)nmem);
}

/* lpf_core (common_lpfgm.f90:213-263) into wmat; src optional [nmonte][nmem] */
static void lpf_core(const sbletkf_params *p, int nobsl, const real *hdxf, const real *rdiag, const real *rloc,
                     const real *dep, const double *uni, int32_t *src, real *wout, core_buf_t *b) {
  int k = p->nmem;
  double *ll = b->wgt;
  for (int j = 0; j < k; ++j) ll[j] = 0.0;
  for (int j = 0; j < k; ++j)
    for (int i = 0; i < nobsl; ++i) {
      real d = dep[i] - hdxf[(int64_t)j * nobsl + i];
      ll[j] = ll[j] - 0.5 * (double)d * (double)d * (double)rloc[i] / (double)rdiag[i];
    }
  double mx = ll[0];
  for (int j = 1; j < k; ++j) mx = ll[j] > mx ? ll[j] : mx;
  double s = 0.0;
  for (int j = 0; j < k; ++j) { ll[j] = exp(ll[j] - mx); }
  for (int j = 0; j < k; ++j) s = s + ll[j];
  for (int j = 0; j < k; ++j) ll[j] = ll[j] / s;
  b->cwgt[0] = ll[0];
  for (int i = 1; i < k; ++i) b->cwgt[i] = b->cwgt[i - 1] + ll[i];
  for (int64_t t = 0; t < (int64_t)k * k; ++t) wout[t] = 0;
  for (int d = 0; d < p->nmonte; ++d) {
    double *r = b->rand;
    if (p->rm == SBLETKF_RM_SR) {
      double u = uni[d];
      r[0] = (u + 1.0 - 1.0) / (double)k;
      double base = p->sr_textbook ? u : r[0];
      for (int i = 2; i <= k; ++i) r[i - 1] = (base + (double)i - 1.0) / (double)k;
    } else {
      for (int i = 0; i < k; ++i) r[i] = uni[(int64_t)d * k + i];
      for (int i = 1; i < k; ++i) { /* ascending sort; only the values matter */
        double x = r[i]; int j = i - 1;
        while (j >= 0 && r[j] > x) { r[j + 1] = r[j]; --j; }
        r[j + 1] = x;
      }
    }
    int *inum = b->inum, *used = b->used;
    for (int j = 0; j < k; ++j) {
      int hit = k - 1;
      for (int i = 0; i < k; ++i)
        if (r[j] <= b->cwgt[i] || i == k - 1) { hit = i; break; }
      inum[j] = hit;
    }
    int *col_src = b->used + k; /* member -> particle */
    if (p->dp) {
      for (int i = 0; i < k; ++i) used[i] = 0;
      for (int i = 0; i < k; ++i) {
        int kk = inum[i];
        if (used[kk]) continue;
        col_src[kk] = kk; used[kk] = 1; inum[i] = -1;
      }
      for (int i = 0; i < k; ++i) {
        if (inum[i] < 0) continue;
        for (int kk = 0; kk < k; ++kk) {
          if (used[kk]) continue;
          col_src[kk] = inum[i]; used[kk] = 1; inum[i] = -1;
          break;
        }
      }
    } else {
      for (int j = 0; j < k; ++j) col_src[j] = inum[j];
    }
    for (int j = 0; j < k; ++j) {
      wout[(int64_t)j * k + col_src[j]] = wout[(int64_t)j * k + col_src[j]] + (real)(1.0 / (double)p->nmonte);
      if (src) src[(int64_t)d * k + j] = col_src[j];
    }
  }
}

/* gm_core (common_lpfgm.f90:279-405) into wout */
static int gm_core(const sbletkf_params *p, int nobsl, const real *hdxf, const real *rdiag, const real *rloc,
                   const real *dep, real *wout, core_buf_t *b) {
  int k = p->nmem;
  int st = letkf_front(k, nobsl, hdxf, rdiag, rloc, p->cov_infl_gm, b);
  if (st) return st;
  for (int kk = 0; kk < k; ++kk)
    for (int i = 0; i < k; ++i) {
      real w = b->work2[i] * (dep[0] - hdxf[(int64_t)kk * nobsl + 0]);
      for (int j = 1; j < nobsl; ++j) w = w + b->work2[(int64_t)j * k + i] * (dep[j] - hdxf[(int64_t)kk * nobsl + j]);
      wout[(int64_t)kk * k + i] = w;
    }
  for (int i = 0; i < k; ++i) wout[(int64_t)i * k + i] += (real)1.0;
  return 0;
}

/* Ensemble_Mean_Spread_Perturbation (common_da.f90:354-401); x is x(nmem,nvd) */
static void emsp(int nmem, int nvd, const real *x, real *m, real *s, real *dx) {
  for (int v = 0; v < nvd; ++v) {
    real a = 0;
    for (int j = 0; j < nmem; ++j) a = a + x[(int64_t)v * nmem + j];
    m[v] = a / (real)nmem;
  }
  for (int v = 0; v < nvd; ++v) {
    real a = 0;
    for (int j = 0; j < nmem; ++j) {
      real d = x[(int64_t)v * nmem + j] - m[v];
      a = a + d * d;
    }
    s[v] = (real)sqrt((double)(a / (real)(nmem - 1)));
  }
  for (int v = 0; v < nvd; ++v)
    for (int j = 0; j < nmem; ++j) dx[(int64_t)v * nmem + j] = x[(int64_t)v * nmem + j] - m[v];
}

/* Analysis_Ensemble + RTPP + RTPS for one block x(nmem,nvd) -> an(nmem,nvd) (common_da.f90:88-113) */
static void update_block(const sbletkf_params *p, int nvd, const real *x, const real *wvec, const real *wmat, real *an,
                         real *tmp) {
  int k = p->nmem;
  real *fm = tmp, *fs = fm + 8, *am = fs + 8, *as = am + 8, *dxf = as + 8, *dxa = dxf + (int64_t)k * 8;
  emsp(k, nvd, x, fm, fs, dxf);
  for (int v = 0; v < nvd; ++v)
    for (int j = 0; j < k; ++j) {
      real a = fm[v];
      for (int i = 0; i < k; ++i) a = a + dxf[(int64_t)v * k + i] * (wvec[i] + wmat[(int64_t)j * k + i]);
      an[(int64_t)v * k + j] = a;
    }
  emsp(k, nvd, an, am, as, dxa);
  if (0.0 < p->alpha_rtpp)
    for (int v = 0; v < nvd; ++v)
      for (int j = 0; j < k; ++j)
        an[(int64_t)v * k + j] = am[v] + (real)p->alpha_rtpp * dxf[(int64_t)v * k + j] +
                                 (real)(1.0 - p->alpha_rtpp) * dxa[(int64_t)v * k + j];
  if (0.0 < p->alpha_rtps)
    for (int v = 0; v < nvd; ++v) {
      real f = (as[v] == 0) ? (real)0 : (real)p->alpha_rtps * fs[v] / as[v] + (real)(1.0 - p->alpha_rtps);
      for (int j = 0; j < k; ++j) an[(int64_t)v * k + j] = am[v] + dxa[(int64_t)v * k + j] * f;
    }
}

/*
 * Analysis of the points listed in pts (p = k*nij1 + i), or of all P points
 * when npts < 0.  State arrays use the reference layouts (sbletkf.h) in r_size;
 * anal arrays receive only the listed points.  The observations must already
 * be in cell order with cellstart[] (the reference's set_obs happens before
 * its ANALYSIS timer).  uniforms/src as in sbletkf_analysis.  nobsl_out [P]
 * optional.  Returns OR-ed status bits.
 */
int SUFFIX(ref_da_main)(const sbletkf_params *p, int nij1, const double *lon1, const double *lat1,
                        const double *ri1, const double *rj1, const double *dlon1, const double *dlat1,
                        const double *phi1, const double *depth1, int nobs, const int64_t *cellstart,
                        const int32_t *elm, const real *olon, const real *olat, const real *olev,
                        const real *oerr, const real *odep, const real *ohdxf, const real *fcst3d,
                        const real *fcst2d, real *anal3d, real *anal2d, const double *uniforms, int32_t *src_out,
                        int32_t *nobsl_out, int npts, const int64_t *pts, int nthreads) {
  const int k = p->nmem, nlev = p->nlev, nv3d = p->nv3d, nv2d = p->nv2d;
  const int64_t P = (int64_t)nlev * nij1;
  if (nobs == 0) { /* common_da.f90:57-61 */
    memcpy(anal3d, fcst3d, sizeof(real) * (size_t)nv3d * k * P);
    memcpy(anal2d, fcst2d, sizeof(real) * (size_t)nv2d * k * nij1);
    return 0;
  }
  ctx_t c = {p, nij1, lon1, lat1, ri1, rj1, dlon1, dlat1, phi1, depth1, nobs, cellstart, elm,
             olon, olat, olev, oerr, odep, ohdxf};
  int64_t n_iter = npts < 0 ? P : npts;
  int status = 0;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
#pragma omp parallel reduction(| : status)
  {
    int *use = (int *)malloc(sizeof(int) * (size_t)nobs);
    int cap = 0;
    real *lh = NULL, *lr = NULL, *ll = NULL, *ld = NULL;
    core_buf_t b;
    memset(&b, 0, sizeof(b));
    size_t kk2 = (size_t)k * k;
    b.work1 = (real *)malloc(sizeof(real) * kk2);
    b.work3 = (real *)malloc(sizeof(real) * kk2);
    b.wmat = (real *)malloc(sizeof(real) * kk2);
    b.wgm = (real *)malloc(sizeof(real) * kk2);
    b.wtmp = (real *)malloc(sizeof(real) * kk2);
    b.wvec = (real *)malloc(sizeof(real) * k);
    b.evec = (double *)malloc(sizeof(double) * kk2);
    b.eval = (double *)malloc(sizeof(double) * k);
    b.dwork = (double *)malloc(sizeof(double) * (4 * k));
    b.wgt = (double *)malloc(sizeof(double) * k);
    b.cwgt = (double *)malloc(sizeof(double) * k);
    b.rand = (double *)malloc(sizeof(double) * k);
    b.inum = (int *)malloc(sizeof(int) * k);
    b.used = (int *)malloc(sizeof(int) * 2 * k);
    real *x = (real *)malloc(sizeof(real) * (size_t)k * 8), *an = (real *)malloc(sizeof(real) * (size_t)k * 8);
    real *tmp = (real *)malloc(sizeof(real) * ((size_t)k * 16 + 64));
    real *wlpf = (real *)malloc(sizeof(real) * kk2);
#pragma omp for schedule(dynamic)
    for (int64_t it = 0; it < n_iter; ++it) {
      int64_t pid = npts < 0 ? it : pts[it];
      int kl = (int)(pid / nij1), i = (int)(pid % nij1);
      real rdep = (real)depth1[pid];
      int nobsl = count_nobsl(&c, i, kl, rdep, use);
      if (nobsl_out) nobsl_out[pid] = nobsl;
      int st = 0;
      if (nobsl == 0) {
        if (p->iswitch_da == SBLETKF_DA_LETKF) noobs(p, &b, sqrt(p->cov_infl_mul));
        else noobs(p, &b, 1.0);
      } else {
        if (nobsl > cap) {
          cap = nobsl;
          lh = (real *)realloc(lh, sizeof(real) * (size_t)cap * k);
          lr = (real *)realloc(lr, sizeof(real) * (size_t)cap);
          ll = (real *)realloc(ll, sizeof(real) * (size_t)cap);
          ld = (real *)realloc(ld, sizeof(real) * (size_t)cap);
          b.rlinv = (real *)realloc(b.rlinv, sizeof(real) * (size_t)cap * k);
          b.work2 = (real *)realloc(b.work2, sizeof(real) * (size_t)cap * k);
        }
        obs_local(&c, i, kl, nobsl, rdep, use, lh, lr, ll, ld);
        if (p->iswitch_da == SBLETKF_DA_LETKF) {
          st = letkf_core(p, nobsl, lh, lr, ll, ld, &b);
        } else {
          const double *u = uniforms + (p->rm == SBLETKF_RM_SR ? pid * p->nmonte : pid * p->nmonte * k);
          int32_t *so = src_out ? src_out + pid * p->nmonte * k : NULL;
          memset(b.wvec, 0, sizeof(real) * k);
          if (p->iswitch_da == SBLETKF_DA_LPF) {
            lpf_core(p, nobsl, lh, lr, ll, ld, u, so, b.wmat, &b);
          } else {
            lpf_core(p, nobsl, lh, lr, ll, ld, u, so, wlpf, &b);
            st = gm_core(p, nobsl, lh, lr, ll, ld, b.wtmp, &b);
            if (!st) gemm('n', 'n', k, k, k, b.wtmp, k, wlpf, k, b.wmat, k);
          }
        }
      }
      status |= st;
      /* 3D update */
      for (int v = 0; v < nv3d; ++v)
        for (int m = 0; m < k; ++m) x[(int64_t)v * k + m] = fcst3d[(((int64_t)v * k + m) * nlev + kl) * nij1 + i];
      update_block(p, nv3d, x, b.wvec, b.wmat, an, tmp);
      for (int v = 0; v < nv3d; ++v)
        for (int m = 0; m < k; ++m) anal3d[(((int64_t)v * k + m) * nlev + kl) * nij1 + i] = an[(int64_t)v * k + m];
      if (kl == nlev - 1 && nv2d > 0) {
        for (int v = 0; v < nv2d; ++v)
          for (int m = 0; m < k; ++m) x[(int64_t)v * k + m] = fcst2d[((int64_t)v * k + m) * nij1 + i];
        update_block(p, nv2d, x, b.wvec, b.wmat, an, tmp);
        for (int v = 0; v < nv2d; ++v)
          for (int m = 0; m < k; ++m) anal2d[((int64_t)v * k + m) * nij1 + i] = an[(int64_t)v * k + m];
      }
      /* round_off (common_da.f90:506-533), applied per point after its update */
      if (p->roff && kl >= 1 && phi1[i] != 1.0) {
        for (int m = 0; m < k; ++m) {
          real *t = &anal3d[(((int64_t)p->iv3d_t * k + m) * nlev + kl) * nij1 + i];
          real *s = &anal3d[(((int64_t)p->iv3d_s * k + m) * nlev + kl) * nij1 + i];
          if (*t < (real)p->tmin) *t = (real)p->tmin;
          if (*t > (real)p->tmax) *t = (real)p->tmax;
          if (*s < (real)p->smin) *s = (real)p->smin;
          if (*s > (real)p->smax) *s = (real)p->smax;
        }
      }
    }
    free(use); free(lh); free(lr); free(ll); free(ld);
    free(b.rlinv); free(b.work1); free(b.work2); free(b.work3); free(b.wmat); free(b.wgm); free(b.wtmp);
    free(b.wvec); free(b.evec); free(b.eval); free(b.dwork); free(b.wgt); free(b.cwgt); free(b.rand);
    free(b.inum); free(b.used); free(x); free(an); free(tmp); free(wlpf);
  }
  return status;
}
