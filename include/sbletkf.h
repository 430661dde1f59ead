/*
 * sbletkf.h -- C ABI of the B200 (sm_100a) sbPOM-LETKF analysis step.
 *
 * This library replaces the analysis step of sbPOM-LETKF v2: the per-grid-point
 * local ensemble transform (LETKF) and the local particle filter (LPF / LPFGM).
 * Every entry point takes plain pointers and sizes, returns an int status and
 * never synchronises the stream unless its comment says so.  All array
 * arguments are DEVICE pointers unless marked "host".
 *
 * Array layouts follow the reference's Fortran column-major arrays, written
 * here as C index order [slowest]...[fastest]:
 *   fcst3d(nij1,nlev,nmem,nv3d)  ->  [nv3d][nmem][nlev][nij1]
 *   fcst2d(nij1,nmem,nv2d)       ->  [nv2d][nmem][nij1]
 *   depth1(nij1,nlev)            ->  [nlev][nij1]
 *   obshdxf(nobs,nmem)           ->  [nmem][nobs]
 * Grid point p of the analysis loop (common_da.f90:67-68, DO k / DO i) is
 * p = (k-1)*nij1 + (i-1).
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   da_main(fcst3d,fcst2d,anal3d,anal2d)      letkf/run/src/common_da.f90:22
 *   letkf_core(nobsl,hdxf,rdiag,rloc,dep,..)  letkf/run/src/common_letkf.f90:61
 *   letkf_core_noobs(wvec,Wmat)               letkf/run/src/common_letkf.f90:37
 *   lpfgm_core(nobsl,hdxf,rdiag,rloc,dep,..)  letkf/run/src/common_lpfgm.f90:444
 *   lpfgm_core_noobs(wvec,Wmat)               letkf/run/src/common_lpfgm.f90:422
 *   obs sort / nobsgrd                        letkf/run/src/common_obs.f90:266-377
 *   compile-time PARAMETERs                   letkf/run/src/common_setting.f90:15-131
 */
#ifndef SBLETKF_H
#define SBLETKF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SBLETKF_ABI_VERSION 1

/* ---- status codes (bit flags; several may be OR-ed together) ---------- */
#define SBLETKF_OK              0
#define SBLETKF_ERR_ARG         1   /* bad pointer, shape or parameter          */
#define SBLETKF_ERR_CUDA        2   /* CUDA runtime error                       */
#define SBLETKF_ERR_WORKSPACE   4   /* call exceeds the workspace's capacity    */
#define SBLETKF_ERR_OBS_CELL    8   /* obs cell index outside [1,nlon-1]x[1,nlat-1] */
#define SBLETKF_ERR_EIG_NOCONV  16  /* Jacobi reached its sweep cap             */
#define SBLETKF_ERR_NONFINITE   32  /* NaN/Inf met in inputs or in the transform */
#define SBLETKF_ERR_EIG_NEG     64  /* all eigenvalues negative (common.f90:1031) */
#define SBLETKF_ERR_ROWS        128 /* local search box has too many grid rows  */
#define SBLETKF_ERR_UNSUPPORTED 256 /* option not supported by this entry point */
#define SBLETKF_ERR_TIMEOUT     512 /* a bounded device wait expired            */

/* ---- enumerations ----------------------------------------------------- */
#define SBLETKF_F32 0               /* dtype codes */
#define SBLETKF_F64 1

#define SBLETKF_PREC_FP64  0        /* every step in FP64 (plain path)          */
#define SBLETKF_PREC_MIXED 1        /* Gram on tcgen05 as a three-way BF16 split
                                       (h+m+l) with FP32 accumulation (points
                                       with > 12288 search-box candidates use
                                       FP64); eigensolve and transform FP64 */

#define SBLETKF_DA_LETKF 1          /* iswitch_da (common_setting.f90:65) */
#define SBLETKF_DA_LPF   2
#define SBLETKF_DA_LPFGM 3

#define SBLETKF_RM_SR 0             /* RM (common_setting.f90:82) */
#define SBLETKF_RM_MR 1

/* ---- run-time parameters (common_setting.f90 PARAMETERs) --------------- */
typedef struct sbletkf_params {
  int32_t nmem;        /* ensemble size k            (common_setting.f90:36)  */
  int32_t nlon, nlat;  /* global grid                 (:37-38)                */
  int32_t nlev;        /* sigma levels, k=nlev is the surface (:39)          */
  int32_t nv3d, nv2d;  /* number of 3D / 2D variables (:40-41)               */
  int32_t iv3d_t;      /* 0-based index of temperature among 3D vars (:44)   */
  int32_t iv3d_s;      /* 0-based index of salinity (:45)                    */
  int32_t iswitch_da;  /* SBLETKF_DA_*                (:65)                   */
  int32_t nmonte;      /* LPF resamplings averaged    (:79)                   */
  int32_t rm;          /* SBLETKF_RM_SR / _MR         (:82)                   */
  int32_t dp;          /* diagonal priority on/off    (:85)                   */
  int32_t sr_textbook; /* 0: reference SR offsets (common_lpfgm.f90:115-117),
                          1: textbook (u+i-1)/k                               */
  int32_t roff;        /* T/S round-off on/off        (:129)                  */
  int32_t id_z_obs;    /* SSH element id              (:59)                   */
  int32_t precision;   /* SBLETKF_PREC_*                                      */
  int32_t max_sweeps;  /* Jacobi sweep cap (status flag when reached)         */
  int32_t iv3d_u;      /* 0-based index of zonal velocity among 3D vars (:42) */
  int32_t iv3d_v;      /* 0-based index of meridional velocity (:43)         */
  int32_t iv2d_z;      /* 0-based index of SSH among 2D vars (:46)           */
  double cov_infl_mul; /* multiplicative inflation rho (:71)                  */
  double cov_infl_gm;  /* LPFGM inflation            (:89)                    */
  double alpha_rtpp;   /* (:74)                                               */
  double alpha_rtps;   /* (:75)                                               */
  double sigma_obs;    /* horizontal localization scale [m] (:94)             */
  double sigma_obsv;   /* vertical scale [m]; <=0 disables it (:95)           */
  double dist_zero;    /* horizontal cutoff [m]      (:97)                    */
  double dist_zerov;   /* vertical cutoff [m]        (:98)                    */
  double tmin, tmax;   /* T round-off bounds         (:130)                   */
  double smin, smax;   /* S round-off bounds         (:131)                   */
  double re;           /* earth radius [m]           (:28)                    */
  double pi;           /* (:27)                                               */
  double jacobi_tol;   /* smallest relative rotation the eigensolve applies;
                          <= 0: k * 2^-52 on the FP64 path, 1e-8 on the mixed
                          path (well under its Gram's ~1e-6 error)          */
  double tc_max_cand;  /* mixed path: points whose search box holds more candidates
                          use the FP64 Gram; <= 0: library default 12288   */
  double jacobi_stop;  /* the eigensolve ends after a sweep whose largest relative
                          rotation |b_p.b_q| / (|b_p||b_q|) was at most this;
                          <= 0: library default, 1e-10 on the FP64 path (1e-7
                          saves a sweep but leaves ~1e-8 relative error in the
                          analysis) and 1e-5 on the mixed path, whose Gram is
                          accurate to ~1e-6: the sweep that meets 1e-5 leaves
                          eigen-residuals of ~1e-10 (quadratic convergence) */
  double reserved_d[1];
} sbletkf_params;

/* Local grid of the points analysed (set_common_mpi_pom, common_pom.f90:125-219) */
typedef struct sbletkf_grid {
  int32_t nij1;                     /* horizontal points                      */
  int32_t reserved;
  const double *lon1, *lat1;        /* [nij1] degrees                         */
  const double *ri1, *rj1;          /* [nij1] 1-based grid indices            */
  const double *dlon1, *dlat1;      /* [nij1] grid spacing [m]                */
  const double *phi1;               /* [nij1] bottom depth h (1 on land)      */
  const double *depth1;             /* [nlev][nij1] depth [m], <=0            */
} sbletkf_grid;

/* Observations after H(x) (module globals of common_setting.f90:182-198)     */
typedef struct sbletkf_obs {
  int32_t nobs;
  int32_t hdxf_dtype;               /* SBLETKF_F32 or SBLETKF_F64             */
  const int32_t *elm;               /* [nobs] element id                      */
  const int32_t *idx, *idy;         /* [nobs] 1-based owning cell (obs_id_uniform) */
  const double *lon, *lat;          /* [nobs] degrees                         */
  const double *lev;                /* [nobs] depth [m], 0 at the surface     */
  const double *err;                /* [nobs] obs error std; rdiag = err^2    */
  const double *dep;                /* [nobs] innovation y - H(xf mean)       */
  const void *hdxf;                 /* [nmem][nobs] dYf = H(dXf)              */
} sbletkf_obs;

typedef struct sbletkf_workspace sbletkf_workspace;

/* Library ABI version and build information (host). */
int32_t sbletkf_abi_version(void);

/* Create a workspace on `device` for nij1 points and up to max_nobs
 * observations.  Allocates all device memory the other entry points use.
 * No reference counterpart (the reference uses module globals). */
int sbletkf_workspace_create(const sbletkf_params *p, int32_t nij1, int32_t max_nobs,
                             int32_t device, sbletkf_workspace **out);
int sbletkf_workspace_destroy(sbletkf_workspace *ws);

/* Bucket the observations by owning cell, row-major (idy, then idx, stable
 * within a cell), build the cumulative cell counts (nobsgrd) and the internal
 * sorted copies of the obs arrays.  Replaces common_obs.f90:266-377. */
int sbletkf_prepare_obs(sbletkf_workspace *ws, const sbletkf_params *p,
                        const sbletkf_obs *obs, void *stream);

/* The analysis step: da_main (common_da.f90:22-124) for every point of the
 * grid, LETKF / LPF / LPFGM by p->iswitch_da, followed by RTPP, RTPS and the
 * T/S round-off.  fcst3d/anal3d are [nv3d][nmem][nlev][nij1] and
 * fcst2d/anal2d [nv2d][nmem][nij1], of state_dtype.  uniforms: NULL for LETKF; for LPF/LPFGM
 * the resampling uniforms, [P][nmonte] (SR) or [P][nmonte][nmem] (MR).
 * resample_src: optional [P][nmonte][nmem] int32, the particle (0-based)
 * taken by each member in each draw.  point_status: optional [P] int32.
 * Asynchronous: errors are latched in the workspace (sbletkf_get_status). */
int sbletkf_analysis(sbletkf_workspace *ws, const sbletkf_params *p,
                     const sbletkf_grid *grid,
                     const void *fcst3d, const void *fcst2d,
                     void *anal3d, void *anal2d, int32_t state_dtype,
                     const double *uniforms, int32_t *resample_src,
                     int32_t *point_status, void *stream);

/* Per-point nobsl (count_nobsl, common_da.f90:133-205) for every point,
 * int32 [P].  Asynchronous. */
int sbletkf_count_nobsl(sbletkf_workspace *ws, const sbletkf_params *p,
                        const sbletkf_grid *grid, int32_t *nobsl, void *stream);

/* Synchronise `stream`, return and clear the latched device status. */
int sbletkf_get_status(sbletkf_workspace *ws, void *stream, int32_t *status);

/* OR `bits` into the workspace's latched device status, in stream order
 * (asynchronous).  Host-side failure injection: a test latches
 * SBLETKF_ERR_TIMEOUT before an analysis to drive the path every later launch
 * takes after a tensor-core wait has expired (no tensor memory allocated, no
 * UMMA issued, every point marked).  No reference counterpart. */
int sbletkf_latch_status(sbletkf_workspace *ws, int32_t bits, void *stream);

/* Ragged batch of per-point cores: letkf_core / letkf_core_noobs
 * (common_letkf.f90:37-210) or lpfgm_core / lpfgm_core_noobs
 * (common_lpfgm.f90:422-494) on npts independent local problems.
 * off[npts+1] (int64) are the row offsets of each point's local obs; point q's
 * hdxf is the Fortran array hdxf(nobsl,nmem) at hdxf + off[q]*nmem, i.e.
 * element (i,m) at off[q]*nmem + m*nobsl_q + i.  rdiag/rloc/dep are [off[npts]].
 * Outputs wvec [npts][nmem] and Wmat [npts][nmem][nmem], Wmat(i,j) of point q
 * at q*nmem*nmem + j*nmem + i.  uniforms/resample_src as in sbletkf_analysis
 * with P = npts.  Uses workspace-free device code; asynchronous. */
int sbletkf_core_batched(const sbletkf_params *p, int32_t npts, const int64_t *off,
                         const double *hdxf, const double *rdiag, const double *rloc,
                         const double *dep, double *wvec, double *wmat,
                         const double *uniforms, int32_t *resample_src,
                         int32_t *point_status, void *stream);

/* Allocation-free analysis for small problems.  No counterpart in the
 * reference.  For callers that cannot call cudaMalloc where they run the
 * analysis -- e.g. a host model whose memory pool already owns the device
 * (cudaMalloc would synchronise the device or fail) -- this entry point needs
 * no workspace: obs bucketing and sbletkf_analysis run with every scratch
 * buffer in one fixed device array of the library (about 13.4 MB, held by every
 * GPU that loads the library until exit).  It calls no allocating routine.
 * Limits: obs->nobs <= SBLETKF_NOALLOC_MAX_OBS, nlon*nlat <=
 * SBLETKF_NOALLOC_MAX_CELLS, nmem <= 128; larger calls return
 * SBLETKF_ERR_WORKSPACE before launching anything.  Runs on the current
 * device; the first call on a device (and in a new context, e.g. after
 * cudaDeviceReset) looks up the array's device address
 * (cudaGetSymbolAddress), so make it before any stream capture.  With CUDA's
 * lazy module loading (the default) that first call is also when the array
 * is allocated: make it before the caller's memory pool reserves the device,
 * or set CUDA_MODULE_LOADING=EAGER.  All calls share the array: calls that
 * overlap on the GPU race and must be serialised.  FP64 path only.
 * point_status ([P] int32) is required: every device-side error -- the
 * observation errors of sbletkf_prepare_obs (SBLETKF_ERR_OBS_CELL,
 * SBLETKF_ERR_NONFINITE), which belong to no point, OR-ed into every entry,
 * and each point's own analysis errors -- is reported there. */
#define SBLETKF_NOALLOC_MAX_OBS   8192
#define SBLETKF_NOALLOC_MAX_CELLS 65536
int sbletkf_analysis_noalloc(const sbletkf_params *p, const sbletkf_grid *grid, const sbletkf_obs *obs,
                             const void *fcst3d, const void *fcst2d, void *anal3d, void *anal2d,
                             int32_t state_dtype, const double *uniforms, int32_t *point_status,
                             void *stream);

/* ---- observation-space preprocessing (set_obs) --------------------------- */
/* Raw observations: what read_obs delivers (common_io.f90:1113-1210). */
typedef struct sbletkf_obs_in {
  int32_t nobs, reserved;
  const int32_t *elm;               /* element id (common_setting.f90:56-60)  */
  const double *lon, *lat;          /* degrees                                */
  const double *lev;                /* depth [m], <= 0 below the surface      */
  const double *dat;                /* observed value                         */
  const double *err;                /* prescribed error standard deviation    */
} sbletkf_obs_in;

/* Per-observation results; any pointer may be NULL (not written). */
typedef struct sbletkf_obs_out {
  int32_t *idx, *idy;               /* cell indices, 1-based, 0 outside       */
  int32_t *qc;                      /* 1 usable, 0 undef or rejected          */
  double *hxmean, *hxsprd;          /* ensemble mean / spread of H(x)         */
  double *dep;                      /* innovation dat - hxmean                */
  double *err;                      /* error std after AOEI                   */
  double *hdxf;                     /* [nmem][nobs] H(x_m) - hxmean           */
} sbletkf_obs_out;

#define SBLETKF_OBSOP_GROSS_QC 1    /* LGE_IO: gross-error check (only with AOEI off) */
#define SBLETKF_OBSOP_AOEI     2    /* adaptive observation error inflation   */

/* Observation operator and departures: set_obs (common_obs.f90:24-265,
 * 380-399) with Trans_XtoY (common.f90:391-500) and obs_id_uniform
 * (common.f90:112-168) for every member, on the device.  Grid arrays are
 * global, [nlat*nlon] with longitude fastest (lon, lat, fsm = sea mask,
 * 0 on land) and depth [nlev][nlat*nlon]; state3d [nv3d][nmem][nlev][nlat*nlon],
 * state2d [nv2d][nmem][nlat*nlon] (state_dtype).  Undef results are NaN.
 * stats (optional, [(nv3d+nv2d)*3], added to): count, sum dep, sum dep^2 of
 * the qc = 1 observations per variable (monit_dep, common.f90:602-675).
 * Needs nlev >= 6 (the Akima stencil). */
int sbletkf_obs_operator(const sbletkf_params *p, const double *glon, const double *glat, const double *gfsm,
                         const double *gdepth, const void *state3d, const void *state2d, int32_t state_dtype,
                         const sbletkf_obs_in *obs, int32_t flags, const sbletkf_obs_out *out, double *stats,
                         void *stream);

/* Observation-space monitors: monit_mean (common.f90:681-840) and
 * monit_sprd (:846-978), which write_ens_mpi applies to H(mean) and
 * H(spread) of the forecast and of the analysis (common_io.f90:1039-1045).
 * For every observation whose hx[o] is defined (not NaN, the reference's
 * undef) the value v = dat[o] - hx[o] (SBLETKF_MONIT_DEPARTURE; dat may be
 * NULL otherwise) or v = hx[o] (SBLETKF_MONIT_VALUE) is added to
 * stats[(ivd*3 + c)*3 + j]: ivd the variable of the element id (iv3d_u,
 * iv3d_v, iv3d_t, iv3d_s; SSH nv3d + iv2d_z), c = 0 all, 1 surface
 * (lev == 0), 2 interior (3D variables only), j = 0 count, 1 sum of v,
 * 2 sum of v^2.  stats ([(nv3d+nv2d)*9] FP64, device) is added to: zero it
 * first.  Bias = sum/count, RMSD = sqrt(sum of squares/count), spread =
 * sum/count.  Asynchronous. */
#define SBLETKF_MONIT_DEPARTURE 0
#define SBLETKF_MONIT_VALUE     1
int sbletkf_obs_monitor(const sbletkf_params *p, int32_t nobs, const int32_t *elm, const double *lev,
                        const double *dat, const double *hx, int32_t mode, double *stats, void *stream);

/* Ensemble mean and spread (k-1) of a state, per variable, level and point
 * (ensemble_mesp, common.f90:505-596): state3d [nv3d][nmem][nlev][nij1] ->
 * mean3d / sprd3d [nv3d][nlev][nij1], state2d [nv2d][nmem][nij1] -> mean2d /
 * sprd2d [nv2d][nij1], all in state_dtype; the spread pointers may be NULL.
 * Spread is NaN (the reference's undef) for nmem = 1. */
int sbletkf_ensemble_mean_spread(const sbletkf_params *p, int32_t nij1, const void *state3d, const void *state2d,
                                 int32_t state_dtype, void *mean3d, void *sprd3d, void *mean2d, void *sprd2d,
                                 void *stream);

/* Launch schedule of sbletkf_analysis for this workspace.
 * SBLETKF_SCHED_AUTO (the default): SBLETKF_SCHED_PIPELINE for the mixed
 * path with 65 <= nmem <= 112 (where a point's eigensolve outweighs the
 * producer's tensor-core Gram), SBLETKF_SCHED_COLUMNS for the other LETKF /
 * LPFGM cases (the FP64 Gram is faster in the 256-thread CTA),
 * SBLETKF_SCHED_POINT for the LPF.
 * SBLETKF_SCHED_COLUMNS: one persistent 256-thread CTA per SM takes items of
 * up to 8 grid columns, nlon apart (neighbours along a meridian), from an
 * atomic queue and walks their levels in snake order, starting every k x k
 * eigensolve from the eigenvectors of the previous one; items narrow to 1
 * column when the grid has fewer than 32 items of 8 per CTA.
 * SBLETKF_SCHED_PIPELINE (LETKF and LPFGM with nmem <= 112; otherwise the
 * column queue runs): the same walk by a warp-specialised 384-thread CTA per SM, whose 4 producer
 * warps select the local observations of the next point (and, mixed
 * precision, accumulate its Gram on the tensor cores) while its 8 consumer
 * warps run the eigensolve and update of the current one.  The workspace
 * then holds two local-obs lists of max_nobs entries per SM (12 bytes each).
 * SBLETKF_SCHED_POINT: one CTA per grid point (the LPF has no eigensolve to
 * warm-start).  All give the same analysis to rounding.
 * No reference counterpart (the reference's OpenMP DYNAMIC loop over (k,i),
 * common_da.f90:66-68, is the scheduling it replaces). */
#define SBLETKF_SCHED_AUTO     (-1)
#define SBLETKF_SCHED_POINT    0
#define SBLETKF_SCHED_COLUMNS  1
#define SBLETKF_SCHED_PIPELINE 2
int sbletkf_workspace_set_schedule(sbletkf_workspace *ws, int32_t schedule);

/* Columns per item of the column queue (SBLETKF_SCHED_COLUMNS and _PIPELINE):
 * 0 (the default) picks 8 when the grid gives at least 32 items of 8 per
 * CTA and narrower otherwise; 1..8 fixes it (the autotuner's knob).  Any
 * width gives the same analysis to rounding.  No reference counterpart. */
int sbletkf_workspace_set_item_width(sbletkf_workspace *ws, int32_t width);

/* Vector-Jacobian product of the LETKF analysis (iswitch_da = 1, with RTPP,
 * RTPS and the T/S round-off): given dJ/d anal3d and dJ/d anal2d (same layouts
 * as the state, state_dtype), accumulate dJ/d dep and dJ/d rdiag ([nobs],
 * caller's obs order, FP64, added to), dJ/d cov_infl_mul and dJ/d sigma_obs
 * (one FP64 each, added to); all four are device pointers.  dist_zero is held
 * fixed.  Recomputes each point's eigensolve in FP64 whatever p->precision
 * says.  nmem <= 112 (larger: SBLETKF_ERR_UNSUPPORTED).  Uses the
 * observations of the last sbletkf_prepare_obs.  No reference counterpart
 * (new capability). */
int sbletkf_backward(sbletkf_workspace *ws, const sbletkf_params *p,
                     const sbletkf_grid *grid,
                     const void *fcst3d, const void *fcst2d, int32_t state_dtype,
                     const void *grad_anal3d, const void *grad_anal2d,
                     double *grad_dep, double *grad_rdiag,
                     double *grad_infl, double *grad_sigma_obs, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* SBLETKF_H */
