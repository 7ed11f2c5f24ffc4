/*
 * cansfz.h -- C ABI of the B200-native CaNS-Fizzy per-time-step hot path.
 *
 * One GPU, one 1x1 pencil.  All fields use the reference's storage convention:
 * FP64, Fortran column-major (x fastest), one ghost layer, i.e. a field of the
 * interior size n = (nx,ny,nz) is an array a(0:nx+1,0:ny+1,0:nz+1) of
 * (nx+2)*(ny+2)*(nz+2) doubles.  Tendency arrays (the AB2 histories) are
 * interior-only, a(1:nx,1:ny,1:nz).  1-D z metrics (dzci, dzfi, ...) are
 * a(0:nz+1).
 *
 * Every entry point returns an int status (CANSFZ_OK == 0).  The reference
 * returns nothing and aborts with `error stop`; a Fortran shim maps a non-zero
 * status to the reference's abort message.
 *
 * Per-procedure entries take DEVICE pointers (what `!$acc host_data
 * use_device(...)` hands a bind(C) interface) and run on the context's stream.
 * Scalars are passed by value.  Hidden `save` state of the reference (AB2
 * histories, dlmin, first-call flags) lives in the context.
 */
#ifndef CANSFZ_H
#define CANSFZ_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define CANSFZ_OK               0
#define CANSFZ_ERR_ARG          1  /* bad size, pointer or parameter        */
#define CANSFZ_ERR_CUDA         2  /* a CUDA runtime call failed            */
#define CANSFZ_ERR_TIMEOUT      3  /* a bounded device wait ran out         */
#define CANSFZ_ERR_NAN          4  /* NaN in the divergence check           */
#define CANSFZ_ERR_DIVERGENCE   5  /* max divergence above `small`          */
#define CANSFZ_ERR_DT           6  /* dt_cfl < small, or dt_f above limit   */
#define CANSFZ_ERR_UNSUPPORTED  7  /* BC / option not built for the GPU     */
#define CANSFZ_ERR_NOMEM        8  /* device allocation failed              */
#define CANSFZ_ERR_NOT_FOUND    9  /* no CUDA device / extension missing    */

/* ---- runtime switches for the reference's compile-time macros ------------ */
enum { CANSFZ_ACDI = 0, CANSFZ_VOF_THINC = 1 };    /* _INTERFACE_CAPTURING_VOF */
enum { CANSFZ_FORM_FP64 = 0, CANSFZ_FORM_MIXED = 1 };

/*
 * Run parameters: the namelists &dns, &two_fluid and &scalar of input.nml
 * (src/param.f90:91-120) plus the derived quantities and the macros that the
 * reference fixes at compile time.  Character arrays keep Fortran order, e.g.
 * cbcvel(0:1,3,3) -> cbcvel[ivel][idir][ibound], so a bind(C) derived type
 * with the same members maps onto this struct member by member.
 */
typedef struct cansfz_params {
  /* &dns */
  int32_t ng[3];
  double  l[3];
  int32_t gtype;
  double  gr;
  double  cfl, dtmax, dt_f;
  int32_t is_solve_ns, is_track_interface;
  int32_t icheck;
  char    cbcvel[3][3][2];
  double  bcvel[3][3][2];
  char    cbcpre[3][2];
  double  bcpre[3][2];
  double  bforce[3], gacc[3];
  /* &two_fluid */
  char    cbcpsi[3][2];
  double  bcpsi[3][2];
  char    cbcnor[3][3][2];
  double  bcnor[3][3][2];
  double  sigma, rho12[2], mu12[2], beta12[2];
  double  psi_thickness_factor;
  double  acdi_gam_factor, acdi_gam_min;   /* not namelist inputs in the reference */
  /* compile-time macros of the reference (src/param.f90, configs/flags.mk) */
  int32_t interface_capturing;  /* CANSFZ_ACDI (default) or CANSFZ_VOF_THINC   */
  int32_t sdf_normals;          /* _SDF_NORMALS, default 1                     */
  int32_t brackbill;            /* _CAPILLARY_BRACKBILL_NORMALIZATION, default 1 */
  int32_t balanced;             /* _BALANCED_CAPILLARY_PRESSURE_SPLIT, default 0:
                                   the surf?_n/surf?_o histories live in the context
                                   (cansfz_get_aux "surfx_n" ... "surfz_o")      */
  /* scalar transport: _SCALAR and _BOUSSINESQ_BUOYANCY (compile-time macros
   * of the reference, default 0), &scalar, and ka12/cp12 of &two_fluid    */
  int32_t scalar;               /* transport the scalar s (rk_scal every step) */
  int32_t boussinesq;           /* buoyancy term in mom_xyz_oth (needs scalar) */
  char    cbcsca[3][2];
  double  bcsca[3][2];
  double  ssource;
  double  ka12[2], cp12[2];
  /* forms of this library (no reference counterpart) */
  int32_t form;                 /* CANSFZ_FORM_FP64 (drop-in) or CANSFZ_FORM_MIXED */
  int32_t refine_sweeps;        /* mixed form: FP64-residual refinement sweeps of the
                                   FP32 Poisson solve; -1: the Poisson solve in FP64 */
  int32_t fp32_transforms;      /* mixed form, FP32 solve: 0 = x/y line transforms as
                                   split-BF16 GEMMs on the tensor cores (tcgen05) where
                                   the line lengths are 64, 128 or 256, shared-memory FFTs
                                   otherwise; 1 = shared-memory FFTs always          */
  int32_t reserved[7];
} cansfz_params;

/* Per-step diagnostics, mirrored from the device (main.f90 prints). */
typedef struct cansfz_diag {
  double  time;
  int64_t istep;
  double  dt, dto, dt_cfl;
  double  gam, seps;
  double  divtot, divmax;     /* last chkdt/chkdiv evaluation (every icheck) */
  double  mass12[2];          /* phase masses, cmpt_mean_mass (output.f90:759) */
  int32_t status;             /* last abort reason, CANSFZ_OK when none      */
  int32_t reserved[7];
} cansfz_diag;

typedef struct cansfz_ctx cansfz_ctx;

/* ---- lifecycle ----------------------------------------------------------
 * cansfz_create: replaces the set-up part of program cans
 *   (src/main.f90:147-412): initmpi (1x1 pencil), initgrid, initsolver,
 *   acdi_set_epsilon, device allocation of every field and workspace.
 * `stream` is a cudaStream_t (NULL: the context creates its own).          */
int cansfz_create(const cansfz_params* prm, void* stream, cansfz_ctx** out);
int cansfz_destroy(cansfz_ctx* ctx);
const char* cansfz_status_string(int status);
int cansfz_version(void);

/* Field I/O in the reference halo layout.  `on_device` != 0: the pointers
 * are device pointers; otherwise host pointers (pinned or pageable).
 * Replaces `!$acc enter data copyin(u,v,w,p,psi)` + boundary fills and the
 * restart read `load_one('r',...)` (src/main.f90:321-356).               */
int cansfz_set_fields(cansfz_ctx* ctx, const double* u, const double* v,
                      const double* w, const double* p, const double* psi,
                      int on_device);
int cansfz_get_fields(cansfz_ctx* ctx, double* u, double* v, double* w,
                      double* p, double* psi, int on_device);
/* Read one auxiliary field (phi, kappa, normx, normy, normz, psiflx_x..z,
 * psio, pn, po; s with the scalar) by name into a halo-layout buffer.     */
int cansfz_get_aux(cansfz_ctx* ctx, const char* name, double* out, int on_device);
/* The scalar s (halo layout) of a case created with scalar = 1: the
 * `copyin(s)` and restart read of s (src/main.f90:316-318,327-329);
 * read it back with cansfz_get_aux(ctx, "s", ...).  CANSFZ_ERR_UNSUPPORTED
 * without the scalar.                                                     */
int cansfz_set_scalar(cansfz_ctx* ctx, const double* s, int on_device);

/* Initial conditions computed on the device into the context's fields (no
 * host field arrays; cansfz_prepare follows):
 * init2fl (src/two_fluid.f90:247-437): inipsi 'uni', 'zer', 'flm',
 *   'bub1/2/3', 'drp1/2/3', 'dis1/2/3'; spheres = nspheres rows (x, y, z, r)
 *   as read_sphere_file reads spheres.in (:439-471), NULL/0 for the
 *   reference's default sphere;
 * initflow (src/initflow.f90:16-361): inivel 'zer', 'uni', 'cou', 'poi'
 *   (with set_mean), 'voy', 'vox' (at the context's time);
 * initscal (src/initflow.f90:363-429): inisca 'zer', 'uni', 'cou', 'dhc'
 *   (CANSFZ_ERR_UNSUPPORTED without the scalar).
 * An unknown name returns CANSFZ_ERR_ARG, where the reference aborts.     */
int cansfz_init2fl(cansfz_ctx* ctx, const char* inipsi, const double* spheres, int nspheres);
int cansfz_initflow(cansfz_ctx* ctx, const char* inivel);
int cansfz_initscal(cansfz_ctx* ctx, const char* inisca);

/* Finish the start-up sequence after set_fields: BCs (the scalar's too),
 * phi, normals, curvature, Gamma and the first chkdt
 * (src/main.f90:337-412).                                                  */
int cansfz_prepare(cansfz_ctx* ctx);

/* Advance n time steps: the loop body of src/main.f90:422-562 (AB2 phase
 * update, the scalar's rk_scal when built with it, momentum, projection,
 * pressure update, Gamma every step,
 * chkdt/chkdiv every icheck).  Captured as a CUDA graph after the first
 * call.  Returns CANSFZ_ERR_DIVERGENCE / _NAN / _DT on the reference's abort
 * conditions, after finishing the step that triggered them.              */
int cansfz_step(cansfz_ctx* ctx, int nsteps);
int cansfz_get_diag(cansfz_ctx* ctx, cansfz_diag* d);
/* The per-step scalars of cansfz_get_diag (time, istep, dt, Gamma, status,
 * divergence of the last check) without the phase-mass reduction, which the
 * reference evaluates only on output steps: mass12 is set to NaN.        */
int cansfz_get_status(cansfz_ctx* ctx, cansfz_diag* d);
/* Device stream the context runs on (cudaStream_t). */
void* cansfz_stream(cansfz_ctx* ctx);

/* ---- per-procedure drop-in entries (device pointers) ---------------------
 * Argument order follows the reference.  n = interior sizes of the 1x1
 * pencil (must equal the context's).                                      */

/* rk_2fl (src/rk.f90:193-254): AB2 phase update + clip; keeps the
 * dpsidtrk/dpsidtrko histories in ctx.  ACDI or THINC per the context.   */
int cansfz_rk_2fl(cansfz_ctx* ctx, const double rkpar[2], double dt,
                  double gam, double seps, double beta,
                  const double* u, const double* v, const double* w,
                  const double* normx, const double* normy, const double* normz,
                  const double* phi, double* psi,
                  double* psiflx_x, double* psiflx_y, double* psiflx_z);

/* acdi_transport_pf (src/acdi.f90:64-225): dpsidt (interior) + face fluxes */
int cansfz_acdi_transport_pf(cansfz_ctx* ctx, double gam, double seps,
                             const double* u, const double* v, const double* w,
                             const double* normx, const double* normy,
                             const double* normz, const double* phi,
                             const double* psi, double* dpsidt,
                             double* flux_x, double* flux_y, double* flux_z);

/* vof_thinc_transport_psi (src/vof_thinc_qq.f90:39-133) */
int cansfz_vof_thinc_transport_psi(cansfz_ctx* ctx, double beta,
                                   const double* u, const double* v, const double* w,
                                   const double* normx, const double* normy,
                                   const double* normz, const double* phi,
                                   const double* psi, double* dpsidt,
                                   double* flux_x, double* flux_y, double* flux_z);

/* acdi_cmpt_phi (src/acdi.f90:227-248), vof_thinc_cmpt_phi
 * (src/vof_thinc_qq.f90:135-157): SDF proxy over the full halo array.     */
int cansfz_acdi_cmpt_phi(cansfz_ctx* ctx, double seps, const double* psi, double* phi);
int cansfz_vof_thinc_cmpt_phi(cansfz_ctx* ctx, double beta, const double* psi, double* phi);

/* acdi_set_gamma (src/acdi.f90:32-62): returns Gamma = sqrt(max|u_c|^2)*gam_factor */
int cansfz_acdi_set_gamma(cansfz_ctx* ctx, double gam_factor, const double* u,
                          const double* v, const double* w, double* gam);

/* cmpt_norm_curv_youngs (src/two_fluid.f90:60-175) */
int cansfz_cmpt_norm_curv_youngs(cansfz_ctx* ctx, const double* psi,
                                 double* normx, double* normy, double* normz,
                                 double* kappa);

/* clip_field (src/two_fluid.f90:35-58), full halo array */
int cansfz_clip_field(cansfz_ctx* ctx, double rmin, double rmax, double* p);

/* rk (src/rk.f90:16-131): momentum AB2 with the density ratio, then the
 * pressure-split, surface-tension, gravity, body-force and (boussinesq)
 * buoyancy terms.  Keeps the d?dtrk/d?dtrko histories in ctx.  s: the
 * scalar of the buoyancy term; NULL allowed without boussinesq.            */
int cansfz_rk(cansfz_ctx* ctx, const double rkpar[2], double dt, double dt_r,
              const double rho_av[3], const double* psi, const double* kappa,
              const double* p, const double* pn, const double* po, const double* s,
              const double* psio, const double* psiflx_x, const double* psiflx_y,
              const double* psiflx_z, double* u, double* v, double* w);

/* mom_xyz_ad (src/mom.f90:505-851) and mom_xyz_oth (src/mom.f90:853-1039):
 * interior-only tendencies.                                               */
int cansfz_mom_xyz_ad(cansfz_ctx* ctx, const double* psiflx_x, const double* psiflx_y,
                      const double* psiflx_z, const double* u, const double* v,
                      const double* w, const double* psi,
                      double* dudt, double* dvdt, double* dwdt);
int cansfz_mom_xyz_oth(cansfz_ctx* ctx, double dt_r, const double rho_av[3],
                       const double* p, const double* psi, const double* kappa,
                       const double* s, const double* pn, const double* po,
                       double* dudt, double* dvdt, double* dwdt);

/* scal_ad (src/scal.f90:13-66): dsdt (interior) of the scalar s advected
 * by rho*cp*u + (rho1*cp1 - rho2*cp2)*psiflx and diffused with the phase-
 * weighted ka12.  rk_scal (src/rk.f90:133-191): its AB2 update of s in
 * place (interior), keeping dsdtrk/dsdtrko in ctx.  Both need scalar = 1. */
int cansfz_scal_ad(cansfz_ctx* ctx, const double* psiflx_x, const double* psiflx_y,
                   const double* psiflx_z, const double* psi, const double* u,
                   const double* v, const double* w, const double* s, double* dsdt);
int cansfz_rk_scal(cansfz_ctx* ctx, const double rkpar[2], double dt, const double* psi,
                   const double* u, const double* v, const double* w, const double* psio,
                   const double* psiflx_x, const double* psiflx_y, const double* psiflx_z,
                   double* s);

/* fillps (src/fillps.f90:13-51): p = rho0*div(u)/dt on the interior */
int cansfz_fillps(cansfz_ctx* ctx, double dti, const double* u, const double* v,
                  const double* w, double* p);

/* updt_rhs_b (src/bound.f90:341-396) with the context's rhsb planes */
int cansfz_updt_rhs_b(cansfz_ctx* ctx, double* p);

/* solver_gpu (src/solver_gpu.f90:31-163): constant-coefficient Poisson
 * solve in place on the interior of p (halo layout), 1x1 pencil, in-HBM
 * transforms; plans, eigenvalues and tridiagonal coefficients come from
 * the context (initsolver, src/initsolver.f90:15-79).                      */
int cansfz_solver(cansfz_ctx* ctx, double* p);

/* correc (src/correc.f90:13-67), updatep (src/updatep.f90:13-24) */
int cansfz_correc(cansfz_ctx* ctx, double dt, const double* p,
                  double* u, double* v, double* w);
int cansfz_updatep(cansfz_ctx* ctx, const double* pp, double* p);

/* boundp / bounduvw (src/bound.f90:15-124) with the context's BCs.
 * which: 0 = cbcpre, 1 = cbcpsi, 2 = cbccur (kappa), 3..5 = cbcnor(:,:,1..3),
 * 6 = cbcsca (the scalar)                                                  */
int cansfz_boundp(cansfz_ctx* ctx, int which, double* p);
int cansfz_bounduvw(cansfz_ctx* ctx, int is_correc, double* u, double* v, double* w);

/* chkdt (src/chkdt.f90:15-94), chkdiv (src/chkdiv.f90:15-49),
 * bulk_mean_12_stag (src/utils.f90:68-136), cmpt_mean_mass
 * (src/output.f90:759-790)                                                */
int cansfz_chkdt(cansfz_ctx* ctx, const double* u, const double* v, const double* w,
                 double gam, double seps, double* dtmax);
int cansfz_chkdiv(cansfz_ctx* ctx, const double* u, const double* v, const double* w,
                  double* divtot, double* divmax);
int cansfz_bulk_mean_12_stag(cansfz_ctx* ctx, int idir, const double* psi, double* mean);
int cansfz_cmpt_mean_mass(cansfz_ctx* ctx, const double* psi, double mass12[2]);

/* ---- grid and solver set-up (host arrays) ------------------------------- */
/* initgrid (src/initgrid.f90:14-78): dzc,dzf,zc,zf of size nz+2 */
int cansfz_initgrid(int gtype, int nz, double gr, double lz,
                    double* dzc, double* dzf, double* zc, double* zf);
/* The context's z metrics (host copies, nz+2 each) */
int cansfz_get_grid(cansfz_ctx* ctx, double* dzc, double* dzf, double* zc,
                    double* zf, double* dzci, double* dzfi);

/* ---- library controls and measurement (no reference counterpart) -------- */
/* Time and step counter of the next step (restart: the [time, istep] pair
 * stored at the end of a checkpoint file, src/load.f90:94-134).            */
int cansfz_set_time(cansfz_ctx* ctx, double time, long long istep);
/* Prescribed velocity of is_solve_ns = .false. runs ('voy', 'vox', 'zer'
 * of initflow, src/initflow.f90:242-275), re-evaluated every step.         */
int cansfz_set_inivel(cansfz_ctx* ctx, const char* inivel);
/* Kernel launches per captured time step. */
int cansfz_kernels_per_step(cansfz_ctx* ctx, int* count);
/* Run nsteps steps outside the graph with CUDA events between the stages:
 * ms[i] = summed milliseconds of stage i, *nstages stages, names written
 * comma-separated into `names` (cap bytes).  Advances the state.          */
int cansfz_profile_stages(cansfz_ctx* ctx, int nsteps, double* ms, int maxstages,
                          int* nstages, char* names, int cap);

/* ---- mixed form (no reference counterpart) ------------------------------
 * FP32 spectral solve of the same discrete operator as cansfz_solver, then
 * `sweeps` refinement sweeps p += S32(rhs - L(p)) with the FP64 residual of
 * the 7-point Laplacian.  rhs and p: halo-layout device fields (p's ghost
 * layer is filled on return).  Homogeneous pressure BCs only.             */
int cansfz_solver_refined(cansfz_ctx* ctx, const double* rhs, double* p, int sweeps);
/* FP64 residual res = rhs - L(p) of that operator (p's ghosts are filled). */
int cansfz_poisson_residual(cansfz_ctx* ctx, const double* rhs, double* p, double* res);
/* The dense matrix F (row-major n x n, host array, out[j] = sum_k F[j*n+k]
 * in[k]) of one line transform of the FP32 solve's tensor-core path: kind 0
 * the packed real DFT (r0, r_{n/2}, r1, i1, ...) and its unnormalised
 * inverse, kind 1 DCT-II / DCT-III, kind 2 DST-II / DST-III (FFTW's REDFT10,
 * REDFT01, RODFT10, RODFT01); dir > 0 forward, dir < 0 backward.          */
int cansfz_xform_matrix(int kind, int dir, int n, double* F);

/* ---- launch plans and the autotuner (no reference counterpart) ----------
 * The launch shapes that suit a grid and a GPU, chosen by measurement.    */
typedef struct cansfz_plan {
  int32_t phase_slots;      /* blocks per SM that the z split of the ACDI/THINC
                               and Youngs tiles aims at (default 24)          */
  int32_t momentum_slots;   /* the same for the momentum tile (default 48)   */
  int32_t zsolve;           /* Poisson z solve of grids with >= 32768 columns:
                               0 the partitioned 32-column tiles where nz is
                               8 x (8, 12, 16, 24 or 32), 1 one column per
                               thread                                         */
  int32_t fp32_transforms;  /* mixed form's FP32 solve: 0 tensor-core GEMMs
                               where the line lengths allow, 1 FFTs           */
  double  ms_per_step;      /* step time measured with the plan by
                               cansfz_autotune (0: not measured)              */
  int32_t tile_tma;         /* momentum tile: 1 stages its FP64 planes with
                               TMA tensor copies (default; the mixed form's
                               FP32 planes are element copies beside them), 0
                               all planes with element-wise cp.async          */
  int32_t ghost_images;     /* periodic directions: 1 the kernels that produce
                               a field in the step also write its periodic
                               ghost images, so the ghost fills after them
                               skip those copies (default); 0 the fills copy
                               them.  The ghost values are the same bits     */
  int32_t line_transforms;  /* x and y transforms of the periodic kind with
                               64, 128 or 256 points: 0 two register passes
                               per line with one block barrier (default), 1
                               one warp per line (x lines of 128 or 256) or
                               the shared-memory Stockham FFT                */
  int32_t reserved[3];
} cansfz_plan;
int cansfz_get_plan(cansfz_ctx* ctx, cansfz_plan* plan);
/* Takes effect at the next step (the step graphs are captured again).    */
int cansfz_set_plan(cansfz_ctx* ctx, const cansfz_plan* plan);
/* Time candidate plans on a copy of the case (same parameters, the case's
 * current fields; the case itself does not advance) by a coordinate search
 * over the seven knobs, and apply the fastest.  cache_file (NULL: none): a
 * text file with one line per key (grid, form, refinement sweeps, options,
 * GPU name); a key found there is applied without timing, a new one is
 * appended.  report (NULL or cap bytes): a one-line account of the choice. */
int cansfz_autotune(cansfz_ctx* ctx, const char* cache_file, cansfz_plan* chosen, char* report, int cap);

/* ---- batched ensemble (no reference counterpart: the reference runs one
 * case per program) -----------------------------------------------------
 * Groups independent, prepared contexts (any grid sizes and parameters, all
 * at the same step parity, i.e. stepped the same number of times).  Each
 * step is one CUDA graph launch holding every case's whole step as a
 * parallel branch; the cases keep their own state and can be read back
 * with cansfz_get_fields / cansfz_get_diag.  stream: origin stream of the
 * graph launches (NULL: the ensemble creates one).  A case that aborts
 * stops the ensemble (later calls return its status), as the reference
 * program stops.                                                        */
typedef struct cansfz_ensemble cansfz_ensemble;
int cansfz_ensemble_create(cansfz_ctx* const* cases, int ncases, void* stream, cansfz_ensemble** out);
/* status_out: NULL or ncases entries, each case's status after the steps;
 * the return value is the first non-zero of them (CANSFZ_OK if none).   */
int cansfz_ensemble_step(cansfz_ensemble* ens, int nsteps, int* status_out);
int cansfz_ensemble_destroy(cansfz_ensemble* ens);
/* Batched launches (off by default, cases_per_launch = 1): cases of the same
 * grid and options (they differ only in physical parameters, initial fields
 * and time step) run as groups of up to cases_per_launch cases whose
 * kernels are one launch per kernel for the whole group, each case with its
 * own arguments; results are bit for bit those of the cases' own launches.
 * Takes effect at the next step (the step graphs are rebuilt).           */
int cansfz_ensemble_set_batching(cansfz_ensemble* ens, int cases_per_launch);
/* After a step: the number of groups (a case that shares its launches with
 * no other case is a group of one) and of cases in groups of two or more. */
int cansfz_ensemble_info(cansfz_ensemble* ens, int* ngroups, int* grouped_cases);

/* ---- allocation-free Poisson solve (no reference counterpart) ---------
 * solver_gpu for callers that may not allocate device memory while they
 * run: the spectral work buffer and the twiddle tables are static device
 * arrays of this library (16 MiB + 64 KiB on every GPU that loads it), so
 * no cudaMalloc or cudaFree runs.  Limits: nx*ny*nz <= 128^3 cells, nx and
 * ny even and <= 1024, nz <= 1536, x/y pressure BCs PP, NN or DD, z not
 * periodic; beyond them the call returns CANSFZ_ERR_ARG or
 * CANSFZ_ERR_UNSUPPORTED and launches nothing.  A CUDA error already
 * pending when the call starts is returned as CANSFZ_ERR_CUDA before any
 * launch, and left pending.  n: interior sizes; cbc: cbcpre(0:1,1:3); normfft,
 * lambdaxy (nx*ny, packed spectral order), a, b, c (nz): initsolver's
 * outputs as cansfz_solver uses them (device pointers); p: halo-layout
 * device field, right-hand side in, solution out (interior).  The first
 * call on a device (with that device current) does the set-up; make it
 * before any stream capture.  Calls share the static arrays, so calls
 * whose kernels overlap on the GPU race.                                 */
int cansfz_solver_static(const int n[3], const char cbc[3][2], double normfft, const double* lambdaxy,
                         const double* a, const double* b, const double* c, double* p, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CANSFZ_H */
