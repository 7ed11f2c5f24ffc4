// Internal definitions of libcansfz (sm_100a).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "../../include/cansfz.h"

#define CANSFZ_EPS 2.220446049250313e-16  // epsilon(1._rp), src/param.f90:18

#ifdef __CUDACC__
// 1/x correctly rounded: the value of the IEEE division 1./x (1.f/x), by the
// reciprocal intrinsic, which takes fewer instructions than a division
__device__ __forceinline__ double recip_rn(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float recip_rn(float x) { return __frcp_rn(x); }
#endif

namespace cansfz {

// ---------------------------------------------------------------------------
// geometry of one case on the device: the 1x1 pencil, halo strides, z metrics
// ---------------------------------------------------------------------------
struct Geo {
  int nx, ny, nz;     // interior sizes
  int sx, sxy;        // halo-layout strides: (i,j,k) -> i + sx*j + sxy*k
  double dxi, dyi;    // dli(1:2)
  double dx, dy;      // dl(1:2)
  const double* dzci; // (0:nz+1)
  const double* dzfi; // (0:nz+1)
  const double* dzc;  // (0:nz+1)
  const double* dzf;  // (0:nz+1)
  __host__ __device__ inline int h(int i, int j, int k) const { return i + sx * j + sxy * k; }
  __host__ __device__ inline int t(int i, int j, int k) const {
    return (i - 1) + nx * ((j - 1) + ny * (k - 1));
  }
  __host__ __device__ inline int hsize() const { return sxy * (nz + 2); }
  __host__ __device__ inline int tsize() const { return nx * ny * nz; }
};

// Periodic ghost images written by the kernel that produces a field.  A
// periodic ghost fill copies a(n) into a(0) and a(1) into a(n+1) along each
// periodic direction (src/bound.f90:126-293 for x, updthalo for y and z);
// the kernel that computes interior point (i,j,k) can store the same value
// into those images itself, edges and corners included (every combination
// of the directions in which the point is a first or last interior one).
// wrap: bit d set when direction d is periodic and the images along it are
// to be written (never for n = 1, where both images come from one point).
// The ghost fill that follows then skips those directions: the values match
// the reference's fill order, because its later stages (the non-periodic
// faces) read the same images.
#ifdef __CUDACC__
// the image offsets of (i,j,k) along x, y and z (0: none)
__device__ __forceinline__ int wrap_ox(const Geo& g, int wrap, int i) {
  return (wrap & 1) ? (i == 1 ? g.nx : (i == g.nx ? -g.nx : 0)) : 0;
}
__device__ __forceinline__ int wrap_oy(const Geo& g, int wrap, int j) {
  return (wrap & 2) ? (j == 1 ? g.ny * g.sx : (j == g.ny ? -g.ny * g.sx : 0)) : 0;
}
__device__ __forceinline__ int wrap_oz(const Geo& g, int wrap, int k) {
  return (wrap & 4) ? (k == 1 ? g.nz * g.sxy : (k == g.nz ? -g.nz * g.sxy : 0)) : 0;
}
// st(h) for every image c + (a combination of the non-zero offsets)
template <typename F>
__device__ __forceinline__ void store_images(int c, int ox, int oy, int oz, F st) {
  const int m = (ox != 0 ? 1 : 0) | (oy != 0 ? 2 : 0) | (oz != 0 ? 4 : 0);
  if (m == 0) return;
#pragma unroll 1
  for (int s = m; s != 0; s = (s - 1) & m)  // every non-empty combination of the image directions
    st(c + ((s & 1) ? ox : 0) + ((s & 2) ? oy : 0) + ((s & 4) ? oz : 0));
}
template <typename F>
__device__ __forceinline__ void store_wraps(const Geo& g, int wrap, int i, int j, int k, F st) {
  store_images(g.h(i, j, k), wrap_ox(g, wrap, i), wrap_oy(g, wrap, j), wrap_oz(g, wrap, k), st);
}
#endif

// ---------------------------------------------------------------------------
// per-step scalars kept on the device so a whole step is graph-capturable.
// Names follow program cans (src/main.f90:414-562).
// ---------------------------------------------------------------------------
struct DevScalars {
  double time, dt, dto, dt_r, dti;   // dti = dtrki = 1/dt
  double tm1, tm2;                   // tm_coeff = [1+dt_r/2, -dt_r/2]
  double f1, f2, f12;                // factor1, factor2, factor12 of rk/rk_2fl
  double gam, seps, beta;            // ACDI Gamma, epsilon; THINC beta
  double rho_av[3];                  // bulk_mean_12_stag results
  double dt_cfl, divtot, divmax;
  double mass12[2];
  long long istep;
  int status;                        // CANSFZ_OK or the abort reason
  int halted;                        // 1 after an abort: later steps do nothing
  int first_rk, first_rk2fl;         // is_first of rk and rk_2fl (save attribute)
  int first_scal;                    // is_first of rk_scal
  int check_now;                     // 1 on icheck steps
  // reduction slots
  unsigned long long max_bits[4];    // non-negative doubles as ordered bits
  double pad[4];
};

// ---------------------------------------------------------------------------
// run constants (set once)
// ---------------------------------------------------------------------------
struct Phys {
  double rho12[2], mu12[2];
  double rho0, irho0;          // rho0 = min(rho12) and its reciprocal
  double sigma, surf_factor;   // sigma or sigma*2/(rho1+rho2) (Brackbill)
  double bforce[3], gacc[3];
  double gam_factor, gam_min;
  double cfl, dtmax, dt_f;
  double dlmin;
  double small;
  int icheck;
  int brackbill;   // _CAPILLARY_BRACKBILL_NORMALIZATION
  int acdi;        // 1: ACDI, 0: THINC
  int sdf;         // _SDF_NORMALS
  int solve_ns, track;
  double mu_over_rho_max, rho_min, gmax;   // chkdt constants
  // scalar transport (_SCALAR) and the Boussinesq buoyancy
  int scalar, boussinesq;
  double ka12[2], rhocp12[2];   // rhocp12 = rho12*cp12 (src/rk.f90:166)
  double ssource;
  double ka_rhocp_max;          // maxval(ka12/(rho12*cp12)), the chkdt constant
  double rhobeta, drhobeta;     // rho2*beta2, rho1*beta1 - rho2*beta2
  int balanced;                 // _BALANCED_CAPILLARY_PRESSURE_SPLIT
};

// ---------------------------------------------------------------------------
// boundary fills (src/bound.f90).  One BcField describes one field: the face
// rules of set_bc in each direction, precomputed on the host exactly as
// set_bc derives factor and sgn.
// ---------------------------------------------------------------------------
enum BcType : int { BC_NONE = 0, BC_P = 1, BC_D = 2, BC_N = 3 };
struct BcFace {
  int type;        // BcType; BC_NONE: face not bounded (periodic halo) or skipped
  int centered;
  double factor;   // as computed by set_bc
  double sgn;
};
struct BcField {
  void* p;               // double*, or float* when f32 (intermediates of the mixed form)
  int f32;
  BcFace face[3][2];     // [idir][ibound]
  int halo_periodic[3];  // y/z periodic self-exchange (updthalo)
  int wrapped;           // directions (bit d) whose periodic images the producing kernel wrote (store_wraps)
};
#define BC_MAXF 6
struct BcGroup {
  int nf;
  BcField f[BC_MAXF];
};

// ---------------------------------------------------------------------------
// Poisson solver plan (initsolver + fftini), device side
// ---------------------------------------------------------------------------
#define FFT_MAXSTAGES 16
struct LinePlan {
  int n;          // real length
  int kind;       // 0: periodic (R2HC/HC2R packed), 1: NN (DCT-II/III), 2: DD (DST-II/III)
  int m;          // complex FFT length (n/2)
  int nst;        // number of radix stages
  int radix[FFT_MAXSTAGES];
  const double2* tw;    // exp(-2 pi i q / m), q = 0..m-1
  const double2* tw2;   // exp(-2 pi i k / n), k = 0..n/2 (real-transform post twiddle)
  const double2* twc;   // exp(-i pi k / (2n)), k = 0..n (DCT/DST twiddle)
  const float2* twf;    // the same three tables rounded to FP32 (mixed form)
  const float2* tw2f;
  const float2* twcf;
};

struct PoissonPlan {
  LinePlan px, py;
  const double* lam;     // eigenvalues in the packed spectral layout, nx*ny
  const double* a;       // tridiagonal coefficients (1:nz)
  const double* b;
  const double* c;
  double normfft;
  int zper;              // periodic z: Sherman-Morrison variant
  double* work;          // nx*ny*nz spectral buffer
  double* work2;         // second buffer (periodic z, DCT remaps)
  float* workf;          // FP32 spectral buffers of the mixed form
  float* work2f;
  int zsing;             // z operator singular (no Dirichlet wall): pin the (0,0) mode in FP32
  // elimination factors of the z systems, which do not change between
  // solves: 1/pivot and c/pivot per (column, level) in the spectral layout
  // (null: the solve evaluates them on the fly)
  double* zpiv;
  double* zdf;
  float* zpivf;
  float* zdff;
  // the FP32 solve's x and y transforms as tensor-core GEMMs (k_xform_gemm.cu):
  // split-BF16 matrices [0] forward, [1] backward; null: the FFT kernels
  const uint16_t* gx[2];
  const uint16_t* gy[2];
  // z solve of grids with many columns: 0 the partitioned tile solve where
  // it applies, 1 one column per thread (cansfz_plan.zsolve)
  int zmode;
  // x and y transforms of the periodic kind: 0 the two-pass register
  // kernels where the length allows, 1 the one-warp-per-line (x) and
  // shared-memory Stockham kernels (cansfz_plan.line_transforms)
  int lmode;
};

// ---------------------------------------------------------------------------
// kernel launchers (host functions), all on `st`
// ---------------------------------------------------------------------------
struct Recorder;  // batch.cuh
struct Launch {
  cudaStream_t st;
  int nsm;
  // 1 while an ensemble graph is captured: other cases fill the GPU, so
  // kernels favour fewer, larger blocks
  int batched;
  // set: launches are recorded for a batched replay instead of issued
  Recorder* rec = nullptr;
  // tunable launch shapes (cansfz_plan): blocks per SM that the z split of
  // the phase-field tiles (ACDI/THINC, Youngs) and of the momentum tile aim at
  int phase_slots = 24;
  int mom_slots = 48;
  // 1: the momentum tile stages its FP64 planes by TMA (tensor maps built
  // per launch), 0: by element-wise cp.async (cansfz_plan.tma)
  int tma = 1;
  // periodic images that the producing kernels of the whole step write
  // (store_wraps); 0 for the per-procedure entries
  int wrap = 0;
};

// the surface-tension histories surf?_n, surf?_o of the balanced capillary
// split (_BALANCED_CAPILLARY_PRESSURE_SPLIT, src/mom.f90:982-1032), interior
// layout: a kernel reads n and o, writes the new force into out_n and, where
// out_o is set, n into out_o (out_n = n, out_o = o: the reference's in-place
// update; out_n = o and no out_o: the new force into the old slot, the
// parity flip of the step then swaps the roles)
struct SurfSplit {
  const double* n[3];
  const double* o[3];
  double* out_n[3];
  double* out_o[3];
};

// init2fl's choices (src/two_fluid.f90:275-305) for the device kernel
struct Init2fl {
  int zer, flm, sphere, swap;
  int idir[3], iperiod[3];
  double l[3], lmax, seps, reach;
  int nsph;
};

// optional stage marker of the step profiler (CUDA events between stages)
struct StageMark {
  void (*fn)(void* arg, const char* name);
  void* arg;
  void mark(const char* name) const { fn(arg, name); }
};

// k_stencil.cu
void launch_acdi_transport(const Launch& L, const Geo& g, const DevScalars* sc, bool sdf,
                           const double* u, const double* v, const double* w,
                           const double* nx, const double* ny, const double* nz,
                           const double* phi, const double* psi, double* dpsidt,
                           double* fx, double* fy, double* fz);
void launch_thinc_transport(const Launch& L, const Geo& g, const DevScalars* sc, bool sdf,
                            const double* u, const double* v, const double* w,
                            const double* nx, const double* ny, const double* nz,
                            const double* phi, const double* psi, double* dpsidt,
                            double* fx, double* fy, double* fz);
void launch_acdi_step(const Launch& L, const Geo& g, const DevScalars* sc, bool sdf,
                      const double* u, const double* v, const double* w, const double* nx,
                      const double* ny, const double* nz, const double* phi, const double* psi,
                      double* psi_out, double* hist, double* fx, double* fy, double* fz);
void launch_thinc_step(const Launch& L, const Geo& g, const DevScalars* sc, bool sdf,
                       const double* u, const double* v, const double* w, const double* nx,
                       const double* ny, const double* nz, const double* phi, const double* psi,
                       double* psi_out, double* hist, double* fx, double* fy, double* fz);
void launch_psi_update(const Launch& L, const Geo& g, const DevScalars* sc,
                       const double* psi_in, double* psi_out, double* dpsidt, double* dpsidto);
void launch_cmpt_phi(const Launch& L, const Geo& g, const DevScalars* sc, bool acdi,
                     const double* psi, double* phi);
void launch_youngs(const Launch& L, const Geo& g, const DevScalars* sc, const double* psi,
                   double* nx, double* ny, double* nz, double* kappa);
void launch_clip(const Launch& L, const Geo& g, double rmin, double rmax, double* p);
void launch_mom_ad(const Launch& L, const Geo& g, const Phys& ph, const double* fx,
                   const double* fy, const double* fz, const double* u, const double* v,
                   const double* w, const double* psi, double* du, double* dv, double* dw);
void launch_mom_oth(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc,
                    const double* p, const double* psi, const double* kappa, const double* s,
                    const SurfSplit* sp, const double* pn, const double* po, double* du, double* dv, double* dw);
void launch_rk_update1(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc,
                       const double* psio, const double* psi, const double* du,
                       const double* dv, const double* dw, double* duo, double* dvo,
                       double* dwo, double* u, double* v, double* w);
void launch_rk_update2(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc,
                       const double* psi, const double* du, const double* dv,
                       const double* dw, double* u, double* v, double* w);
void launch_momentum_fused(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc,
                           const double* u, const double* v, const double* w,
                           const double* psi, const double* psio, const double* fx,
                           const double* fy, const double* fz, const double* p,
                           const double* po, const double* kappa, const double* s, const SurfSplit* sp,
                           double* duo, double* dvo, double* dwo, double* uo, double* vo, double* wo);
// scalar transport: scal_ad (src/scal.f90:13-66), and scal_ad with the AB2
// update of rk_scal (src/rk.f90:133-191) in one pass (s_out interior; the
// new dsdt into `hist`, the dsdtrko slot)
template <typename TI>
void launch_scal_ad(const Launch& L, const Geo& g, const Phys& ph, const TI* fx, const TI* fy, const TI* fz,
                    const double* psi, const double* u, const double* v, const double* w, const double* s,
                    double* dsdt);
template <typename TI>
void launch_scal_step(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const TI* fx,
                      const TI* fy, const TI* fz, const double* psi, const double* psio, const double* u,
                      const double* v, const double* w, const double* s, double* hist, double* s_out);
void launch_scal_update(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* psi,
                        const double* psio, const double* dsdt, double* hist, double* s);
void launch_fillps(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc,
                   const double* u, const double* v, const double* w, double* p);
void launch_correc(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc,
                   const double* p, double* u, double* v, double* w);
void launch_correc_updatep(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* p,
                           double* u, double* v, double* w, const double* pp, double* pout);
void launch_updatep_interior(const Launch& L, const Geo& g, const DevScalars* sc,
                             const double* phi, const double* pp, double* pout);
void launch_updatep_full(const Launch& L, const Geo& g, const double* pp, double* p);
void launch_copy(const Launch& L, size_t n, const double* src, double* dst);
void launch_fill(const Launch& L, size_t n, double val, double* dst);
void launch_fill(const Launch& L, size_t n, float val, float* dst);
void launch_widen(const Launch& L, size_t n, const float* src, double* dst);
void launch_cmpt_phi_f32(const Launch& L, const Geo& g, const DevScalars* sc, bool acdi, const double* psi,
                         float* phi, bool narrow_only);
template <typename TI>
void launch_thinc_step_t(const Launch& L, const Geo& g, const DevScalars* sc, bool sdf, const double* u,
                         const double* v, const double* w, const TI* nx, const TI* ny, const TI* nz, const TI* phi,
                         const double* psi, double* psi_out, TI* hist, TI* fx, TI* fy, TI* fz);

// reductions: results land in DevScalars
void launch_gamma(const Launch& L, const Geo& g, const Phys& ph, DevScalars* sc, double* partial,
                  const double* u, const double* v, const double* w, bool apply_floor);
void launch_chkdt(const Launch& L, const Geo& g, const Phys& ph, DevScalars* sc, double* partial,
                  const double* u, const double* v, const double* w, bool only_on_check);
void launch_step_reductions(const Launch& L, const Geo& g, const Phys& ph, DevScalars* sc, double* partial,
                            const double* u, const double* v, const double* w);
void launch_chkdiv(const Launch& L, const Geo& g, DevScalars* sc, double* partial,
                   const double* u, const double* v, const double* w, bool only_on_check);
void launch_bulk_mean(const Launch& L, const Geo& g, const Phys& ph, DevScalars* sc,
                      double* partial, int idir, const double* gvr, const double* psi);
void launch_mass(const Launch& L, const Geo& g, const Phys& ph, DevScalars* sc, double* partial,
                 const double* psi, double vol);

// k_init.cu: initial conditions on the device
void launch_init2fl(const Launch& L, const Geo& g, const Init2fl& a, const double* sph, const double* zc,
                    double* psi);
void launch_fill_zprofile(const Launch& L, const Geo& g, const double* prof, double* f);
void launch_fill_xprofile(const Launch& L, const Geo& g, double b0, double b1, double lx, double* f);

// step bookkeeping kernels
void launch_step_begin(const Launch& L, DevScalars* sc, int icheck);
void launch_step_end(const Launch& L, const Phys& ph, DevScalars* sc);

// k_bc.cu
void launch_bc_group(const Launch& L, const Geo& g, const BcGroup& grp, const DevScalars* sc);
void launch_updt_rhs_b(const Launch& L, const Geo& g, const int is_bound[3][2],
                       const double* rhsbx, const double* rhsby, const double* rhsbz,
                       double* p);

// k_poisson.cu
void poisson_set_attributes();
// tensor-core line transforms of the FP32 solve (k_xform_gemm.cu)
double xform_coef(int kind, int dir, int n, int j, int k);
std::vector<uint16_t> xform_bmat(int kind, int dir, int n);
bool xform_gemm_length(int n);
bool z_part_ok(const Geo& g, const PoissonPlan& pl);
// the x or y transforms have a two-pass register kernel (periodic kind, 64-256 points)
bool poisson_y2_applies(const PoissonPlan& pl);
int xform_gemm_set_attributes();
void launch_xform_gemm(const Launch& L, const Geo& g, int mode, bool add, const uint16_t* bmat, int n,
                       const void* src, void* dst, double normfft, DevScalars* sc);
// the z systems' elimination factors of `pl` (FP64, or FP32 for the mixed
// form) into piv/df, evaluated exactly as the solve's forward sweep does
void launch_z_factors(const Launch& L, const Geo& g, const PoissonPlan& pl, bool f32, void* piv, void* df);

// z-marching tile kernels (k_tiles.cu), TI = double (drop-in) or float (mixed form)
template <typename TI>
void launch_youngs_t(const Launch& L, const Geo& g, const DevScalars* sc, const TI* phi, TI* nx, TI* ny, TI* nz,
                     TI* kappa);
template <typename TI>
void launch_acdi_t(const Launch& L, const Geo& g, const DevScalars* sc, bool sdf, bool upd, const double* u,
                   const double* v, const double* w, const TI* nx, const TI* ny, const TI* nz, const TI* phi,
                   const double* psi, double* psi_out, TI* hist, TI* fx, TI* fy, TI* fz);
template <typename TI>
void launch_momentum_t(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* u,
                       const double* v, const double* w, const double* psi, const double* psio, const TI* fx,
                       const TI* fy, const TI* fz, const double* p, const double* po, const TI* kappa,
                       const double* s, const SurfSplit* sp, TI* duo, TI* dvo, TI* dwo, double* uo, double* vo,
                       double* wo);
void tiles_set_attributes();
void momentum_set_attributes();
void launch_poisson(const Launch& L, const Geo& g, const PoissonPlan& pl, const DevScalars* sc,
                    double* p, const StageMark* mk = nullptr);
// mixed form: FP32 spectral solve (dst = S(src) or dst += S(src)) and the
// FP64 residual res = rhs - L(phi) of the refinement
void launch_poisson_f32(const Launch& L, const Geo& g, const PoissonPlan& pl, const DevScalars* sc,
                        const double* src, double* dst, bool add, const StageMark* mk = nullptr);
void launch_residual(const Launch& L, const Geo& g, const DevScalars* sc, const double* rhs,
                     const double* phi, double* res);
void launch_poisson_fused_rhs(const Launch& L, const Geo& g, const PoissonPlan& pl,
                              const Phys& ph, const DevScalars* sc, const double* u,
                              const double* v, const double* w, const double* rhsb_planes,
                              double* phi, const StageMark* mk = nullptr);

}  // namespace cansfz
