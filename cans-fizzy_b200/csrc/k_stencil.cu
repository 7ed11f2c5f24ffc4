// Stencil, update and reduction kernels of the per-step hot path (FP64).
//
// Index convention: Fortran indices of the reference, interior 1..n, ghosts
// 0 and n+1, halo-layout strides from Geo.  Each kernel cites the reference
// loop it computes; expressions keep the reference's operation order.
#include <cfloat>

#include "batch.cuh"

namespace cansfz {

#define HALTED(sc) ((sc) != nullptr && (sc)->halted)

static inline dim3 blk_interior(const Geo& g) {
  int bx = g.nx >= 128 ? 128 : (g.nx >= 64 ? 64 : 32);
  return dim3(bx);
}
static inline dim3 grd_interior(const Geo& g, dim3 b) {
  return dim3((g.nx + b.x - 1) / b.x, g.ny, g.nz);
}
#define INTERIOR_IJK(g)                                   \
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1; \
  if (i > (g).nx) return;                                 \
  const int j = blockIdx.y + 1;                           \
  const int k = blockIdx.z + 1;
// the same for a kernel body run with block index bk (batch.cuh)
#define INTERIOR_IJK_B(g, bk)                             \
  const int i = (bk).x * blockDim.x + threadIdx.x + 1;    \
  if (i > (g).nx) return;                                 \
  const int j = (bk).y + 1;                               \
  const int k = (bk).z + 1;

__device__ __forceinline__ double sq(double x) { return x * x; }
#define LD(p, q) __ldg((p) + (q))

// ---------------------------------------------------------------------------
// acdi_transport_pf, src/acdi.f90:64-225: the z-marching tile kernel of
// k_tiles.cu (face fluxes computed once per face)
// ---------------------------------------------------------------------------
void launch_acdi_transport(const Launch& L, const Geo& g, const DevScalars* sc, bool sdf,
                           const double* u, const double* v, const double* w, const double* nx,
                           const double* ny, const double* nz, const double* phi, const double* psi,
                           double* dpsidt, double* fx, double* fy, double* fz) {
  launch_acdi_t<double>(L, g, sc, sdf, false, u, v, w, nx, ny, nz, phi, psi, nullptr, dpsidt, fx, fy, fz);
}

void launch_acdi_step(const Launch& L, const Geo& g, const DevScalars* sc, bool sdf, const double* u,
                      const double* v, const double* w, const double* nx, const double* ny, const double* nz,
                      const double* phi, const double* psi, double* psi_out, double* hist, double* fx, double* fy,
                      double* fz) {
  launch_acdi_t<double>(L, g, sc, sdf, true, u, v, w, nx, ny, nz, phi, psi, psi_out, hist, fx, fy, fz);
}

// ---------------------------------------------------------------------------
// vof_thinc_transport_psi, src/vof_thinc_qq.f90:39-133: fluxes over faces
// 0..n, then the flux divergence on the interior.
// ---------------------------------------------------------------------------
template <typename TI, bool SDF>
struct ThincFlux {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const DevScalars* __restrict__ sc,
      const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ w,
      const TI* __restrict__ nx_, const TI* __restrict__ ny_, const TI* __restrict__ nz_,
      const TI* __restrict__ phi, const double* __restrict__ psi, TI* __restrict__ fx, TI* __restrict__ fy,
      TI* __restrict__ fz) {
    typedef TI T;  // FP64 in the drop-in, FP32 in the mixed form
    if (HALTED(sc)) return;
    const int i = bk.x * blockDim.x + threadIdx.x;  // 0..n
    if (i > g.nx) return;
    const int j = bk.y, k = bk.z;
    const T beta = (T)sc->beta;
    const int c = g.h(i, j, k);
    const T vel_x = (T)LD(u, c), vel_y = (T)LD(v, c), vel_z = (T)LD(w, c);
    int ci, cj, ck;
    T xx, yy, zz;
    if (vel_x > T(0.)) { ci = c; xx = T(0.5); } else { ci = c + 1; xx = T(-0.5); }
    if (vel_y > T(0.)) { cj = c; yy = T(0.5); } else { cj = c + g.sx; yy = T(-0.5); }
    if (vel_z > T(0.)) { ck = c; zz = T(0.5); } else { ck = c + g.sxy; zz = T(-0.5); }
    const T lnormx_x = LD(nx_, ci), lnormy_y = LD(ny_, cj), lnormz_z = LD(nz_, ck);
    T d_x, d_y, d_z;
    if (SDF) {
      d_x = LD(phi, ci); d_y = LD(phi, cj); d_z = LD(phi, ck);
    } else {
      const T hb = T(-.5) / beta;
      d_x = hb * log(T(1.) / ((T)LD(psi, ci) + T(CANSFZ_EPS)) - T(1.) + T(CANSFZ_EPS));
      d_y = hb * log(T(1.) / ((T)LD(psi, cj) + T(CANSFZ_EPS)) - T(1.) + T(CANSFZ_EPS));
      d_z = hb * log(T(1.) / ((T)LD(psi, ck) + T(CANSFZ_EPS)) - T(1.) + T(CANSFZ_EPS));
    }
    const T m2b = T(-2.) * beta;
    fx[c] = vel_x * (T(1.) / (T(1.) + exp(m2b * (lnormx_x * xx + d_x))));
    fy[c] = vel_y * (T(1.) / (T(1.) + exp(m2b * (lnormy_y * yy + d_y))));
    fz[c] = vel_z * (T(1.) / (T(1.) + exp(m2b * (lnormz_z * zz + d_z))));
  }
};
template <typename TI, bool SDF>
__global__ void k_thinc_flux(Geo g, const DevScalars* __restrict__ sc,
    const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ w,
    const TI* __restrict__ nx_, const TI* __restrict__ ny_, const TI* __restrict__ nz_,
    const TI* __restrict__ phi, const double* __restrict__ psi,
    TI* __restrict__ fx, TI* __restrict__ fy, TI* __restrict__ fz) {
  ThincFlux<TI, SDF>::run(blk_here(), g, sc, u, v, w, nx_, ny_, nz_, phi, psi, fx, fy, fz);
}

__global__ void k_thinc_div(Geo g, const DevScalars* __restrict__ sc, const double* __restrict__ fx,
                            const double* __restrict__ fy, const double* __restrict__ fz,
                            double* __restrict__ dpsidt) {
  if (HALTED(sc)) return;
  INTERIOR_IJK(g)
  const int c = g.h(i, j, k);
  dpsidt[g.t(i, j, k)] = -(g.dxi * (LD(fx, c) - LD(fx, c - 1)) + g.dyi * (LD(fy, c) - LD(fy, c - g.sx)) +
                           g.dzfi[k] * (LD(fz, c) - LD(fz, c - g.sxy)));
}

// flux divergence + rk_2fl update (history in place), src/vof_thinc_qq.f90:122-132, src/rk.f90:240-248
template <typename TI>
struct ThincDivUpdate {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const DevScalars* __restrict__ sc,
      const TI* __restrict__ fx, const TI* __restrict__ fy, const TI* __restrict__ fz,
      const double* __restrict__ psi, TI* __restrict__ hist, double* __restrict__ psi_out) {
    typedef TI T;
    if (HALTED(sc)) return;
    INTERIOR_IJK_B(g, bk)
    const int c = g.h(i, j, k), t = g.t(i, j, k);
    const T d = -((T)g.dxi * (LD(fx, c) - LD(fx, c - 1)) + (T)g.dyi * (LD(fy, c) - LD(fy, c - g.sx)) +
                  (T)g.dzfi[k] * (LD(fz, c) - LD(fz, c - g.sxy)));
    const T dO = sc->first_rk2fl ? d : hist[t];
    psi_out[c] = fmin(fmax(0., LD(psi, c) + sc->f1 * (double)d + sc->f2 * (double)dO), 1.);
    hist[t] = d;
  }
};
template <typename TI>
__global__ void k_thinc_div_update(Geo g, const DevScalars* __restrict__ sc, const TI* __restrict__ fx,
                                   const TI* __restrict__ fy, const TI* __restrict__ fz,
                                   const double* __restrict__ psi, TI* __restrict__ hist,
                                   double* __restrict__ psi_out) {
  ThincDivUpdate<TI>::run(blk_here(), g, sc, fx, fy, fz, psi, hist, psi_out);
}

template <typename TI>
void launch_thinc_step_t(const Launch& L, const Geo& g, const DevScalars* sc, bool sdf, const double* u,
                         const double* v, const double* w, const TI* nx, const TI* ny, const TI* nz, const TI* phi,
                         const double* psi, double* psi_out, TI* hist, TI* fx, TI* fy, TI* fz) {
  dim3 b(g.nx + 1 >= 128 ? 128 : 64), gr((g.nx + 1 + b.x - 1) / b.x, g.ny + 1, g.nz + 1);
  if (sdf) kgo<ThincFlux<TI, true>, 128, 1>(L, k_thinc_flux<TI, true>, gr, b, 0, g, sc, u, v, w, nx, ny, nz, phi, psi,
      fx, fy, fz);
  else kgo<ThincFlux<TI, false>, 128, 1>(L, k_thinc_flux<TI, false>, gr, b, 0, g, sc, u, v, w, nx, ny, nz, phi, psi,
      fx, fy, fz);
  dim3 bi = blk_interior(g), gi = grd_interior(g, bi);
  kgo<ThincDivUpdate<TI>, 128, 1>(L, k_thinc_div_update<TI>, gi, bi, 0, g, sc, fx, fy, fz, psi, hist, psi_out);
}
template void launch_thinc_step_t<float>(const Launch&, const Geo&, const DevScalars*, bool, const double*,
                                         const double*, const double*, const float*, const float*, const float*,
                                         const float*, const double*, double*, float*, float*, float*, float*);

void launch_thinc_step(const Launch& L, const Geo& g, const DevScalars* sc, bool sdf, const double* u,
                       const double* v, const double* w, const double* nx, const double* ny, const double* nz,
                       const double* phi, const double* psi, double* psi_out, double* hist, double* fx, double* fy,
                       double* fz) {
  launch_thinc_step_t<double>(L, g, sc, sdf, u, v, w, nx, ny, nz, phi, psi, psi_out, hist, fx, fy, fz);
}

void launch_thinc_transport(const Launch& L, const Geo& g, const DevScalars* sc, bool sdf,
                            const double* u, const double* v, const double* w, const double* nx,
                            const double* ny, const double* nz, const double* phi, const double* psi,
                            double* dpsidt, double* fx, double* fy, double* fz) {
  dim3 b(g.nx + 1 >= 128 ? 128 : 64), gr((g.nx + 1 + b.x - 1) / b.x, g.ny + 1, g.nz + 1);
  if (sdf) kgo<ThincFlux<double, true>, 128, 1>(L, k_thinc_flux<double, true>, gr, b, 0, g, sc, u, v, w, nx, ny, nz,
      phi, psi, fx, fy, fz);
  else kgo<ThincFlux<double, false>, 128, 1>(L, k_thinc_flux<double, false>, gr, b, 0, g, sc, u, v, w, nx, ny, nz,
      phi, psi, fx, fy, fz);
  dim3 bi = blk_interior(g), gi = grd_interior(g, bi);
  k_thinc_div<<<gi, bi, 0, L.st>>>(g, sc, fx, fy, fz, dpsidt);
}

// ---------------------------------------------------------------------------
// rk_2fl update + clip, src/rk.f90:234-248 (the clip of the halo is dropped:
// every ghost cell is overwritten by boundp(psi) right after)
// ---------------------------------------------------------------------------
__global__ void k_psi_update(Geo g, const DevScalars* __restrict__ sc, const double* __restrict__ psi_in,
                             double* __restrict__ psi_out, const double* __restrict__ dn,
                             double* __restrict__ dold) {
  if (HALTED(sc)) return;
  INTERIOR_IJK(g)
  const int c = g.h(i, j, k), t = g.t(i, j, k);
  const double d = dn[t];
  const double dO = sc->first_rk2fl ? d : dold[t];
  const double val = LD(psi_in, c) + sc->f1 * d + sc->f2 * dO;
  psi_out[c] = fmin(fmax(0., val), 1.);
}

void launch_psi_update(const Launch& L, const Geo& g, const DevScalars* sc, const double* psi_in,
                       double* psi_out, double* dpsidt, double* dpsidto) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  k_psi_update<<<gr, b, 0, L.st>>>(g, sc, psi_in, psi_out, dpsidt, dpsidto);
}

// ---------------------------------------------------------------------------
// acdi_cmpt_phi (src/acdi.f90:227-248), vof_thinc_cmpt_phi
// (src/vof_thinc_qq.f90:135-157): whole halo array
// ---------------------------------------------------------------------------
constexpr int kPhiPer = 4;  // points per thread of k_cmpt_phi
template <bool ACDI, typename TO>
struct CmptPhi {
  static __device__ __forceinline__ void run(const Blk& bk, int n, const DevScalars* __restrict__ sc,
      const double* __restrict__ psi, TO* __restrict__ phi) {
    if (HALTED(sc)) return;
    // kPhiPer points per thread, a block's points contiguous: loads first
    const int q0 = bk.x * blockDim.x * kPhiPer + threadIdx.x;
    double ps[kPhiPer];
#pragma unroll
    for (int m = 0; m < kPhiPer; ++m) {
      const int q = q0 + m * blockDim.x;
      ps[m] = q < n ? LD(psi, q) : 0.;
    }
#pragma unroll
    for (int m = 0; m < kPhiPer; ++m) {
      const int q = q0 + m * blockDim.x;
      if (q >= n) break;
      if (ACDI) {
        phi[q] = (TO)(sc->seps * log((ps[m] + CANSFZ_EPS) / (1. - ps[m] + CANSFZ_EPS)));
      } else {
        const double pa = fmin(fmax(ps[m], CANSFZ_EPS), 1. - CANSFZ_EPS);
        phi[q] = (TO)(0.5 / sc->beta * log(pa / (1. - pa)));
      }
    }
  }
};
template <bool ACDI, typename TO>
__global__ void k_cmpt_phi(int n, const DevScalars* __restrict__ sc, const double* __restrict__ psi,
                           TO* __restrict__ phi) {
  CmptPhi<ACDI, TO>::run(blk_here(), n, sc, psi, phi);
}

void launch_cmpt_phi(const Launch& L, const Geo& g, const DevScalars* sc, bool acdi, const double* psi,
                     double* phi) {
  const int n = g.hsize();
  const int nb = (n + 256 * kPhiPer - 1) / (256 * kPhiPer);
  if (acdi) kgo<CmptPhi<true, double>, 256, 1>(L, k_cmpt_phi<true, double>, nb, 256, 0, n, sc, psi, phi);
  else kgo<CmptPhi<false, double>, 256, 1>(L, k_cmpt_phi<false, double>, nb, 256, 0, n, sc, psi, phi);
}
// the mixed form: phi evaluated in FP64 and stored in FP32
// (narrow_only: Youngs without SDF normals works on psi itself, stored in FP32)
struct Narrow {
  static __device__ __forceinline__ void run(const Blk& bk, int n, const DevScalars* __restrict__ sc,
      const double* __restrict__ src, float* __restrict__ dst) {
    if (HALTED(sc)) return;
    const int q = bk.x * blockDim.x + threadIdx.x;
    if (q < n) dst[q] = (float)src[q];
  }
};
__global__ void k_narrow(int n, const DevScalars* __restrict__ sc, const double* __restrict__ src,
                         float* __restrict__ dst) {
  Narrow::run(blk_here(), n, sc, src, dst);
}
void launch_cmpt_phi_f32(const Launch& L, const Geo& g, const DevScalars* sc, bool acdi, const double* psi,
                         float* phi, bool narrow_only) {
  const int n = g.hsize();
  if (narrow_only) kgo<Narrow, 256, 1>(L, k_narrow, (n + 255) / 256, 256, 0, n, sc, psi, phi);
  else if (acdi)
    kgo<CmptPhi<true, float>, 256, 1>(L, k_cmpt_phi<true, float>, (n + 256 * kPhiPer - 1) / (256 * kPhiPer), 256, 0,
                                      n, sc, psi, phi);
  else
    kgo<CmptPhi<false, float>, 256, 1>(L, k_cmpt_phi<false, float>, (n + 256 * kPhiPer - 1) / (256 * kPhiPer), 256,
                                       0, n, sc, psi, phi);
}

// ---------------------------------------------------------------------------
// cmpt_norm_curv_youngs, src/two_fluid.f90:60-175
// ---------------------------------------------------------------------------
void launch_youngs(const Launch& L, const Geo& g, const DevScalars* sc, const double* psi, double* nx, double* ny,
                   double* nz, double* kappa) {
  launch_youngs_t<double>(L, g, sc, psi, nx, ny, nz, kappa);
}

// clip_field, src/two_fluid.f90:35-58 (whole halo array)
__global__ void k_clip(int n, double rmin, double rmax, double* __restrict__ p) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) p[q] = fmin(fmax(rmin, p[q]), rmax);
}
void launch_clip(const Launch& L, const Geo& g, double rmin, double rmax, double* p) {
  const int n = g.hsize();
  k_clip<<<(n + 255) / 256, 256, 0, L.st>>>(n, rmin, rmax, p);
}

// ---------------------------------------------------------------------------
// momentum: mom_xyz_ad (src/mom.f90:505-851, default diffusion branch)
// ---------------------------------------------------------------------------
struct AdOut { double du, dv, dw; };

__device__ __forceinline__ AdOut mom_ad_cell(const Geo& g, const Phys& ph, int i, int j, int k,
                                             const double* __restrict__ psiflx_x,
                                             const double* __restrict__ psiflx_y,
                                             const double* __restrict__ psiflx_z,
                                             const double* __restrict__ u, const double* __restrict__ v,
                                             const double* __restrict__ w, const double* __restrict__ psi) {
  const double rho = ph.rho12[1], drho = ph.rho12[0] - ph.rho12[1];
  const double mu = ph.mu12[1], dmu = ph.mu12[0] - ph.mu12[1];
  const double dxi = g.dxi, dyi = g.dyi;
  const int c = g.h(i, j, k), sx = g.sx, sxy = g.sxy;
#define A_(f, a, b, cc) LD(f, c + (a) + (b) * sx + (cc) * sxy)
  const double u_ccm = A_(u, 0, 0, -1), u_cmc = A_(u, 0, -1, 0), u_mcc = A_(u, -1, 0, 0),
               u_ccc = A_(u, 0, 0, 0), u_pcc = A_(u, 1, 0, 0), u_mpc = A_(u, -1, 1, 0),
               u_cpc = A_(u, 0, 1, 0), u_mcp = A_(u, -1, 0, 1), u_ccp = A_(u, 0, 0, 1);
  const double v_ccm = A_(v, 0, 0, -1), v_cmc = A_(v, 0, -1, 0), v_pmc = A_(v, 1, -1, 0),
               v_mcc = A_(v, -1, 0, 0), v_ccc = A_(v, 0, 0, 0), v_pcc = A_(v, 1, 0, 0),
               v_cpc = A_(v, 0, 1, 0), v_cmp = A_(v, 0, -1, 1), v_ccp = A_(v, 0, 0, 1);
  const double w_ccm = A_(w, 0, 0, -1), w_pcm = A_(w, 1, 0, -1), w_cpm = A_(w, 0, 1, -1),
               w_cmc = A_(w, 0, -1, 0), w_mcc = A_(w, -1, 0, 0), w_ccc = A_(w, 0, 0, 0),
               w_pcc = A_(w, 1, 0, 0), w_cpc = A_(w, 0, 1, 0), w_ccp = A_(w, 0, 0, 1);
  const double c_ccm = A_(psi, 0, 0, -1), c_pcm = A_(psi, 1, 0, -1), c_cpm = A_(psi, 0, 1, -1),
               c_cmc = A_(psi, 0, -1, 0), c_pmc = A_(psi, 1, -1, 0), c_mcc = A_(psi, -1, 0, 0),
               c_ccc = A_(psi, 0, 0, 0), c_pcc = A_(psi, 1, 0, 0), c_mpc = A_(psi, -1, 1, 0),
               c_cpc = A_(psi, 0, 1, 0), c_cmp = A_(psi, 0, -1, 1), c_mcp = A_(psi, -1, 0, 1),
               c_ccp = A_(psi, 0, 0, 1), c_cpp = A_(psi, 0, 1, 1), c_ppc = A_(psi, 1, 1, 0),
               c_pcp = A_(psi, 1, 0, 1);
  const double flx_x_mcc = rho * u_mcc + drho * A_(psiflx_x, -1, 0, 0);
  const double flx_x_ccc = rho * u_ccc + drho * A_(psiflx_x, 0, 0, 0);
  const double flx_x_pcc = rho * u_pcc + drho * A_(psiflx_x, 1, 0, 0);
  const double flx_x_mpc = rho * u_mpc + drho * A_(psiflx_x, -1, 1, 0);
  const double flx_x_cpc = rho * u_cpc + drho * A_(psiflx_x, 0, 1, 0);
  const double flx_x_mcp = rho * u_mcp + drho * A_(psiflx_x, -1, 0, 1);
  const double flx_x_ccp = rho * u_ccp + drho * A_(psiflx_x, 0, 0, 1);
  const double flx_y_cmc = rho * v_cmc + drho * A_(psiflx_y, 0, -1, 0);
  const double flx_y_ccc = rho * v_ccc + drho * A_(psiflx_y, 0, 0, 0);
  const double flx_y_cpc = rho * v_cpc + drho * A_(psiflx_y, 0, 1, 0);
  const double flx_y_pmc = rho * v_pmc + drho * A_(psiflx_y, 1, -1, 0);
  const double flx_y_pcc = rho * v_pcc + drho * A_(psiflx_y, 1, 0, 0);
  const double flx_y_cmp = rho * v_cmp + drho * A_(psiflx_y, 0, -1, 1);
  const double flx_y_ccp = rho * v_ccp + drho * A_(psiflx_y, 0, 0, 1);
  const double flx_z_ccm = rho * w_ccm + drho * A_(psiflx_z, 0, 0, -1);
  const double flx_z_ccc = rho * w_ccc + drho * A_(psiflx_z, 0, 0, 0);
  const double flx_z_ccp = rho * w_ccp + drho * A_(psiflx_z, 0, 0, 1);
  const double flx_z_pcm = rho * w_pcm + drho * A_(psiflx_z, 1, 0, -1);
  const double flx_z_pcc = rho * w_pcc + drho * A_(psiflx_z, 1, 0, 0);
  const double flx_z_cpm = rho * w_cpm + drho * A_(psiflx_z, 0, 1, -1);
  const double flx_z_cpc = rho * w_cpc + drho * A_(psiflx_z, 0, 1, 0);
#undef A_
  const double dzci_c = g.dzci[k], dzci_m = g.dzci[k - 1], dzfi_c = g.dzfi[k], dzfi_p = g.dzfi[k + 1];
  const double uuip = 0.25 * (flx_x_pcc + flx_x_ccc) * (u_ccc + u_pcc);
  const double uuim = 0.25 * (flx_x_mcc + flx_x_ccc) * (u_ccc + u_mcc);
  const double vujp = 0.25 * (flx_y_pcc + flx_y_ccc) * (u_ccc + u_cpc);
  const double vujm = 0.25 * (flx_y_pmc + flx_y_cmc) * (u_ccc + u_cmc);
  const double wukp = 0.25 * (flx_z_pcc + flx_z_ccc) * (u_ccc + u_ccp);
  const double wukm = 0.25 * (flx_z_pcm + flx_z_ccm) * (u_ccc + u_ccm);
  double dudt_aux = dxi * (-uuip + uuim) + dyi * (-vujp + vujm) + dzfi_c * (-wukp + wukm);
  const double uvip = 0.25 * (flx_x_ccc + flx_x_cpc) * (v_ccc + v_pcc);
  const double uvim = 0.25 * (flx_x_mcc + flx_x_mpc) * (v_ccc + v_mcc);
  const double vvjp = 0.25 * (flx_y_ccc + flx_y_cpc) * (v_ccc + v_cpc);
  const double vvjm = 0.25 * (flx_y_ccc + flx_y_cmc) * (v_ccc + v_cmc);
  const double wvkp = 0.25 * (flx_z_ccc + flx_z_cpc) * (v_ccc + v_ccp);
  const double wvkm = 0.25 * (flx_z_ccm + flx_z_cpm) * (v_ccc + v_ccm);
  double dvdt_aux = dxi * (-uvip + uvim) + dyi * (-vvjp + vvjm) + dzfi_c * (-wvkp + wvkm);
  const double uwip = 0.25 * (flx_x_ccc + flx_x_ccp) * (w_ccc + w_pcc);
  const double uwim = 0.25 * (flx_x_mcc + flx_x_mcp) * (w_ccc + w_mcc);
  const double vwjp = 0.25 * (flx_y_ccc + flx_y_ccp) * (w_ccc + w_cpc);
  const double vwjm = 0.25 * (flx_y_cmc + flx_y_cmp) * (w_ccc + w_cmc);
  const double wwkp = 0.25 * (flx_z_ccc + flx_z_ccp) * (w_ccc + w_ccp);
  const double wwkm = 0.25 * (flx_z_ccc + flx_z_ccm) * (w_ccc + w_ccm);
  double dwdt_aux = dxi * (-uwip + uwim) + dyi * (-vwjp + vwjm) + dzci_c * (-wwkp + wwkm);
  {
    const double dudxp = (u_pcc - u_ccc) * dxi, dudxm = (u_ccc - u_mcc) * dxi;
    const double dvdxp = (v_pcc - v_ccc) * dxi, dvdxm = (v_pmc - v_cmc) * dxi;
    const double dudyp = (u_cpc - u_ccc) * dyi, dudym = (u_ccc - u_cmc) * dyi;
    const double dudzp = (u_ccp - u_ccc) * dzci_c, dudzm = (u_ccc - u_ccm) * dzci_m;
    const double dwdxp = (w_pcc - w_ccc) * dxi, dwdxm = (w_pcm - w_ccm) * dxi;
    const double muxp = mu + dmu * c_pcc, muxm = mu + dmu * c_ccc;
    const double muyp = mu + dmu * 0.25 * (c_ccc + c_cpc + c_ppc + c_pcc);
    const double muym = mu + dmu * 0.25 * (c_ccc + c_cmc + c_pmc + c_pcc);
    const double muzp = mu + dmu * 0.25 * (c_ccc + c_pcc + c_ccp + c_pcp);
    const double muzm = mu + dmu * 0.25 * (c_ccc + c_pcc + c_ccm + c_pcm);
    dudt_aux = dudt_aux + dxi * ((dudxp + dudxp) * muxp - (dudxm + dudxm) * muxm) +
               dyi * ((dudyp + dvdxp) * muyp - (dudym + dvdxm) * muym) +
               dzfi_c * ((dudzp + dwdxp) * muzp - (dudzm + dwdxm) * muzm);
  }
  {
    const double dvdxp = (v_pcc - v_ccc) * dxi, dvdxm = (v_ccc - v_mcc) * dxi;
    const double dudyp = (u_cpc - u_ccc) * dyi, dudym = (u_mpc - u_mcc) * dyi;
    const double dvdyp = (v_cpc - v_ccc) * dyi, dvdym = (v_ccc - v_cmc) * dyi;
    const double dvdzp = (v_ccp - v_ccc) * dzci_c, dvdzm = (v_ccc - v_ccm) * dzci_m;
    const double dwdyp = (w_cpc - w_ccc) * dyi, dwdym = (w_cpm - w_ccm) * dyi;
    const double muxp = mu + dmu * 0.25 * (c_ccc + c_pcc + c_ppc + c_cpc);
    const double muxm = mu + dmu * 0.25 * (c_ccc + c_mcc + c_mpc + c_cpc);
    const double muyp = mu + dmu * c_cpc, muym = mu + dmu * c_ccc;
    const double muzp = mu + dmu * 0.25 * (c_ccc + c_cpc + c_cpp + c_ccp);
    const double muzm = mu + dmu * 0.25 * (c_ccc + c_cpc + c_cpm + c_ccm);
    dvdt_aux = dvdt_aux + dxi * ((dvdxp + dudyp) * muxp - (dvdxm + dudym) * muxm) +
               dyi * ((dvdyp + dvdyp) * muyp - (dvdym + dvdym) * muym) +
               dzfi_c * ((dvdzp + dwdyp) * muzp - (dvdzm + dwdym) * muzm);
  }
  {
    const double dwdxp = (w_pcc - w_ccc) * dxi, dwdxm = (w_ccc - w_mcc) * dxi;
    const double dudzp = (u_ccp - u_ccc) * dzci_c, dudzm = (u_mcp - u_mcc) * dzci_c;
    const double dwdyp = (w_cpc - w_ccc) * dyi, dwdym = (w_ccc - w_cmc) * dyi;
    const double dvdzp = (v_ccp - v_ccc) * dzci_c, dvdzm = (v_cmp - v_cmc) * dzci_c;
    const double dwdzp = (w_ccp - w_ccc) * dzfi_p, dwdzm = (w_ccc - w_ccm) * dzfi_c;
    const double muxp = mu + dmu * 0.25 * (c_ccc + c_pcc + c_ccp + c_pcp);
    const double muxm = mu + dmu * 0.25 * (c_ccc + c_mcc + c_ccp + c_mcp);
    const double muyp = mu + dmu * 0.25 * (c_ccc + c_cpc + c_ccp + c_cpp);
    const double muym = mu + dmu * 0.25 * (c_ccc + c_cmc + c_ccp + c_cmp);
    const double muzp = mu + dmu * c_ccp, muzm = mu + dmu * c_ccc;
    dwdt_aux = dwdt_aux + dxi * ((dwdxp + dudzp) * muxp - (dwdxm + dudzm) * muxm) +
               dyi * ((dwdyp + dvdzp) * muyp - (dwdym + dvdzm) * muym) +
               dzci_c * ((dwdzp + dwdzp) * muzp - (dwdzm + dwdzm) * muzm);
  }
  return {dudt_aux, dvdt_aux, dwdt_aux};
}

// mom_xyz_oth, src/mom.f90:912-1038 (CONSTANT_COEFFS_POISSON, Brackbill per
// Phys; with s, the Boussinesq buoyancy of src/mom.f90:1017-1024; with sp,
// the balanced capillary split of src/mom.f90:982-1032)
__device__ __forceinline__ AdOut mom_oth_cell(const Geo& g, const Phys& ph, double dt_r, const double* rho_av,
                                              int i, int j, int k, const double* __restrict__ p,
                                              const double* __restrict__ psi, const double* __restrict__ kappa,
                                              const double* __restrict__ s, const SurfSplit* sp,
                                              const double* __restrict__ pn, const double* __restrict__ po) {
  const double rho = ph.rho12[1], drho = ph.rho12[0] - ph.rho12[1];
  const double dxi = g.dxi, dyi = g.dyi, dzci_c = g.dzci[k];
  const int ccc = g.h(i, j, k), pcc = ccc + 1, cpc = ccc + g.sx, ccp = ccc + g.sxy;
  const double p_ccc = LD(p, ccc), p_pcc = LD(p, pcc), p_cpc = LD(p, cpc), p_ccp = LD(p, ccp);
  const double q_ccc = (1. + dt_r) * LD(pn, ccc) - dt_r * LD(po, ccc);
  const double q_pcc = (1. + dt_r) * LD(pn, pcc) - dt_r * LD(po, pcc);
  const double q_cpc = (1. + dt_r) * LD(pn, cpc) - dt_r * LD(po, cpc);
  const double q_ccp = (1. + dt_r) * LD(pn, ccp) - dt_r * LD(po, ccp);
  const double k_ccc = LD(kappa, ccc), k_pcc = LD(kappa, pcc), k_cpc = LD(kappa, cpc), k_ccp = LD(kappa, ccp);
  const double c_ccc = LD(psi, ccc), c_pcc = LD(psi, pcc), c_cpc = LD(psi, cpc), c_ccp = LD(psi, ccp);
  const double psixp = 0.5 * (c_pcc + c_ccc), psiyp = 0.5 * (c_cpc + c_ccc), psizp = 0.5 * (c_ccp + c_ccc);
  const double rhoxp = rho + drho * psixp, rhoyp = rho + drho * psiyp, rhozp = rho + drho * psizp;
  const double dpdx = (p_pcc - p_ccc) * dxi, dpdy = (p_cpc - p_ccc) * dyi, dpdz = (p_ccp - p_ccc) * dzci_c;
  double dudt_aux = ph.bforce[0] + (rhoxp - rho_av[0]) * ph.gacc[0];
  double dvdt_aux = ph.bforce[1] + (rhoyp - rho_av[1]) * ph.gacc[1];
  double dwdt_aux = ph.bforce[2] + (rhozp - rho_av[2]) * ph.gacc[2];
  double skappaxp = 0.5 * (k_pcc + k_ccc) * ph.surf_factor;
  double skappayp = 0.5 * (k_cpc + k_ccc) * ph.surf_factor;
  double skappazp = 0.5 * (k_ccp + k_ccc) * ph.surf_factor;
  if (ph.brackbill) {  // _CAPILLARY_BRACKBILL_NORMALIZATION
    skappaxp = skappaxp * rhoxp; skappayp = skappayp * rhoyp; skappazp = skappazp * rhozp;
  }
  const double surfx = skappaxp * (c_pcc - c_ccc) * dxi;
  const double surfy = skappayp * (c_cpc - c_ccc) * dyi;
  const double surfz = skappazp * (c_ccp - c_ccc) * dzci_c;
  double dpdx_e = (q_pcc - q_ccc) * dxi, dpdy_e = (q_cpc - q_ccc) * dyi, dpdz_e = (q_ccp - q_ccc) * dzci_c;
  double dpx = dpdx, dpy = dpdy, dpz = dpdz;
  if (sp) {
    const int t = g.t(i, j, k);
    const double sxn = sp->n[0][t], syn = sp->n[1][t], szn = sp->n[2][t];
    const double sxe = (1. + dt_r) * sxn - dt_r * sp->o[0][t];
    const double sye = (1. + dt_r) * syn - dt_r * sp->o[1][t];
    const double sze = (1. + dt_r) * szn - dt_r * sp->o[2][t];
    dpx = dpx - surfx; dpy = dpy - surfy; dpz = dpz - surfz;
    dpdx_e = dpdx_e - sxe; dpdy_e = dpdy_e - sye; dpdz_e = dpdz_e - sze;
    if (sp->out_o[0]) { sp->out_o[0][t] = sxn; sp->out_o[1][t] = syn; sp->out_o[2][t] = szn; }
    sp->out_n[0][t] = surfx; sp->out_n[1][t] = surfy; sp->out_n[2][t] = surfz;
  } else {
    dudt_aux = dudt_aux + surfx;
    dvdt_aux = dvdt_aux + surfy;
    dwdt_aux = dwdt_aux + surfz;
  }
  dudt_aux = dudt_aux - (dpdx_e + rhoxp * ph.irho0 * (dpx - dpdx_e));
  dvdt_aux = dvdt_aux - (dpdy_e + rhoyp * ph.irho0 * (dpy - dpdy_e));
  dwdt_aux = dwdt_aux - (dpdz_e + rhozp * ph.irho0 * (dpz - dpdz_e));
  if (s) {
    const double s_ccc = LD(s, ccc), s_pcc = LD(s, pcc), s_cpc = LD(s, cpc), s_ccp = LD(s, ccp);
    const double factorxp = ph.rhobeta + ph.drhobeta * psixp;
    const double factoryp = ph.rhobeta + ph.drhobeta * psiyp;
    const double factorzp = ph.rhobeta + ph.drhobeta * psizp;
    dudt_aux = dudt_aux - ph.gacc[0] * factorxp * 0.5 * (s_pcc + s_ccc);
    dvdt_aux = dvdt_aux - ph.gacc[1] * factoryp * 0.5 * (s_cpc + s_ccc);
    dwdt_aux = dwdt_aux - ph.gacc[2] * factorzp * 0.5 * (s_ccp + s_ccc);
  }
  return {dudt_aux, dvdt_aux, dwdt_aux};
}

__global__ void __launch_bounds__(128) k_mom_ad(Geo g, Phys ph, const double* __restrict__ fx,
    const double* __restrict__ fy, const double* __restrict__ fz, const double* __restrict__ u,
    const double* __restrict__ v, const double* __restrict__ w, const double* __restrict__ psi,
    double* __restrict__ du, double* __restrict__ dv, double* __restrict__ dw) {
  INTERIOR_IJK(g)
  const AdOut r = mom_ad_cell(g, ph, i, j, k, fx, fy, fz, u, v, w, psi);
  const int t = g.t(i, j, k);
  du[t] = r.du; dv[t] = r.dv; dw[t] = r.dw;
}

void launch_mom_ad(const Launch& L, const Geo& g, const Phys& ph, const double* fx, const double* fy,
                   const double* fz, const double* u, const double* v, const double* w, const double* psi,
                   double* du, double* dv, double* dw) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  k_mom_ad<<<gr, b, 0, L.st>>>(g, ph, fx, fy, fz, u, v, w, psi, du, dv, dw);
}

__global__ void k_mom_oth(Geo g, Phys ph, const DevScalars* __restrict__ sc, const double* __restrict__ p,
                          const double* __restrict__ psi, const double* __restrict__ kappa,
                          const double* __restrict__ s, const SurfSplit sp, int with_sp,
                          const double* __restrict__ pn, const double* __restrict__ po, double* __restrict__ du,
                          double* __restrict__ dv, double* __restrict__ dw) {
  INTERIOR_IJK(g)
  const AdOut r = mom_oth_cell(g, ph, sc->dt_r, sc->rho_av, i, j, k, p, psi, kappa, s, with_sp ? &sp : nullptr, pn,
                               po);
  const int t = g.t(i, j, k);
  du[t] = r.du; dv[t] = r.dv; dw[t] = r.dw;
}

void launch_mom_oth(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* p,
                    const double* psi, const double* kappa, const double* s, const SurfSplit* sp, const double* pn,
                    const double* po, double* du, double* dv, double* dw) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  const SurfSplit none{};
  k_mom_oth<<<gr, b, 0, L.st>>>(g, ph, sc, p, psi, kappa, s, sp ? *sp : none, sp ? 1 : 0, pn, po, du, dv, dw);
}

// rk update 1 (src/rk.f90:86-101): u = u*rho_n/rho_p + (f1 R + f2 Ro)/rho_p; on the
// first call Ro := R.  The new R is written into the history slot `duo`
// (the swap of src/rk.f90:106-108 becomes the caller's pointer swap).
__global__ void k_rk_update1(Geo g, Phys ph, const DevScalars* __restrict__ sc, const double* __restrict__ psio,
                             const double* __restrict__ psi, const double* __restrict__ du,
                             const double* __restrict__ dv, const double* __restrict__ dw,
                             double* __restrict__ duo, double* __restrict__ dvo, double* __restrict__ dwo,
                             double* __restrict__ u, double* __restrict__ v, double* __restrict__ w) {
  INTERIOR_IJK(g)
  const double rho = ph.rho12[1], drho = ph.rho12[0] - ph.rho12[1];
  const int c = g.h(i, j, k), t = g.t(i, j, k);
  const double po_c = LD(psio, c), ps_c = LD(psi, c);
  const double rhox_n = rho + drho * 0.5 * (po_c + LD(psio, c + 1));
  const double rhoy_n = rho + drho * 0.5 * (po_c + LD(psio, c + g.sx));
  const double rhoz_n = rho + drho * 0.5 * (po_c + LD(psio, c + g.sxy));
  const double rhox_p = rho + drho * 0.5 * (ps_c + LD(psi, c + 1));
  const double rhoy_p = rho + drho * 0.5 * (ps_c + LD(psi, c + g.sx));
  const double rhoz_p = rho + drho * 0.5 * (ps_c + LD(psi, c + g.sxy));
  const double Ru = du[t], Rv = dv[t], Rw = dw[t];
  const bool first = sc->first_rk;
  const double Ruo = first ? Ru : duo[t], Rvo = first ? Rv : dvo[t], Rwo = first ? Rw : dwo[t];
  const double f1 = sc->f1, f2 = sc->f2;
  u[c] = u[c] * rhox_n / rhox_p + (f1 * Ru + f2 * Ruo) / rhox_p;
  v[c] = v[c] * rhoy_n / rhoy_p + (f1 * Rv + f2 * Rvo) / rhoy_p;
  w[c] = w[c] * rhoz_n / rhoz_p + (f1 * Rw + f2 * Rwo) / rhoz_p;
}

void launch_rk_update1(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* psio,
                       const double* psi, const double* du, const double* dv, const double* dw, double* duo,
                       double* dvo, double* dwo, double* u, double* v, double* w) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  k_rk_update1<<<gr, b, 0, L.st>>>(g, ph, sc, psio, psi, du, dv, dw, duo, dvo, dwo, u, v, w);
}

// rk update 2 (src/rk.f90:118-130): u = u + f12*R/rho_p
__global__ void k_rk_update2(Geo g, Phys ph, const DevScalars* __restrict__ sc, const double* __restrict__ psi,
                             const double* __restrict__ du, const double* __restrict__ dv,
                             const double* __restrict__ dw, double* __restrict__ u, double* __restrict__ v,
                             double* __restrict__ w) {
  INTERIOR_IJK(g)
  const double rho = ph.rho12[1], drho = ph.rho12[0] - ph.rho12[1];
  const int c = g.h(i, j, k), t = g.t(i, j, k);
  const double ps_c = LD(psi, c);
  const double rhox_p = rho + drho * 0.5 * (ps_c + LD(psi, c + 1));
  const double rhoy_p = rho + drho * 0.5 * (ps_c + LD(psi, c + g.sx));
  const double rhoz_p = rho + drho * 0.5 * (ps_c + LD(psi, c + g.sxy));
  const double f12 = sc->f12;
  u[c] = u[c] + f12 * du[t] / rhox_p;
  v[c] = v[c] + f12 * dv[t] / rhoy_p;
  w[c] = w[c] + f12 * dw[t] / rhoz_p;
}

void launch_rk_update2(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* psi,
                       const double* du, const double* dv, const double* dw, double* u, double* v, double* w) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  k_rk_update2<<<gr, b, 0, L.st>>>(g, ph, sc, psi, du, dv, dw, u, v, w);
}

// ---------------------------------------------------------------------------
// The whole of rk (src/rk.f90:16-131) in one pass: the z-marching tile kernel
// of k_tiles.cu (reads p for pn, as the driver calls rk with pn = p)
// ---------------------------------------------------------------------------
void launch_momentum_fused(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* u,
                           const double* v, const double* w, const double* psi, const double* psio,
                           const double* fx, const double* fy, const double* fz, const double* p,
                           const double* po, const double* kappa, const double* s, const SurfSplit* sp,
                           double* duo, double* dvo, double* dwo, double* uo, double* vo, double* wo) {
  launch_momentum_t<double>(L, g, ph, sc, u, v, w, psi, psio, fx, fy, fz, p, po, kappa, s, sp, duo, dvo, dwo, uo, vo,
                            wo);
}

// ---------------------------------------------------------------------------
// scalar transport (_SCALAR): scal_ad, src/scal.f90:13-66, per interior cell
// (the advecting flux is rho*cp*u + (rho1*cp1 - rho2*cp2)*psiflx; TI is the
// storage type of the phase fluxes), and the AB2 update of rk_scal,
// src/rk.f90:172-186
// ---------------------------------------------------------------------------
template <typename TI>
__device__ __forceinline__ double scal_ad_cell(const Geo& g, const Phys& ph, int i, int j, int k,
                                               const TI* __restrict__ fx, const TI* __restrict__ fy,
                                               const TI* __restrict__ fz, const double* __restrict__ psi,
                                               const double* __restrict__ u, const double* __restrict__ v,
                                               const double* __restrict__ w, const double* __restrict__ s) {
  const double ka = ph.ka12[1], dka = ph.ka12[0] - ph.ka12[1];
  const double rhocp = ph.rhocp12[1], drhocp = ph.rhocp12[0] - ph.rhocp12[1];
  const double dxi = g.dxi, dyi = g.dyi, dzfi_c = g.dzfi[k];
  const int c = g.h(i, j, k), xm = c - 1, xp = c + 1, ym = c - g.sx, yp = c + g.sx, zm = c - g.sxy, zp = c + g.sxy;
  const double s_c = LD(s, c), s_xp = LD(s, xp), s_xm = LD(s, xm), s_yp = LD(s, yp), s_ym = LD(s, ym),
               s_zp = LD(s, zp), s_zm = LD(s, zm);
  const double usip = 0.5 * (rhocp * LD(u, c) + drhocp * (double)LD(fx, c)) * (s_xp + s_c);
  const double usim = 0.5 * (rhocp * LD(u, xm) + drhocp * (double)LD(fx, xm)) * (s_xm + s_c);
  const double vsjp = 0.5 * (rhocp * LD(v, c) + drhocp * (double)LD(fy, c)) * (s_yp + s_c);
  const double vsjm = 0.5 * (rhocp * LD(v, ym) + drhocp * (double)LD(fy, ym)) * (s_ym + s_c);
  const double wskp = 0.5 * (rhocp * LD(w, c) + drhocp * (double)LD(fz, c)) * (s_zp + s_c);
  const double wskm = 0.5 * (rhocp * LD(w, zm) + drhocp * (double)LD(fz, zm)) * (s_zm + s_c);
  const double ps_c = LD(psi, c);
  const double kaxp = ka + dka * 0.5 * (LD(psi, xp) + ps_c), kaxm = ka + dka * 0.5 * (ps_c + LD(psi, xm));
  const double kayp = ka + dka * 0.5 * (LD(psi, yp) + ps_c), kaym = ka + dka * 0.5 * (ps_c + LD(psi, ym));
  const double kazp = ka + dka * 0.5 * (LD(psi, zp) + ps_c), kazm = ka + dka * 0.5 * (ps_c + LD(psi, zm));
  const double dsdxp = (s_xp - s_c) * dxi, dsdxm = (s_c - s_xm) * dxi;
  const double dsdyp = (s_yp - s_c) * dyi, dsdym = (s_c - s_ym) * dyi;
  const double dsdzp = (s_zp - s_c) * g.dzci[k], dsdzm = (s_c - s_zm) * g.dzci[k - 1];
  return dxi * (-usip + usim) + dyi * (-vsjp + vsjm) + dzfi_c * (-wskp + wskm) +
         ((kaxp * dsdxp - kaxm * dsdxm) * dxi + (kayp * dsdyp - kaym * dsdym) * dyi +
          (kazp * dsdzp - kazm * dsdzm) * dzfi_c);
}

// s_new = s*rhocp_n/rhocp_p + (f1*dsdt + f2*dsdto + f12*ssource)/rhocp_p
__device__ __forceinline__ double scal_update(const Phys& ph, const DevScalars* __restrict__ sc, double s_c,
                                              double ps_c, double pso_c, double d, double dO) {
  const double rhocp = ph.rhocp12[1], drhocp = ph.rhocp12[0] - ph.rhocp12[1];
  const double rhocp_p = rhocp + drhocp * ps_c;
  const double rhocp_n = rhocp + drhocp * pso_c;
  return s_c * rhocp_n / rhocp_p + (sc->f1 * d + sc->f2 * dO + sc->f12 * ph.ssource) / rhocp_p;
}

template <typename TI>
struct ScalAd {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const Phys& ph, const TI* __restrict__ fx,
      const TI* __restrict__ fy, const TI* __restrict__ fz, const double* __restrict__ psi,
      const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ w,
      const double* __restrict__ s, double* __restrict__ dsdt) {
    INTERIOR_IJK_B(g, bk)
    dsdt[g.t(i, j, k)] = scal_ad_cell<TI>(g, ph, i, j, k, fx, fy, fz, psi, u, v, w, s);
  }
};
template <typename TI>
__global__ void k_scal_ad(Geo g, Phys ph, const TI* __restrict__ fx, const TI* __restrict__ fy,
                          const TI* __restrict__ fz, const double* __restrict__ psi, const double* __restrict__ u,
                          const double* __restrict__ v, const double* __restrict__ w, const double* __restrict__ s,
                          double* __restrict__ dsdt) {
  ScalAd<TI>::run(blk_here(), g, ph, fx, fy, fz, psi, u, v, w, s, dsdt);
}
template <typename TI>
void launch_scal_ad(const Launch& L, const Geo& g, const Phys& ph, const TI* fx, const TI* fy, const TI* fz,
                    const double* psi, const double* u, const double* v, const double* w, const double* s,
                    double* dsdt) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  kgo<ScalAd<TI>, 128, 1>(L, k_scal_ad<TI>, gr, b, 0, g, ph, fx, fy, fz, psi, u, v, w, s, dsdt);
}

// the step's rk_scal in one pass: scal_ad of the old scalar, the AB2 update
// into s_out (another buffer, so the stencil reads stay unmodified) and the
// new dsdt into the history slot (the swap of src/rk.f90:190 is implicit)
template <typename TI>
struct ScalStep {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const Phys& ph,
      const DevScalars* __restrict__ sc, const TI* __restrict__ fx, const TI* __restrict__ fy,
      const TI* __restrict__ fz, const double* __restrict__ psi, const double* __restrict__ psio,
      const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ w,
      const double* __restrict__ s, double* __restrict__ hist, double* __restrict__ s_out) {
    if (HALTED(sc)) return;
    INTERIOR_IJK_B(g, bk)
    const double d = scal_ad_cell<TI>(g, ph, i, j, k, fx, fy, fz, psi, u, v, w, s);
    const int c = g.h(i, j, k), t = g.t(i, j, k);
    const double dO = sc->first_scal ? d : hist[t];
    s_out[c] = scal_update(ph, sc, LD(s, c), LD(psi, c), LD(psio, c), d, dO);
    hist[t] = d;
  }
};
template <typename TI>
__global__ void k_scal_step(Geo g, Phys ph, const DevScalars* __restrict__ sc, const TI* __restrict__ fx,
                            const TI* __restrict__ fy, const TI* __restrict__ fz, const double* __restrict__ psi,
                            const double* __restrict__ psio, const double* __restrict__ u,
                            const double* __restrict__ v, const double* __restrict__ w,
                            const double* __restrict__ s, double* __restrict__ hist, double* __restrict__ s_out) {
  ScalStep<TI>::run(blk_here(), g, ph, sc, fx, fy, fz, psi, psio, u, v, w, s, hist, s_out);
}
template <typename TI>
void launch_scal_step(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const TI* fx,
                      const TI* fy, const TI* fz, const double* psi, const double* psio, const double* u,
                      const double* v, const double* w, const double* s, double* hist, double* s_out) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  kgo<ScalStep<TI>, 128, 1>(L, k_scal_step<TI>, gr, b, 0, g, ph, sc, fx, fy, fz, psi, psio, u, v, w, s, hist, s_out);
}

// the second loop of rk_scal alone (src/rk.f90:176-186), in place: dsdt from
// scal_ad, the history slot takes it
__global__ void k_scal_update(Geo g, Phys ph, const DevScalars* __restrict__ sc, const double* __restrict__ psi,
                              const double* __restrict__ psio, const double* __restrict__ dsdt,
                              double* __restrict__ hist, double* __restrict__ s) {
  INTERIOR_IJK(g)
  const int c = g.h(i, j, k), t = g.t(i, j, k);
  const double d = dsdt[t];
  const double dO = sc->first_scal ? d : hist[t];
  s[c] = scal_update(ph, sc, s[c], LD(psi, c), LD(psio, c), d, dO);
  hist[t] = d;
}
void launch_scal_update(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* psi,
                        const double* psio, const double* dsdt, double* hist, double* s) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  k_scal_update<<<gr, b, 0, L.st>>>(g, ph, sc, psi, psio, dsdt, hist, s);
}

template void launch_scal_ad<double>(const Launch&, const Geo&, const Phys&, const double*, const double*,
                                     const double*, const double*, const double*, const double*, const double*,
                                     const double*, double*);
template void launch_scal_step<double>(const Launch&, const Geo&, const Phys&, const DevScalars*, const double*,
                                       const double*, const double*, const double*, const double*, const double*,
                                       const double*, const double*, const double*, double*, double*);
template void launch_scal_step<float>(const Launch&, const Geo&, const Phys&, const DevScalars*, const float*,
                                      const float*, const float*, const double*, const double*, const double*,
                                      const double*, const double*, const double*, double*, double*);

// ---------------------------------------------------------------------------
// fillps, src/fillps.f90:13-51
// ---------------------------------------------------------------------------
struct Fillps {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const Phys& ph,
      const DevScalars* __restrict__ sc, const double* __restrict__ u, const double* __restrict__ v,
      const double* __restrict__ w, double* __restrict__ p) {
    if (HALTED(sc)) return;
    INTERIOR_IJK_B(g, bk)
    const double dti = sc->dti, dtidxi = dti * g.dxi, dtidyi = dti * g.dyi;
    const int c = g.h(i, j, k);
    p[c] = ph.rho0 * ((LD(w, c) - LD(w, c - g.sxy)) * dti * g.dzfi[k] + (LD(v, c) - LD(v, c - g.sx)) * dtidyi +
                      (LD(u, c) - LD(u, c - 1)) * dtidxi);
  }
};
__global__ void k_fillps(Geo g, Phys ph, const DevScalars* __restrict__ sc, const double* __restrict__ u,
                         const double* __restrict__ v, const double* __restrict__ w, double* __restrict__ p) {
  Fillps::run(blk_here(), g, ph, sc, u, v, w, p);
}
void launch_fillps(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* u,
                   const double* v, const double* w, double* p) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  kgo<Fillps, 128, 1>(L, k_fillps, gr, b, 0, g, ph, sc, u, v, w, p);
}

// ---------------------------------------------------------------------------
// correc, src/correc.f90:13-67: the three loops, ghost ranges included.
// One thread per (i,j,k) of the halo array; each component updates over its
// own index range.
// ---------------------------------------------------------------------------
__global__ void k_correc(Geo g, Phys ph, const DevScalars* __restrict__ sc, const double* __restrict__ p,
                         double* __restrict__ u, double* __restrict__ v, double* __restrict__ w) {
  if (HALTED(sc)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > g.nx + 1) return;
  const int j = blockIdx.y, k = blockIdx.z;
  const double dt = sc->dt, rhop = ph.rho0;
  const int c = g.h(i, j, k);
  const double pc = LD(p, c);
  if (i <= g.nx) u[c] = u[c] - dt * g.dxi * (LD(p, c + 1) - pc) / rhop;
  if (j <= g.ny) v[c] = v[c] - dt * g.dyi * (LD(p, c + g.sx) - pc) / rhop;
  if (k <= g.nz) w[c] = w[c] - dt * g.dzci[k] * (LD(p, c + g.sxy) - pc) / rhop;
}
void launch_correc(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* p, double* u,
                   double* v, double* w) {
  dim3 b(g.nx + 2 >= 128 ? 128 : 64), gr((g.nx + 2 + b.x - 1) / b.x, g.ny + 2, g.nz + 2);
  k_correc<<<gr, b, 0, L.st>>>(g, ph, sc, p, u, v, w);
}

// correc (src/correc.f90:13-67) and updatep (src/updatep.f90:13-24) of the
// step in one pass: both read the correction phi, and updatep needs none of
// the velocity ghost fills that follow correc.  32x8 point tiles of the halo
// array; pout = phi + pp on the interior (the new pressure into the po slot).
//
// wrap (bit d: direction d periodic, its images written here).  correc
// already updates the whole halo range but u at i = nx+1, v at j = ny+1 and
// w at k = nz+1, and with periodic ghosts of its operands (phi, and the
// predicted velocity, both filled before) the values it computes at a ghost
// point equal those at the point's periodic image, operation for operation
// (w at k = 0 takes dzci(nz), the metric of its image).
// So the periodic fill after correc only has to supply those three planes:
// the thread of u(1), v(1) or w(1) stores its value there (no thread reads
// them here).  pout is also evaluated at the ghost points of the wrapped
// directions, from the periodic ghosts of phi and pp.
constexpr int kCorrecLevels = 2;  // z levels per thread of k_correc_updatep
struct CorrecUpdatep {
  // each thread owns one (i, j) column and kCorrecLevels consecutive levels:
  // all loads first (p at level k+1 is the next level's own p), then the
  // updates, so that a warp has many independent loads in flight
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const Phys& ph,
      const DevScalars* __restrict__ sc, const double* __restrict__ p, double* __restrict__ u,
      double* __restrict__ v, double* __restrict__ w, const double* __restrict__ pp, double* __restrict__ pout,
      int wrap) {
    constexpr int KC = kCorrecLevels;
    if (HALTED(sc)) return;
    const int i = bk.x * 32 + threadIdx.x, j = bk.y * 8 + threadIdx.y, k0 = bk.z * KC;
    if (i > g.nx + 1 || j > g.ny + 1) return;
    const double dt = sc->dt, rhop = ph.rho0;
    const int c0 = g.h(i, j, k0);
    const bool xin = i <= g.nx, yin = j <= g.ny, ij_int = i >= 1 && xin && j >= 1 && yin;
    // pout at (i,j): interior, or a ghost of a wrapped direction
    const bool ij_p = (((wrap & 1) != 0) || (i >= 1 && xin)) && (((wrap & 2) != 0) || (j >= 1 && yin));
    auto k_p = [&](int k) { return ((wrap & 4) != 0) || (k >= 1 && k <= g.nz); };
    double pc[KC + 1], px[KC], py[KC], uo[KC], vo[KC], wo[KC], pq[KC];
#pragma unroll
    for (int q = 0; q < KC; ++q) {
      const int k = k0 + q, c = c0 + q * g.sxy;
      if (k <= g.nz + 1) {
        pc[q] = LD(p, c);
        px[q] = xin ? LD(p, c + 1) : 0.;
        py[q] = yin ? LD(p, c + g.sx) : 0.;
        uo[q] = xin ? u[c] : 0.;
        vo[q] = yin ? v[c] : 0.;
        wo[q] = k <= g.nz ? w[c] : 0.;
        pq[q] = (ij_p && k_p(k)) ? LD(pp, c) : 0.;
      }
    }
    pc[KC] = (k0 + KC - 1 <= g.nz) ? LD(p, c0 + KC * g.sxy) : 0.;
#pragma unroll
    for (int q = 0; q < KC; ++q) {
      const int k = k0 + q, c = c0 + q * g.sxy;
      if (k > g.nz + 1) break;
      if (xin) {
        const double un = uo[q] - dt * g.dxi * (px[q] - pc[q]) / rhop;
        u[c] = un;
        if ((wrap & 1) && i == 1) u[c + g.nx] = un;
      }
      if (yin) {
        const double vn = vo[q] - dt * g.dyi * (py[q] - pc[q]) / rhop;
        v[c] = vn;
        if ((wrap & 2) && j == 1) v[c + g.ny * g.sx] = vn;
      }
      if (k <= g.nz) {
        // with periodic z, w(0) is w(nz)'s image: the same operands, and
        // dzci(nz), which may differ from dzci(0) in its last bits
        const double dzk = ((wrap & 4) && k == 0) ? g.dzci[g.nz] : g.dzci[k];
        const double wn = wo[q] - dt * dzk * (pc[q + 1] - pc[q]) / rhop;
        w[c] = wn;
        if ((wrap & 4) && k == 1) w[c + g.nz * g.sxy] = wn;
      }
      if (ij_p && k_p(k)) pout[c] = pc[q] + pq[q];
    }
  }
};
__global__ void __launch_bounds__(256) k_correc_updatep(Geo g, Phys ph, const DevScalars* __restrict__ sc,
                                                        const double* __restrict__ p, double* __restrict__ u,
                                                        double* __restrict__ v, double* __restrict__ w,
                                                        const double* __restrict__ pp, double* __restrict__ pout,
                                                        int wrap) {
  CorrecUpdatep::run(blk_here(), g, ph, sc, p, u, v, w, pp, pout, wrap);
}
void launch_correc_updatep(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* p,
                           double* u, double* v, double* w, const double* pp, double* pout) {
  const dim3 b(32, 8), gr((g.nx + 2 + 31) / 32, (g.ny + 2 + 7) / 8, (g.nz + 2 + kCorrecLevels - 1) / kCorrecLevels);
  kgo<CorrecUpdatep, 256, 1>(L, k_correc_updatep, gr, b, 0, g, ph, sc, p, u, v, w, pp, pout, L.wrap);
}

// updatep, src/updatep.f90:13-24
__global__ void k_updatep_interior(Geo g, const DevScalars* __restrict__ sc, const double* __restrict__ phi,
                                   const double* __restrict__ pp, double* __restrict__ pout) {
  if (HALTED(sc)) return;
  INTERIOR_IJK(g)
  const int c = g.h(i, j, k);
  pout[c] = LD(phi, c) + LD(pp, c);
}
void launch_updatep_interior(const Launch& L, const Geo& g, const DevScalars* sc, const double* phi,
                             const double* pp, double* pout) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  k_updatep_interior<<<gr, b, 0, L.st>>>(g, sc, phi, pp, pout);
}
__global__ void k_add_full(int n, const double* __restrict__ pp, double* __restrict__ p) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) p[q] = p[q] + pp[q];
}
void launch_updatep_full(const Launch& L, const Geo& g, const double* pp, double* p) {
  const int n = g.hsize();
  k_add_full<<<(n + 255) / 256, 256, 0, L.st>>>(n, pp, p);
}
struct Copy {
  static __device__ __forceinline__ void run(const Blk& bk, size_t n, const double* __restrict__ s,
      double* __restrict__ d) {
    const size_t q = (size_t)bk.x * blockDim.x + threadIdx.x;
    if (q < n) d[q] = s[q];
  }
};
__global__ void k_copy(size_t n, const double* __restrict__ s, double* __restrict__ d) {
  Copy::run(blk_here(), n, s, d);
}
void launch_copy(const Launch& L, size_t n, const double* src, double* dst) {
  kgo<Copy, 256, 1>(L, k_copy, (unsigned)((n + 255) / 256), 256, 0, n, src, dst);
}
struct FillV {
  static __device__ __forceinline__ void run(const Blk& bk, size_t n, double val, double* __restrict__ d) {
    const size_t q = (size_t)bk.x * blockDim.x + threadIdx.x;
    if (q < n) d[q] = val;
  }
};
__global__ void k_fillv(size_t n, double val, double* __restrict__ d) {
  FillV::run(blk_here(), n, val, d);
}
void launch_fill(const Launch& L, size_t n, double val, double* dst) {
  kgo<FillV, 256, 1>(L, k_fillv, (unsigned)((n + 255) / 256), 256, 0, n, val, dst);
}
struct FillF {
  static __device__ __forceinline__ void run(const Blk& bk, size_t n, float val, float* __restrict__ d) {
    const size_t q = (size_t)bk.x * blockDim.x + threadIdx.x;
    if (q < n) d[q] = val;
  }
};
__global__ void k_fillf(size_t n, float val, float* __restrict__ d) {
  FillF::run(blk_here(), n, val, d);
}
void launch_fill(const Launch& L, size_t n, float val, float* dst) {
  kgo<FillF, 256, 1>(L, k_fillf, (unsigned)((n + 255) / 256), 256, 0, n, val, dst);
}
__global__ void k_widen(size_t n, const float* __restrict__ s, double* __restrict__ d) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < n) d[q] = (double)s[q];
}
void launch_widen(const Launch& L, size_t n, const float* src, double* dst) {
  k_widen<<<(unsigned)((n + 255) / 256), 256, 0, L.st>>>(n, src, dst);
}

// ---------------------------------------------------------------------------
// reductions.  Maxima of non-negative doubles via atomicMax on the bit
// pattern (order independent); sums via per-block partials reduced in a
// fixed order (deterministic).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double block_max(double v) {
  __shared__ double s[32];
  v = warp_max(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) s[wid] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? s[threadIdx.x] : 0.;
  if (wid == 0) v = warp_max(v);
  return v;
}
// deterministic block sum: fixed tree order for a given blockDim
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double s[32];
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) s[wid] = v;
  __syncthreads();
  const int nw = (blockDim.x + 31) >> 5;
  v = (threadIdx.x < nw) ? s[threadIdx.x] : 0.;
  if (wid == 0) v = warp_sum(v);
  return v;
}
// |u_c|^2 of acdi_set_gamma (src/acdi.f90:52-55): (uc^2 + vc^2) + wc^2,
// rounded at each operation as the reference evaluates it (no contraction
// into FMAs), the same bits in every kernel that forms it
__device__ __forceinline__ double vel2(double uc, double vc, double wc) {
  return __dadd_rn(__dadd_rn(__dmul_rn(uc, uc), __dmul_rn(vc, vc)), __dmul_rn(wc, wc));
}
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* slot, double v) {
  atomicMax(slot, (unsigned long long)__double_as_longlong(v));
}

// acdi_set_gamma, src/acdi.f90:32-62: max over the interior of |u_c|^2
__global__ void k_gamma_max(Geo g, DevScalars* __restrict__ sc, double* __restrict__ part,
                            const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ w) {
  if (HALTED(sc)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y + 1, k = blockIdx.z + 1;
  double vel = 0.;
  if (i <= g.nx) {
    const int c = g.h(i, j, k);
    const double uc = 0.5 * (LD(u, c) + LD(u, c - 1));
    const double vc = 0.5 * (LD(v, c) + LD(v, c - g.sx));
    const double wc = 0.5 * (LD(w, c) + LD(w, c - g.sxy));
    vel = vel2(uc, vc, wc);
  }
  vel = block_max(vel);
  if (threadIdx.x == 0) part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = vel;
}
// maximum of n non-negative partials, one block
__device__ __forceinline__ double reduce_max_partials(int n, const double* __restrict__ part) {
  double m = 0.;
  for (int q = threadIdx.x; q < n; q += blockDim.x) m = fmax(m, part[q]);
  return block_max(m);
}
__device__ __forceinline__ void gamma_finish(const Phys& ph, DevScalars* sc, double velmax, int apply_floor) {
  double gam = sqrt(velmax) * ph.gam_factor;
  if (apply_floor) gam = fmax(gam, ph.gam_min);
  sc->gam = gam;
}
__global__ void k_gamma_final(Phys ph, DevScalars* __restrict__ sc, int n, const double* __restrict__ part,
                              int apply_floor) {
  if (HALTED(sc)) return;
  const double velmax = reduce_max_partials(n, part);
  if (threadIdx.x != 0) return;
  gamma_finish(ph, sc, velmax, apply_floor);
}
void launch_gamma(const Launch& L, const Geo& g, const Phys& ph, DevScalars* sc, double* partial, const double* u,
                  const double* v, const double* w, bool apply_floor) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  k_gamma_max<<<gr, b, 0, L.st>>>(g, sc, partial, u, v, w);
  k_gamma_final<<<1, 1024, 0, L.st>>>(ph, sc, (int)(gr.x * gr.y * gr.z), partial, apply_floor ? 1 : 0);
}

// the per-point maximum of chkdt (src/chkdt.f90:47-78)
__device__ __forceinline__ double chkdt_cell(const Geo& g, int i, int j, int k, const double* __restrict__ u,
                                             const double* __restrict__ v, const double* __restrict__ w) {
  const int c = g.h(i, j, k), sx = g.sx, sxy = g.sxy;
  const double dxi = recip_rn(g.dx), dyi = recip_rn(g.dy);
  const double ux = fabs(LD(u, c));
  const double vx = 0.25 * fabs(LD(v, c) + LD(v, c - sx) + LD(v, c + 1) + LD(v, c + 1 - sx));
  const double wx = 0.25 * fabs(LD(w, c) + LD(w, c - sxy) + LD(w, c + 1) + LD(w, c + 1 - sxy));
  const double dtix = ux * dxi + vx * dyi + wx * g.dzfi[k];
  const double uy = 0.25 * fabs(LD(u, c) + LD(u, c + sx) + LD(u, c - 1 + sx) + LD(u, c - 1));
  const double vy = fabs(LD(v, c));
  const double wy = 0.25 * fabs(LD(w, c) + LD(w, c + sx) + LD(w, c + sx - sxy) + LD(w, c - sxy));
  const double dtiy = uy * dxi + vy * dyi + wy * g.dzfi[k];
  const double uz = 0.25 * fabs(LD(u, c) + LD(u, c - 1) + LD(u, c - 1 + sxy) + LD(u, c + sxy));
  const double vz = 0.25 * fabs(LD(v, c) + LD(v, c - sx) + LD(v, c - sx + sxy) + LD(v, c + sxy));
  const double wz = fabs(LD(w, c));
  const double dtiz = uz * dxi + vz * dyi + wz * g.dzci[k];
  return fmax(dtix, fmax(dtiy, dtiz));
}

// chkdt, src/chkdt.f90:15-94
__global__ void k_chkdt_max(Geo g, DevScalars* __restrict__ sc, int only_on_check, double* __restrict__ part,
                            const double* __restrict__ u, const double* __restrict__ v,
                            const double* __restrict__ w) {
  if (HALTED(sc) || (only_on_check && !sc->check_now)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y + 1, k = blockIdx.z + 1;
  double dti = 0.;
  if (i <= g.nx) dti = chkdt_cell(g, i, j, k, u, v, w);
  dti = block_max(dti);
  if (threadIdx.x == 0) part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = dti;
}
// the dt update of src/main.f90:530-551 from the maximum of chkdt
__device__ __forceinline__ void chkdt_finish(const Phys& ph, DevScalars* sc, double dti, int in_loop) {
  double dtipsi;
  if (ph.acdi) {
    dtipsi = sc->gam * sc->seps / (ph.dlmin * ph.dlmin);
    if (dtipsi == 0.) dtipsi = 1.;
  } else {
    dtipsi = dti;
  }
  double dtmax;
  if (!ph.solve_ns) {
    dtmax = fmin(1. / dti, 1. / dtipsi);
  } else {
    const double dtiv = ph.mu_over_rho_max * 2. * (3. / (ph.dlmin * ph.dlmin));
    const double dtik = sqrt(ph.sigma / ph.rho_min / (ph.dlmin * ph.dlmin * ph.dlmin));
    const double dtig = ph.gmax / ph.dlmin;
    dti = 0.5 * (dti + dtiv + sqrt((dti + dtiv) * (dti + dtiv) + 4. * (dtig * dtig + dtik * dtik)));
    if (dti == 0.) dti = 1.;
    dtmax = 1. / dti;
    if (ph.track) dtmax = fmin(dtmax, 1. / dtipsi);
  }
  if (ph.scalar) {  // the scalar's diffusion limit, src/chkdt.f90:88-93
    dti = ph.ka_rhocp_max / (ph.dlmin * ph.dlmin);
    if (dti == 0.) dti = 1.;
    dtmax = fmin(dtmax, 1. / dti);
  }
  sc->dt_cfl = dtmax;
  double dt = fmin(ph.cfl * dtmax, ph.dtmax);
  if (ph.dt_f > 0.) {
    if (ph.dt_f > dt && in_loop) sc->status = CANSFZ_ERR_DT;
    else dt = ph.dt_f;
  }
  sc->dt = dt;
  sc->dti = 1. / dt;
  if (in_loop && dtmax < ph.small) sc->status = CANSFZ_ERR_DT;
}

// completes chkdt and the dt update of src/main.f90:530-551
__global__ void k_chkdt_final(Phys ph, DevScalars* __restrict__ sc, int only_on_check, int in_loop, int n,
                              const double* __restrict__ part) {
  if (HALTED(sc) || (only_on_check && !sc->check_now)) return;
  const double dti = reduce_max_partials(n, part);
  if (threadIdx.x != 0) return;
  chkdt_finish(ph, sc, dti, in_loop);
}
void launch_chkdt(const Launch& L, const Geo& g, const Phys& ph, DevScalars* sc, double* partial, const double* u,
                  const double* v, const double* w, bool only_on_check) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  const int oc = only_on_check ? 1 : 0;
  k_chkdt_max<<<gr, b, 0, L.st>>>(g, sc, oc, partial, u, v, w);
  k_chkdt_final<<<1, 1024, 0, L.st>>>(ph, sc, oc, oc, (int)(gr.x * gr.y * gr.z), partial);
}

// chkdiv, src/chkdiv.f90:15-49: per-block partial sums, max via atomics
__global__ void k_chkdiv_part(Geo g, DevScalars* __restrict__ sc, int only_on_check, double* __restrict__ part,
                              const double* __restrict__ u, const double* __restrict__ v,
                              const double* __restrict__ w) {
  if (HALTED(sc) || (only_on_check && !sc->check_now)) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y + 1, k = blockIdx.z + 1;
  double div = 0.;
  if (i <= g.nx) {
    const int c = g.h(i, j, k);
    div = (LD(w, c) - LD(w, c - g.sxy)) * g.dzfi[k] + (LD(v, c) - LD(v, c - g.sx)) * g.dyi +
          (LD(u, c) - LD(u, c - 1)) * g.dxi;
  }
  const double m = block_max(fabs(div));
  const double s = block_sum(div);
  if (threadIdx.x == 0) {
    const int nb = gridDim.x * gridDim.y * gridDim.z;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    part[bid] = s;
    part[nb + bid] = m;
  }
}
struct SumPartials {
  static __device__ __forceinline__ void run(const Blk& bk, int n, const double* __restrict__ part,
      double* __restrict__ out, DevScalars* __restrict__ sc, int only_on_check) {
    if (HALTED(sc) || (only_on_check && !sc->check_now)) return;
    double s = 0.;
    for (int q = threadIdx.x; q < n; q += blockDim.x) s += part[q];
    s = block_sum(s);
    if (threadIdx.x == 0) *out = s;
  }
};
__global__ void k_sum_partials(int n, const double* __restrict__ part, double* __restrict__ out,
                               DevScalars* __restrict__ sc, int only_on_check) {
  SumPartials::run(blk_here(), n, part, out, sc, only_on_check);
}
__device__ __forceinline__ void chkdiv_finish(double small, DevScalars* sc, double divmax, int only_on_check) {
  sc->divmax = divmax;
  // src/main.f90:552-561, after the dt checks (an earlier dt abort is kept)
  if (only_on_check && sc->status == CANSFZ_OK) {
    if (isnan(sc->divtot)) sc->status = CANSFZ_ERR_NAN;
    else if (sc->divmax > small) sc->status = CANSFZ_ERR_DIVERGENCE;
  }
}
__global__ void k_chkdiv_final(Phys ph, DevScalars* __restrict__ sc, int only_on_check, int n,
                               const double* __restrict__ part) {
  if (HALTED(sc) || (only_on_check && !sc->check_now)) return;
  const double m = reduce_max_partials(n, part + n);
  if (threadIdx.x != 0) return;
  chkdiv_finish(ph.small, sc, m, only_on_check);
}
void launch_chkdiv(const Launch& L, const Geo& g, DevScalars* sc, double* partial, const double* u,
                   const double* v, const double* w, bool only_on_check) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  const int oc = only_on_check ? 1 : 0;
  k_chkdiv_part<<<gr, b, 0, L.st>>>(g, sc, oc, partial, u, v, w);
  kgo<SumPartials, 1024, 1>(L, k_sum_partials, 1, 1024, 0, (int)(gr.x * gr.y * gr.z), partial, &sc->divtot, sc, oc);
  Phys ph{};
  ph.small = CANSFZ_EPS * 1.0e7;
  k_chkdiv_final<<<1, 1024, 0, L.st>>>(ph, sc, oc, (int)(gr.x * gr.y * gr.z), partial);
}

// ---------------------------------------------------------------------------
// End of a step: acdi_set_gamma every step and, on icheck steps, chkdt and
// chkdiv -- one pass over u, v, w.  Blocks walk (j,k) rows with a grid
// stride, threads the points of a row; four partials per block (|u_c|^2
// max, dt^-1 max, divergence sum and |div| max), then one block finishes
// gamma, the dt update and the divergence checks in the reference's order
// (src/main.f90:530-561).  Maxima are order independent; the divergence sum
// (used only for its NaN test) is summed in a fixed order.
// ---------------------------------------------------------------------------
constexpr int kReduceThreads = 256;
struct StepReduce {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, DevScalars* __restrict__ sc, int acdi,
      double* __restrict__ part, const double* __restrict__ u, const double* __restrict__ v,
      const double* __restrict__ w) {
    if (HALTED(sc)) return;
    const bool chk = sc->check_now != 0;
    if (!acdi && !chk) return;
    double velmax = 0., dtimax = 0., divsum = 0., divmax = 0.;
    const int nrows = g.ny * g.nz;
    if (!chk) {
      // Gamma only (every step): R rows per pass, their loads issued together
      constexpr int R = 2;
      for (int i = threadIdx.x + 1; i <= g.nx; i += blockDim.x) {
        for (int r0 = bk.x; r0 < nrows; r0 += R * bk.nx) {
          double u0[R], u1[R], v0[R], v1[R], w0[R], w1[R];
#pragma unroll
          for (int q = 0; q < R; ++q) {
            const int r = r0 + q * bk.nx;
            if (r < nrows) {
              const int c = g.h(i, r % g.ny + 1, r / g.ny + 1);
              u0[q] = LD(u, c);
              u1[q] = LD(u, c - 1);
              v0[q] = LD(v, c);
              v1[q] = LD(v, c - g.sx);
              w0[q] = LD(w, c);
              w1[q] = LD(w, c - g.sxy);
            }
          }
#pragma unroll
          for (int q = 0; q < R; ++q) {
            if (r0 + q * bk.nx >= nrows) break;
            const double uc = 0.5 * (u0[q] + u1[q]);
            const double vc = 0.5 * (v0[q] + v1[q]);
            const double wc = 0.5 * (w0[q] + w1[q]);
            velmax = fmax(velmax, vel2(uc, vc, wc));
          }
        }
      }
    } else {
      for (int r = bk.x; r < nrows; r += bk.nx) {
        const int j = r % g.ny + 1, k = r / g.ny + 1;
        for (int i = threadIdx.x + 1; i <= g.nx; i += blockDim.x) {
          const int c = g.h(i, j, k);
          if (acdi) {
            const double uc = 0.5 * (LD(u, c) + LD(u, c - 1));
            const double vc = 0.5 * (LD(v, c) + LD(v, c - g.sx));
            const double wc = 0.5 * (LD(w, c) + LD(w, c - g.sxy));
            velmax = fmax(velmax, vel2(uc, vc, wc));
          }
          dtimax = fmax(dtimax, chkdt_cell(g, i, j, k, u, v, w));
          const double div = (LD(w, c) - LD(w, c - g.sxy)) * g.dzfi[k] + (LD(v, c) - LD(v, c - g.sx)) * g.dyi +
                             (LD(u, c) - LD(u, c - 1)) * g.dxi;
          divsum += div;
          divmax = fmax(divmax, fabs(div));
        }
      }
    }
    velmax = block_max(velmax);
    dtimax = block_max(dtimax);
    divsum = block_sum(divsum);
    divmax = block_max(divmax);
    if (threadIdx.x == 0) {
      const int nb = bk.nx;
      part[bk.x] = velmax;
      part[nb + bk.x] = dtimax;
      part[2 * nb + bk.x] = divsum;
      part[3 * nb + bk.x] = divmax;
    }
  }
};
__global__ void __launch_bounds__(kReduceThreads) k_step_reduce(Geo g, DevScalars* __restrict__ sc, int acdi,
                                                                double* __restrict__ part,
                                                                const double* __restrict__ u,
                                                                const double* __restrict__ v,
                                                                const double* __restrict__ w) {
  StepReduce::run(blk_here(), g, sc, acdi, part, u, v, w);
}
struct StepReduceFinal {
  static __device__ __forceinline__ void run(const Blk& bk, const Phys& ph, DevScalars* __restrict__ sc, int nb,
      const double* __restrict__ part) {
    if (HALTED(sc)) return;
    const bool chk = sc->check_now != 0;
    if (!ph.acdi && !chk) return;
    const double velmax = reduce_max_partials(nb, part);
    const double dtimax = reduce_max_partials(nb, part + nb);
    double s = 0.;
    for (int q = threadIdx.x; q < nb; q += blockDim.x) s += part[2 * nb + q];
    s = block_sum(s);
    const double divmax = reduce_max_partials(nb, part + 3 * nb);
    if (threadIdx.x != 0) return;
    if (ph.acdi) gamma_finish(ph, sc, velmax, 1);
    if (chk) {
      chkdt_finish(ph, sc, dtimax, 1);
      sc->divtot = s;
      chkdiv_finish(CANSFZ_EPS * 1.0e7, sc, divmax, 1);
    }
  }
};
__global__ void k_step_reduce_final(Phys ph, DevScalars* __restrict__ sc, int nb, const double* __restrict__ part) {
  StepReduceFinal::run(blk_here(), ph, sc, nb, part);
}
void launch_step_reductions(const Launch& L, const Geo& g, const Phys& ph, DevScalars* sc, double* partial,
                            const double* u, const double* v, const double* w) {
  const int nrows = g.ny * g.nz;
  // one wave: four blocks of 256 threads per SM are resident at the
  // kernel's 60 registers (eight, as two waves, left a tail: 0.107 against
  // 0.096 ms at 256^3)
  int nb = (L.nsm > 0 ? L.nsm : 148) * 4;
  if (nb > nrows) nb = nrows;
  kgo<StepReduce, 256, 1>(L, k_step_reduce, nb, kReduceThreads, 0, g, sc, ph.acdi, partial, u, v, w);
  kgo<StepReduceFinal, 1024, 1>(L, k_step_reduce_final, 1, 1024, 0, ph, sc, nb, partial);
}

// bulk_mean_12_stag, src/utils.f90:68-136
struct BulkPart {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const Phys& ph,
      const DevScalars* __restrict__ sc, int idir, const double* __restrict__ gvr, const double* __restrict__ psi,
      double* __restrict__ part) {
    if (HALTED(sc)) return;
    const int i = bk.x * blockDim.x + threadIdx.x + 1;
    const int j = bk.y + 1, k = bk.z + 1;
    double s = 0.;
    if (i <= g.nx) {
      const int c = g.h(i, j, k);
      double pl;
      if (idir == 1) pl = 0.5 * (LD(psi, c + 1) + LD(psi, c));
      else if (idir == 2) pl = 0.5 * (LD(psi, c + g.sx) + LD(psi, c));
      else pl = 0.5 * (LD(psi, c + g.sxy) + LD(psi, c));
      s = (pl * ph.rho12[0] + (1. - pl) * ph.rho12[1]) * gvr[k];
    }
    s = block_sum(s);
    if (threadIdx.x == 0) part[bk.x + bk.nx * (bk.y + bk.ny * bk.z)] = s;
  }
};
__global__ void k_bulk_part(Geo g, Phys ph, const DevScalars* __restrict__ sc, int idir,
                            const double* __restrict__ gvr, const double* __restrict__ psi,
                            double* __restrict__ part) {
  BulkPart::run(blk_here(), g, ph, sc, idir, gvr, psi, part);
}
void launch_bulk_mean(const Launch& L, const Geo& g, const Phys& ph, DevScalars* sc, double* partial, int idir,
                      const double* gvr, const double* psi) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  kgo<BulkPart, 128, 1>(L, k_bulk_part, gr, b, 0, g, ph, sc, idir, gvr, psi, partial);
  kgo<SumPartials, 1024, 1>(L, k_sum_partials, 1, 1024, 0, (int)(gr.x * gr.y * gr.z), partial, &sc->rho_av[idir - 1],
      sc, 0);
}

// cmpt_mean_mass, src/output.f90:759-790
__global__ void k_mass_part(Geo g, Phys ph, const double* __restrict__ psi, double* __restrict__ part) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  const int j = blockIdx.y + 1, k = blockIdx.z + 1;
  double m1 = 0., m2 = 0.;
  if (i <= g.nx) {
    const double vcell = g.dx * g.dy * g.dzf[k];
    const double ps = LD(psi, g.h(i, j, k));
    m1 = ph.rho12[0] * ps * vcell;
    m2 = ph.rho12[1] * (1. - ps) * vcell;
  }
  m1 = block_sum(m1);
  m2 = block_sum(m2);
  if (threadIdx.x == 0) {
    const int nb = gridDim.x * gridDim.y * gridDim.z;
    const int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    part[bid] = m1;
    part[nb + bid] = m2;
  }
}
__global__ void k_mass_final(int nb, const double* __restrict__ part, DevScalars* __restrict__ sc, double vol) {
  double s1 = 0., s2 = 0.;
  for (int q = threadIdx.x; q < nb; q += blockDim.x) { s1 += part[q]; s2 += part[nb + q]; }
  s1 = block_sum(s1);
  s2 = block_sum(s2);
  if (threadIdx.x == 0) { sc->mass12[0] = s1 / vol; sc->mass12[1] = s2 / vol; }
}
void launch_mass(const Launch& L, const Geo& g, const Phys& ph, DevScalars* sc, double* partial, const double* psi,
                 double vol) {
  dim3 b = blk_interior(g), gr = grd_interior(g, b);
  k_mass_part<<<gr, b, 0, L.st>>>(g, ph, psi, partial);
  k_mass_final<<<1, 1024, 0, L.st>>>((int)(gr.x * gr.y * gr.z), partial, sc, vol);
}

// ---------------------------------------------------------------------------
// step bookkeeping, src/main.f90:414-425 and :515-529
// ---------------------------------------------------------------------------
struct StepBegin {
  static __device__ __forceinline__ void run(const Blk& bk, DevScalars* sc, int icheck) {
    if (sc->status != CANSFZ_OK) sc->halted = 1;
    if (sc->halted) return;
    sc->istep = sc->istep + 1;
    sc->time = sc->time + sc->dt;
    const double dt_r = sc->dt / sc->dto;
    sc->dt_r = dt_r;
    sc->tm1 = 1. + 0.5 * dt_r;
    sc->tm2 = -0.5 * dt_r;
    sc->f1 = sc->tm1 * sc->dt;
    sc->f2 = sc->tm2 * sc->dt;
    sc->f12 = sc->f1 + sc->f2;
    sc->dti = 1. / sc->dt;
    sc->check_now = (icheck > 0 && (sc->istep % icheck) == 0) ? 1 : 0;
  }
};
__global__ void k_step_begin(DevScalars* sc, int icheck) {
  StepBegin::run(blk_here(), sc, icheck);
}
void launch_step_begin(const Launch& L, DevScalars* sc, int icheck) {
  kgo<StepBegin, 1, 1>(L, k_step_begin, 1, 1, 0, sc, icheck);
}
struct StepEnd {
  static __device__ __forceinline__ void run(const Blk& bk, DevScalars* sc) {
    if (sc->halted) return;
    sc->dto = sc->dt;
    sc->first_rk = 0;
    sc->first_rk2fl = 0;
    sc->first_scal = 0;
  }
};
__global__ void k_step_end(DevScalars* sc) {
  StepEnd::run(blk_here(), sc);
}
void launch_step_end(const Launch& L, const Phys& ph, DevScalars* sc) {
  (void)ph;
  kgo<StepEnd, 1, 1>(L, k_step_end, 1, 1, 0, sc);
}

}  // namespace cansfz
