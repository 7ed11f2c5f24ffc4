// The z-marching momentum tile kernel: the whole of rk (src/rk.f90:16-131)
// in one pass per step, with its compile-time variants (Boussinesq buoyancy,
// balanced capillary split).  It shares the tile helpers of k_tiles.cuh with
// the phase-field tiles of k_tiles.cu.
#include <cstring>

#include "batch.cuh"
#include "k_tiles.cuh"
#include "tma.cuh"

namespace cansfz {

#define HALTED(sc) ((sc) != nullptr && (sc)->halted)

// ---------------------------------------------------------------------------
// Momentum: the whole of rk (src/rk.f90:16-131) per u/v/w point -- mom_xyz_ad
// (src/mom.f90:505-851, default diffusion branch), the first AB2 update with
// the density ratio, mom_xyz_oth (src/mom.f90:912-1038), the second update.
//
// u, v, w, psi and the three phase fluxes are staged per plane (k and k+1;
// k+2 in flight).  Every plane-(k-1) value a point needs is one that the
// same thread read at level k-1 from plane k with the same x/y offset, so it
// is carried in registers and the ring never needs three planes at once.
// psio, p, po and kappa enter only at (0,0,0), (1,0,0), (0,1,0), (0,0,1):
// read through the read-only cache, the own-column value carried upwards.
// Those loads and the history reads are issued at the top of each level, so
// that the stencil arithmetic hides their latency, and the next level's
// history lines are prefetched into L2 meanwhile; holding them takes up to
// 128 registers; the kernel runs on 32x4 tiles (128 threads), four blocks per
// SM, so that a block's two barriers per level couple four warps, not eight.
// The expressions are those of the per-point kernels (same operand order).
// The whole update is evaluated in FP64.  TI is the storage type of the phase
// fluxes, the curvature and the AB2 histories: double in the drop-in, float
// in the mixed form (an FP32 RHS was 3% faster and left a 1e-6 pressure
// error; with the RHS in FP64 the mixed form's error is 5e-9).
// OPT selects two compile-time variants of mom_xyz_oth: kMomBuoy adds the
// Boussinesq buoyancy of the scalar s (_SCALAR with _BOUSSINESQ_BUOYANCY,
// src/mom.f90:1017-1024) after the pressure terms; kMomBal is the balanced
// capillary split (_BALANCED_CAPILLARY_PRESSURE_SPLIT, src/mom.f90:982-1032):
// the surface-tension force leaves the right-hand side and is subtracted from
// the pressure gradient, its extrapolated value (1+dt_r)*surf_n - dt_r*surf_o
// from the extrapolated one, and the new force goes to the history slot.
// ---------------------------------------------------------------------------
namespace {
// the plane slot pitch: with TMA staging (and for the FP64 drop-in) the
// ring slots start on 128-byte boundaries, where the TMA plane copies land
template <typename TI, int TYV, int STG>
constexpr int mom_pitch() {
  using SH = tile::Shape<TYV>;
  return (sizeof(TI) == 8 || STG) ? (SH::PXY + 15) / 16 * 16 : SH::PXY;
}
// STG: the planes are staged by TMA, and then psio, p, po and kappa as well,
// so that their +x, +y, +z neighbours come from shared memory; otherwise
// seven fields by element copies and those four through the read-only cache.
// With TI = float (the mixed form) only the FP64 fields can be TMA copies: a
// tensor map needs row strides that are multiples of 16 bytes, and an FP32
// halo row of nx + 2 values is not one in general; the three FP32 fluxes
// and kappa are then element copies into the ring beside them.
template <typename TI, int STG>
constexpr int mom_extra() { return STG ? 4 : 0; }
template <typename TI, int TYV, int STG>
constexpr size_t mom_smem() {
  using namespace tile;
  using SH = Shape<TYV>;
  constexpr int SP = mom_pitch<TI, TYV, STG>(), NSLOT = SH::NSLOT;
  // FP64 drop-in: u v w c | fx fy fz | psio p po kappa; mixed form with
  // STG: u v w c | psio p po (FP64) | fx fy fz kappa (FP32); else u v w c | fx fy fz
  constexpr size_t nd = 4 + (sizeof(TI) == 8 ? mom_extra<TI, STG>() : (STG ? 3 : 0));
  constexpr size_t nt = 3 + ((sizeof(TI) != 8 && STG) ? 1 : 0);
  return (size_t)NSLOT * SP * (nd * sizeof(double) + nt * sizeof(TI)) + NSLOT * sizeof(uint64_t);
}
}  // namespace

enum { kMomBuoy = 1, kMomBal = 2 };
// blocks per SM that the momentum tile's z split aims at: shorter blocks than
// the phase-field tiles' (0.711 -> 0.683 ms at 256^3 against 24)
constexpr int kMomSlots = 48;

template <typename TI, int TYV, int OPT, int STG>
struct MomentumTile {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const Phys& ph,
      const DevScalars* __restrict__ sc, int kz, const double* __restrict__ u, const double* __restrict__ v,
      const double* __restrict__ w, const double* __restrict__ psi, const double* __restrict__ psio,
      const TI* __restrict__ fx, const TI* __restrict__ fy, const TI* __restrict__ fz, const double* __restrict__ p,
      const double* __restrict__ po, const TI* __restrict__ kappa, const double* __restrict__ s,
      const SurfSplit& sp, TI* __restrict__ duo, TI* __restrict__ dvo, TI* __restrict__ dwo, double* __restrict__ uo,
      double* __restrict__ vo, double* __restrict__ wo, const HaloMaps& maps, int wrap) {
    constexpr bool BUOY = (OPT & kMomBuoy) != 0, BAL = (OPT & kMomBal) != 0;
    using namespace tile;
    using SH = Shape<TYV>;
    constexpr int TX = SH::TX, TY = SH::TY, NT = SH::NT, PX = SH::PX, PXY = SH::PXY, NSLOT = SH::NSLOT;
    constexpr int SP = mom_pitch<TI, TYV, STG>();
    // TMA plane copies for the staged FP64 fields; element copies for the
    // rest (all fields without STG; the FP32 fluxes and kappa of the mixed
    // form with it).  A tensor map must sit on a 64-byte boundary.
    constexpr bool tmaon = STG != 0;
    constexpr bool mixstg = STG != 0 && sizeof(TI) != 8;  // FP32 planes beside the TMA ones
    (void)TY;
    typedef double T;  // the RHS in FP64 for both storage types
    extern __shared__ __align__(128) unsigned char smem[];
    double* s_u = reinterpret_cast<double*>(smem);  // each [NSLOT][SP]
    double* s_v = s_u + NSLOT * SP;
    double* s_w = s_v + NSLOT * SP;
    double* s_c = s_w + NSLOT * SP;
    constexpr int NX4 = mom_extra<TI, STG>();  // staged psio, p, po, kappa
    // mixed form with STG: psio, p, po (FP64) follow c, then fx fy fz kappa
    TI* s_fx = mixstg ? reinterpret_cast<TI*>(s_c + 4 * NSLOT * SP) : reinterpret_cast<TI*>(s_c + NSLOT * SP);
    TI* s_fy = s_fx + NSLOT * SP;
    TI* s_fz = s_fy + NSLOT * SP;
    TI* s_kf = s_fz + NSLOT * SP;  // kappa, mixed form with STG only
    double* s_ps = mixstg ? s_c + NSLOT * SP : reinterpret_cast<double*>(s_fz + NSLOT * SP);  // [NX4][NSLOT][SP]
    uint64_t* s_bar = mixstg ? reinterpret_cast<uint64_t*>(s_kf + NSLOT * SP)
                             : reinterpret_cast<uint64_t*>(s_ps + NX4 * NSLOT * SP);  // [NSLOT]
    if (HALTED(sc)) return;
    if (tmaon && (reinterpret_cast<uintptr_t>(&maps) & 63) != 0) {
      // a tensor map must sit on a 64-byte boundary (the host aligns them)
      if (threadIdx.x == 0 && threadIdx.y == 0) {
        DevScalars* scw = const_cast<DevScalars*>(sc);
        atomicCAS(&scw->status, CANSFZ_OK, CANSFZ_ERR_ARG);
        scw->halted = 1;
      }
      return;
    }
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
    const int i0 = bk.x * TX + 1, j0 = bk.y * TY + 1;
    const int kb = bk.z * kz + 1, ke = min(kb + kz - 1, g.nz);
    const int sx = g.sx, sxy = g.sxy;
    if (tmaon) {
      if (tid == 0) {
        for (int q = 0; q < NSLOT; ++q) tma::bar_init(s_bar + q, 1);
        tma::bar_init_fence();
      }
      __syncthreads();
    }
    // plane kk lives in ring slot (kk - kb) % NSLOT; its TMA fill is that
    // slot's ((kk - kb) / NSLOT)-th, which fixes the mbarrier phase
    auto slot = [&](int kk) { return (kk - kb) % NSLOT; };
    auto phase = [&](int kk) { return (uint32_t)(((kk - kb) / NSLOT) & 1); };

    int issued = kb - 1;  // the last plane whose copies were issued
    auto issue = [&](int kk) {
      const int o = slot(kk) * SP;
      if (tmaon) {
        issued = kk;
        if (tid == 0) {
          uint64_t* bar = s_bar + slot(kk);
          if constexpr (!mixstg) {
            constexpr int NF = 7 + NX4;
            tma::bar_expect_tx(bar, (uint32_t)NF * PXY * 8u);
            double* dst[11] = {s_u + o, s_v + o, s_w + o, s_c + o, reinterpret_cast<double*>(s_fx + o),
                               reinterpret_cast<double*>(s_fy + o), reinterpret_cast<double*>(s_fz + o),
                               s_ps + o, s_ps + NSLOT * SP + o, s_ps + 2 * NSLOT * SP + o, s_ps + 3 * NSLOT * SP + o};
#pragma unroll
            for (int f = 0; f < NF; ++f) tma::load_3d(dst[f], &maps.m[f], i0 - 1, j0 - 1, kk, bar);
          } else {
            // the seven FP64 fields: maps 0-3 (u v w psi) and 7-9 (psio p po)
            tma::bar_expect_tx(bar, 7u * PXY * 8u);
            double* dst[7] = {s_u + o, s_v + o, s_w + o, s_c + o, s_ps + o, s_ps + NSLOT * SP + o,
                              s_ps + 2 * NSLOT * SP + o};
            const int mi[7] = {0, 1, 2, 3, 7, 8, 9};
#pragma unroll
            for (int f = 0; f < 7; ++f) tma::load_3d(dst[f], &maps.m[mi[f]], i0 - 1, j0 - 1, kk, bar);
          }
        }
        if constexpr (mixstg) {
          for (int q = tid; q < PXY; q += NT) {
            int h;
            const bool ok = plane_cell<PX>(g, i0, j0, kk, q, &h);
            const int hh = ok ? h : 0;
            cp_async(s_fx + o + q, fx + hh, ok);
            cp_async(s_fy + o + q, fy + hh, ok);
            cp_async(s_fz + o + q, fz + hh, ok);
            cp_async(s_kf + o + q, kappa + hh, ok);
          }
          cp_commit();
        }
        return;
      }
      for (int q = tid; q < PXY; q += NT) {
        int h;
        const bool ok = plane_cell<PX>(g, i0, j0, kk, q, &h);
        const int hh = ok ? h : 0;
        cp_async(s_u + o + q, u + hh, ok);
        cp_async(s_v + o + q, v + hh, ok);
        cp_async(s_w + o + q, w + hh, ok);
        cp_async(s_c + o + q, psi + hh, ok);
        cp_async(s_fx + o + q, fx + hh, ok);
        cp_async(s_fy + o + q, fy + hh, ok);
        cp_async(s_fz + o + q, fz + hh, ok);
      }
      cp_commit();
    };

    const int i = i0 + tx, j = j0 + ty;
    const bool act = i <= g.nx && j <= g.ny;
    const int qc = (tx + 1) + PX * (ty + 1);
    const T rho = (T)ph.rho12[1], drho = (T)(ph.rho12[0] - ph.rho12[1]);
    const T mu = (T)ph.mu12[1], dmu = (T)(ph.mu12[0] - ph.mu12[1]);
    const T dxi = (T)g.dxi, dyi = (T)g.dyi;
    const double rhod = ph.rho12[1], drhod = ph.rho12[0] - ph.rho12[1];
    const double dt_r = sc->dt_r, f1 = sc->f1, f2 = sc->f2, f12 = sc->f12;
    const bool first = sc->first_rk;

    // values of plane k-1 carried from the level below
    T u_ccm = T(0), v_ccm = T(0), w_ccm = T(0), w_pcm = T(0), w_cpm = T(0);
    T c_ccm = T(0), c_pcm = T(0), c_cpm = T(0), flx_z_ccm = T(0), flx_z_pcm = T(0), flx_z_cpm = T(0);
    // own-column values of the four-point fields at the current level
    double p_c = 0., po_c = 0., pso_c = 0., k_c = 0.;
    if (act) {
      const int cm = g.h(i, j, kb - 1);
      u_ccm = (T)__ldg(u + cm);
      v_ccm = (T)__ldg(v + cm);
      w_ccm = (T)__ldg(w + cm);
      w_pcm = (T)__ldg(w + cm + 1);
      w_cpm = (T)__ldg(w + cm + sx);
      c_ccm = (T)__ldg(psi + cm);
      c_pcm = (T)__ldg(psi + cm + 1);
      c_cpm = (T)__ldg(psi + cm + sx);
      flx_z_ccm = rho * w_ccm + drho * __ldg(fz + cm);
      flx_z_pcm = rho * w_pcm + drho * __ldg(fz + cm + 1);
      flx_z_cpm = rho * w_cpm + drho * __ldg(fz + cm + sx);
      const int c0 = cm + sxy;
      p_c = __ldg(p + c0);
      po_c = __ldg(po + c0);
      pso_c = __ldg(psio + c0);
      k_c = (double)__ldg(kappa + c0);
    }

    issue(kb);
    issue(kb + 1);
    bool fail = false;
    for (int k = kb; k <= ke; ++k) {
      if (k + 2 <= ke + 1) issue(k + 2);
      else if (!tmaon || mixstg) cp_commit();
      if (tmaon) {
        // planes k and k+1 are in (each thread waits for the copies itself)
        if (!tma::bar_wait(s_bar + slot(k), phase(k)) || !tma::bar_wait(s_bar + slot(k + 1), phase(k + 1)))
          fail = true;
        if constexpr (mixstg) {
          cp_wait<1>();
          __syncthreads();  // every thread's element copies of planes k and k+1 are in
        }
      } else {
        cp_wait<1>();
        __syncthreads();  // planes k and k+1 are in; every thread is done with level k-1
      }
      if (act && !fail) {
        const int o0 = slot(k) * SP + qc, o1 = slot(k + 1) * SP + qc;
#define PU(s, a, b) ((T)s_u[o##s + (a) + PX * (b)])
#define PV(s, a, b) ((T)s_v[o##s + (a) + PX * (b)])
#define PW(s, a, b) ((T)s_w[o##s + (a) + PX * (b)])
#define PC(s, a, b) ((T)s_c[o##s + (a) + PX * (b)])
#define FLX(s, a, b) (rho * PU(s, a, b) + drho * s_fx[o##s + (a) + PX * (b)])
#define FLY(s, a, b) (rho * PV(s, a, b) + drho * s_fy[o##s + (a) + PX * (b)])
#define FLZ(s, a, b) (rho * PW(s, a, b) + drho * s_fz[o##s + (a) + PX * (b)])
        // the level's loads from global memory, issued before the stencil
        // arithmetic that hides their latency
        const int c = g.h(i, j, k), t = g.t(i, j, k);
        double pso_x, pso_y, pso_z, p_x, p_y, p_z, po_x, po_y, po_z, k_x, k_y, k_z;
        if constexpr (NX4 > 0) {
          // from the staged planes k and k+1 (own points too: the carried
          // values below are those of the element-copy path)
          const double* sps = s_ps;
          const double* sp_ = s_ps + NSLOT * SP;
          const double* spo = s_ps + 2 * NSLOT * SP;
          const double* sk = s_ps + 3 * NSLOT * SP;
          pso_c = sps[o0]; pso_x = sps[o0 + 1]; pso_y = sps[o0 + PX]; pso_z = sps[o1];
          p_c = sp_[o0]; p_x = sp_[o0 + 1]; p_y = sp_[o0 + PX]; p_z = sp_[o1];
          po_c = spo[o0]; po_x = spo[o0 + 1]; po_y = spo[o0 + PX]; po_z = spo[o1];
          if constexpr (mixstg) {
            k_c = (double)s_kf[o0]; k_x = (double)s_kf[o0 + 1]; k_y = (double)s_kf[o0 + PX]; k_z = (double)s_kf[o1];
          } else {
            k_c = sk[o0]; k_x = sk[o0 + 1]; k_y = sk[o0 + PX]; k_z = sk[o1];
          }
        } else {
          if (k + 1 < ke && (tx & 15) == 0) {
            // the +z neighbours two levels up into L2: they are fresh DRAM
            // reads at the level that needs them (mixed form: 0.743 -> 0.697
            // ms at 256^3)
            const int c2 = c + 2 * sxy;
            asm volatile("prefetch.global.L2 [%0];" ::"l"(psio + c2));
            asm volatile("prefetch.global.L2 [%0];" ::"l"(p + c2));
            asm volatile("prefetch.global.L2 [%0];" ::"l"(po + c2));
            asm volatile("prefetch.global.L2 [%0];" ::"l"(kappa + c2));
          }
          pso_x = __ldg(psio + c + 1); pso_y = __ldg(psio + c + sx); pso_z = __ldg(psio + c + sxy);
          p_x = __ldg(p + c + 1); p_y = __ldg(p + c + sx); p_z = __ldg(p + c + sxy);
          po_x = __ldg(po + c + 1); po_y = __ldg(po + c + sx); po_z = __ldg(po + c + sxy);
          k_x = (double)__ldg(kappa + c + 1); k_y = (double)__ldg(kappa + c + sx);
          k_z = (double)__ldg(kappa + c + sxy);
        }
        const double hu0 = first ? 0. : (double)duo[t], hv0 = first ? 0. : (double)dvo[t],
                     hw0 = first ? 0. : (double)dwo[t];
        if (!first && k < ke && (tx & 15) == 0) {
          // the next level's history lines into L2 while this level computes
          // (one prefetch per 128-byte line of a warp's 32 points): the
          // history reads, the loads that the planes staged in shared memory
          // leave, then come from L2 (0.62 -> 0.57 ms at 256^3)
          const size_t tn = (size_t)t + (size_t)g.nx * g.ny;
          asm volatile("prefetch.global.L2 [%0];" ::"l"(duo + tn));
          asm volatile("prefetch.global.L2 [%0];" ::"l"(dvo + tn));
          asm volatile("prefetch.global.L2 [%0];" ::"l"(dwo + tn));
        }
        double sxn = 0., syn = 0., szn = 0., sxo = 0., syo = 0., szo = 0.;
        if (BAL) {
          sxn = sp.n[0][t]; syn = sp.n[1][t]; szn = sp.n[2][t];
          sxo = sp.o[0][t]; syo = sp.o[1][t]; szo = sp.o[2][t];
        }
        const T dzci_c = (T)g.dzci[k], dzci_m = (T)g.dzci[k - 1], dzfi_c = (T)g.dzfi[k], dzfi_p = (T)g.dzfi[k + 1];
        // the three components one after another, each reading its stencil
        // from shared memory, so that few values are live at a time
        T dudt_aux, dvdt_aux, dwdt_aux;
        {
          const T u_ccc = PU(0, 0, 0), u_pcc = PU(0, 1, 0), u_mcc = PU(0, -1, 0), u_cpc = PU(0, 0, 1),
                  u_cmc = PU(0, 0, -1), u_ccp = PU(1, 0, 0);
          const T flx_x_ccc = FLX(0, 0, 0);
          const T uuip = T(0.25) * (FLX(0, 1, 0) + flx_x_ccc) * (u_ccc + u_pcc);
          const T uuim = T(0.25) * (FLX(0, -1, 0) + flx_x_ccc) * (u_ccc + u_mcc);
          const T vujp = T(0.25) * (FLY(0, 1, 0) + FLY(0, 0, 0)) * (u_ccc + u_cpc);
          const T vujm = T(0.25) * (FLY(0, 1, -1) + FLY(0, 0, -1)) * (u_ccc + u_cmc);
          const T wukp = T(0.25) * (FLZ(0, 1, 0) + FLZ(0, 0, 0)) * (u_ccc + u_ccp);
          const T wukm = T(0.25) * (flx_z_pcm + flx_z_ccm) * (u_ccc + u_ccm);
          dudt_aux = dxi * (-uuip + uuim) + dyi * (-vujp + vujm) + dzfi_c * (-wukp + wukm);
          const T c_ccc = PC(0, 0, 0), c_pcc = PC(0, 1, 0);
          const T dudxp = (u_pcc - u_ccc) * dxi, dudxm = (u_ccc - u_mcc) * dxi;
          const T dvdxp = (PV(0, 1, 0) - PV(0, 0, 0)) * dxi, dvdxm = (PV(0, 1, -1) - PV(0, 0, -1)) * dxi;
          const T dudyp = (u_cpc - u_ccc) * dyi, dudym = (u_ccc - u_cmc) * dyi;
          const T dudzp = (u_ccp - u_ccc) * dzci_c, dudzm = (u_ccc - u_ccm) * dzci_m;
          const T dwdxp = (PW(0, 1, 0) - PW(0, 0, 0)) * dxi, dwdxm = (w_pcm - w_ccm) * dxi;
          const T muxp = mu + dmu * c_pcc, muxm = mu + dmu * c_ccc;
          const T muyp = mu + dmu * T(0.25) * (c_ccc + PC(0, 0, 1) + PC(0, 1, 1) + c_pcc);
          const T muym = mu + dmu * T(0.25) * (c_ccc + PC(0, 0, -1) + PC(0, 1, -1) + c_pcc);
          const T muzp = mu + dmu * T(0.25) * (c_ccc + c_pcc + PC(1, 0, 0) + PC(1, 1, 0));
          const T muzm = mu + dmu * T(0.25) * (c_ccc + c_pcc + c_ccm + c_pcm);
          dudt_aux = dudt_aux + dxi * ((dudxp + dudxp) * muxp - (dudxm + dudxm) * muxm) +
                     dyi * ((dudyp + dvdxp) * muyp - (dudym + dvdxm) * muym) +
                     dzfi_c * ((dudzp + dwdxp) * muzp - (dudzm + dwdxm) * muzm);
        }
        {
          const T v_ccc = PV(0, 0, 0), v_pcc = PV(0, 1, 0), v_mcc = PV(0, -1, 0), v_cpc = PV(0, 0, 1),
                  v_cmc = PV(0, 0, -1), v_ccp = PV(1, 0, 0);
          const T flx_y_ccc = FLY(0, 0, 0);
          const T uvip = T(0.25) * (FLX(0, 0, 0) + FLX(0, 0, 1)) * (v_ccc + v_pcc);
          const T uvim = T(0.25) * (FLX(0, -1, 0) + FLX(0, -1, 1)) * (v_ccc + v_mcc);
          const T vvjp = T(0.25) * (flx_y_ccc + FLY(0, 0, 1)) * (v_ccc + v_cpc);
          const T vvjm = T(0.25) * (flx_y_ccc + FLY(0, 0, -1)) * (v_ccc + v_cmc);
          const T wvkp = T(0.25) * (FLZ(0, 0, 0) + FLZ(0, 0, 1)) * (v_ccc + v_ccp);
          const T wvkm = T(0.25) * (flx_z_ccm + flx_z_cpm) * (v_ccc + v_ccm);
          dvdt_aux = dxi * (-uvip + uvim) + dyi * (-vvjp + vvjm) + dzfi_c * (-wvkp + wvkm);
          const T c_ccc = PC(0, 0, 0), c_cpc = PC(0, 0, 1);
          const T dvdxp = (v_pcc - v_ccc) * dxi, dvdxm = (v_ccc - v_mcc) * dxi;
          const T dudyp = (PU(0, 0, 1) - PU(0, 0, 0)) * dyi, dudym = (PU(0, -1, 1) - PU(0, -1, 0)) * dyi;
          const T dvdyp = (v_cpc - v_ccc) * dyi, dvdym = (v_ccc - v_cmc) * dyi;
          const T dvdzp = (v_ccp - v_ccc) * dzci_c, dvdzm = (v_ccc - v_ccm) * dzci_m;
          const T dwdyp = (PW(0, 0, 1) - PW(0, 0, 0)) * dyi, dwdym = (w_cpm - w_ccm) * dyi;
          const T muxp = mu + dmu * T(0.25) * (c_ccc + PC(0, 1, 0) + PC(0, 1, 1) + c_cpc);
          const T muxm = mu + dmu * T(0.25) * (c_ccc + PC(0, -1, 0) + PC(0, -1, 1) + c_cpc);
          const T muyp = mu + dmu * c_cpc, muym = mu + dmu * c_ccc;
          const T muzp = mu + dmu * T(0.25) * (c_ccc + c_cpc + PC(1, 0, 1) + PC(1, 0, 0));
          const T muzm = mu + dmu * T(0.25) * (c_ccc + c_cpc + c_cpm + c_ccm);
          dvdt_aux = dvdt_aux + dxi * ((dvdxp + dudyp) * muxp - (dvdxm + dudym) * muxm) +
                     dyi * ((dvdyp + dvdyp) * muyp - (dvdym + dvdym) * muym) +
                     dzfi_c * ((dvdzp + dwdyp) * muzp - (dvdzm + dwdym) * muzm);
        }
        {
          const T w_ccc = PW(0, 0, 0), w_pcc = PW(0, 1, 0), w_mcc = PW(0, -1, 0), w_cpc = PW(0, 0, 1),
                  w_cmc = PW(0, 0, -1), w_ccp = PW(1, 0, 0);
          const T flx_z_ccc = FLZ(0, 0, 0);
          const T uwip = T(0.25) * (FLX(0, 0, 0) + FLX(1, 0, 0)) * (w_ccc + w_pcc);
          const T uwim = T(0.25) * (FLX(0, -1, 0) + FLX(1, -1, 0)) * (w_ccc + w_mcc);
          const T vwjp = T(0.25) * (FLY(0, 0, 0) + FLY(1, 0, 0)) * (w_ccc + w_cpc);
          const T vwjm = T(0.25) * (FLY(0, 0, -1) + FLY(1, 0, -1)) * (w_ccc + w_cmc);
          const T wwkp = T(0.25) * (flx_z_ccc + FLZ(1, 0, 0)) * (w_ccc + w_ccp);
          const T wwkm = T(0.25) * (flx_z_ccc + flx_z_ccm) * (w_ccc + w_ccm);
          dwdt_aux = dxi * (-uwip + uwim) + dyi * (-vwjp + vwjm) + dzci_c * (-wwkp + wwkm);
          const T c_ccc = PC(0, 0, 0), c_ccp = PC(1, 0, 0);
          const T dwdxp = (w_pcc - w_ccc) * dxi, dwdxm = (w_ccc - w_mcc) * dxi;
          const T dudzp = (PU(1, 0, 0) - PU(0, 0, 0)) * dzci_c, dudzm = (PU(1, -1, 0) - PU(0, -1, 0)) * dzci_c;
          const T dwdyp = (w_cpc - w_ccc) * dyi, dwdym = (w_ccc - w_cmc) * dyi;
          const T dvdzp = (PV(1, 0, 0) - PV(0, 0, 0)) * dzci_c, dvdzm = (PV(1, 0, -1) - PV(0, 0, -1)) * dzci_c;
          const T dwdzp = (w_ccp - w_ccc) * dzfi_p, dwdzm = (w_ccc - w_ccm) * dzfi_c;
          const T muxp = mu + dmu * T(0.25) * (c_ccc + PC(0, 1, 0) + c_ccp + PC(1, 1, 0));
          const T muxm = mu + dmu * T(0.25) * (c_ccc + PC(0, -1, 0) + c_ccp + PC(1, -1, 0));
          const T muyp = mu + dmu * T(0.25) * (c_ccc + PC(0, 0, 1) + c_ccp + PC(1, 0, 1));
          const T muym = mu + dmu * T(0.25) * (c_ccc + PC(0, 0, -1) + c_ccp + PC(1, 0, -1));
          const T muzp = mu + dmu * c_ccp, muzm = mu + dmu * c_ccc;
          dwdt_aux = dwdt_aux + dxi * ((dwdxp + dudzp) * muxp - (dwdxm + dudzm) * muxm) +
                     dyi * ((dwdyp + dvdzp) * muyp - (dwdym + dvdzm) * muym) +
                     dzci_c * ((dwdzp + dwdzp) * muzp - (dwdzm + dwdzm) * muzm);
        }
        // first AB2 update with the density ratio (src/rk.f90:86-101), FP64
        const double ps_c = s_c[o0], ps_x = s_c[o0 + 1], ps_y = s_c[o0 + PX], ps_z = s_c[o1];
        const double rhox_n = rhod + drhod * 0.5 * (pso_c + pso_x);
        const double rhoy_n = rhod + drhod * 0.5 * (pso_c + pso_y);
        const double rhoz_n = rhod + drhod * 0.5 * (pso_c + pso_z);
        const double rhox_p = rhod + drhod * 0.5 * (ps_c + ps_x);
        const double rhoy_p = rhod + drhod * 0.5 * (ps_c + ps_y);
        const double rhoz_p = rhod + drhod * 0.5 * (ps_c + ps_z);
        const double Ru = (double)dudt_aux, Rv = (double)dvdt_aux, Rw = (double)dwdt_aux;
        const double Ruo = first ? Ru : hu0, Rvo = first ? Rv : hv0, Rwo = first ? Rw : hw0;
        const double irx = recip_rn(rhox_p), iry = recip_rn(rhoy_p), irz = recip_rn(rhoz_p);
        const double un = s_u[o0] * rhox_n * irx + (f1 * Ru + f2 * Ruo) * irx;
        const double vn = s_v[o0] * rhoy_n * iry + (f1 * Rv + f2 * Rvo) * iry;
        const double wn = s_w[o0] * rhoz_n * irz + (f1 * Rw + f2 * Rwo) * irz;
        duo[t] = dudt_aux;
        dvo[t] = dvdt_aux;
        dwo[t] = dwdt_aux;
        // mom_xyz_oth with pn = p (src/mom.f90:912-1038), FP64
        const double q_ccc = (1. + dt_r) * p_c - dt_r * po_c;
        const double q_pcc = (1. + dt_r) * p_x - dt_r * po_x;
        const double q_cpc = (1. + dt_r) * p_y - dt_r * po_y;
        const double q_ccp = (1. + dt_r) * p_z - dt_r * po_z;
        const double psixp = 0.5 * (ps_x + ps_c), psiyp = 0.5 * (ps_y + ps_c), psizp = 0.5 * (ps_z + ps_c);
        const double rhoxp = rhod + drhod * psixp, rhoyp = rhod + drhod * psiyp, rhozp = rhod + drhod * psizp;
        const double dxid = g.dxi, dyid = g.dyi, dzcid = g.dzci[k];
        const double dpdx = (p_x - p_c) * dxid, dpdy = (p_y - p_c) * dyid, dpdz = (p_z - p_c) * dzcid;
        double sdu = ph.bforce[0] + (rhoxp - sc->rho_av[0]) * ph.gacc[0];
        double sdv = ph.bforce[1] + (rhoyp - sc->rho_av[1]) * ph.gacc[1];
        double sdw = ph.bforce[2] + (rhozp - sc->rho_av[2]) * ph.gacc[2];
        double skappaxp = 0.5 * (k_x + k_c) * ph.surf_factor;
        double skappayp = 0.5 * (k_y + k_c) * ph.surf_factor;
        double skappazp = 0.5 * (k_z + k_c) * ph.surf_factor;
        if (ph.brackbill) {
          skappaxp = skappaxp * rhoxp;
          skappayp = skappayp * rhoyp;
          skappazp = skappazp * rhozp;
        }
        const double surfx = skappaxp * (ps_x - ps_c) * dxid;
        const double surfy = skappayp * (ps_y - ps_c) * dyid;
        const double surfz = skappazp * (ps_z - ps_c) * dzcid;
        double dpdx_e = (q_pcc - q_ccc) * dxid, dpdy_e = (q_cpc - q_ccc) * dyid, dpdz_e = (q_ccp - q_ccc) * dzcid;
        double dpx = dpdx, dpy = dpdy, dpz = dpdz;
        if (BAL) {
          const double sxe = (1. + dt_r) * sxn - dt_r * sxo;
          const double sye = (1. + dt_r) * syn - dt_r * syo;
          const double sze = (1. + dt_r) * szn - dt_r * szo;
          dpx = dpx - surfx; dpy = dpy - surfy; dpz = dpz - surfz;
          dpdx_e = dpdx_e - sxe; dpdy_e = dpdy_e - sye; dpdz_e = dpdz_e - sze;
          if (sp.out_o[0]) { sp.out_o[0][t] = sxn; sp.out_o[1][t] = syn; sp.out_o[2][t] = szn; }
          sp.out_n[0][t] = surfx; sp.out_n[1][t] = surfy; sp.out_n[2][t] = surfz;
        } else {
          sdu = sdu + surfx;
          sdv = sdv + surfy;
          sdw = sdw + surfz;
        }
        sdu = sdu - (dpdx_e + rhoxp * ph.irho0 * (dpx - dpdx_e));
        sdv = sdv - (dpdy_e + rhoyp * ph.irho0 * (dpy - dpdy_e));
        sdw = sdw - (dpdz_e + rhozp * ph.irho0 * (dpz - dpdz_e));
        if (BUOY) {
          const double s_c = __ldg(s + c), s_x = __ldg(s + c + 1), s_y = __ldg(s + c + sx), s_z = __ldg(s + c + sxy);
          const double factorxp = ph.rhobeta + ph.drhobeta * psixp;
          const double factoryp = ph.rhobeta + ph.drhobeta * psiyp;
          const double factorzp = ph.rhobeta + ph.drhobeta * psizp;
          sdu = sdu - ph.gacc[0] * factorxp * 0.5 * (s_x + s_c);
          sdv = sdv - ph.gacc[1] * factoryp * 0.5 * (s_y + s_c);
          sdw = sdw - ph.gacc[2] * factorzp * 0.5 * (s_z + s_c);
        }
        {
          const double ua = un + f12 * sdu * irx, va = vn + f12 * sdv * iry, wa = wn + f12 * sdw * irz;
          uo[c] = ua;
          vo[c] = va;
          wo[c] = wa;
          store_wraps(g, wrap, i, j, k, [&](int h) {
            uo[h] = ua;
            vo[h] = va;
            wo[h] = wa;
          });
        }
        // carry upwards
        u_ccm = PU(0, 0, 0); v_ccm = PV(0, 0, 0); w_ccm = PW(0, 0, 0); w_pcm = PW(0, 1, 0); w_cpm = PW(0, 0, 1);
        c_ccm = PC(0, 0, 0); c_pcm = PC(0, 1, 0); c_cpm = PC(0, 0, 1);
        flx_z_ccm = FLZ(0, 0, 0); flx_z_pcm = FLZ(0, 1, 0); flx_z_cpm = FLZ(0, 0, 1);
#undef PU
#undef PV
#undef PW
#undef PC
#undef FLX
#undef FLY
#undef FLZ
        p_c = p_z; po_c = po_z; pso_c = pso_z; k_c = k_z;
      }
      // plane k's slot is refilled at the next level; a plane copy that
      // never completed stops the block
      if (__syncthreads_or(fail)) break;
    }
    if (fail && tid == 0) {
      // the copies still in flight land before the block exits
      for (int kk = max(kb, issued - NSLOT + 1); kk <= issued; ++kk) tma::bar_wait(s_bar + slot(kk), phase(kk));
      DevScalars* scw = const_cast<DevScalars*>(sc);
      atomicCAS(&scw->status, CANSFZ_OK, CANSFZ_ERR_TIMEOUT);
      scw->halted = 1;
    }
    (void)sxy;
  }
};
template <typename TI, int TYV, int OPT, int STG>
__global__ void __launch_bounds__(tile::Shape<TYV>::NT, 512 / tile::Shape<TYV>::NT) k_momentum_tile(Geo g, Phys ph,
    const DevScalars* __restrict__ sc, int kz, const double* __restrict__ u, const double* __restrict__ v,
    const double* __restrict__ w, const double* __restrict__ psi, const double* __restrict__ psio,
    const TI* __restrict__ fx, const TI* __restrict__ fy, const TI* __restrict__ fz, const double* __restrict__ p,
    const double* __restrict__ po, const TI* __restrict__ kappa, const double* __restrict__ s, const SurfSplit sp,
    TI* __restrict__ duo, TI* __restrict__ dvo, TI* __restrict__ dwo, double* __restrict__ uo,
    double* __restrict__ vo, double* __restrict__ wo, const __grid_constant__ HaloMaps maps, int wrap) {
  MomentumTile<TI, TYV, OPT, STG>::run(blk_here(), g, ph, sc, kz, u, v, w, psi, psio, fx, fy, fz, p, po, kappa, s, sp,
      duo, dvo, dwo, uo, vo, wo, maps, wrap);
}


// ---------------------------------------------------------------------------
// tensor maps of halo-layout fields (cuTensorMapEncodeTiled through the
// runtime's driver entry point, so the library needs no libcuda link)
// ---------------------------------------------------------------------------
namespace {
typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(f);
  }
  return fn;
}
}  // namespace

bool make_halo_map(CUtensorMap* m, const void* base, const Geo& g, int bx, int by) {
  EncodeTiled fn = encode_fn();
  if (!fn || !base || ((uintptr_t)base & 15) || (g.sx * 8) % 16 || (bx * 8) % 16) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)g.sx, (cuuint64_t)(g.ny + 2), (cuuint64_t)(g.nz + 2)};
  const cuuint64_t strides[2] = {(cuuint64_t)g.sx * 8, (cuuint64_t)g.sxy * 8};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, 1};
  const cuuint32_t estr[3] = {1, 1, 1};
  return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <typename TI, int TYV, int OPT>
static void momentum_go(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* u,
                        const double* v, const double* w, const double* psi, const double* psio, const TI* fx,
                        const TI* fy, const TI* fz, const double* p, const double* po, const TI* kappa,
                        const double* s, const SurfSplit& sp, TI* duo, TI* dvo, TI* dwo, double* uo, double* vo,
                        double* wo) {
  using S = tile::Shape<TYV>;
  const int kz = tile::kz_of<TYV>(g, L.batched, L.nsm, L.mom_slots > 0 ? L.mom_slots : kMomSlots);
  // the staged fields' tensor maps: all eleven in the FP64 drop-in; the
  // seven FP64 ones (u v w psi, psio p po: entries 0-3 and 7-9) in the mixed
  // form, whose FP32 planes are element copies
  HaloMaps maps;
  std::memset(&maps, 0, sizeof(maps));
  int use_tma = 0;
  if (L.tma) {
    const void* f[11] = {u, v, w, psi, fx, fy, fz, psio, p, po, kappa};
    use_tma = 1;
    for (int q = 0; q < 11; ++q) {
      if (sizeof(TI) != 8 && ((q >= 4 && q <= 6) || q == 10)) continue;
      if (!make_halo_map(&maps.m[q], f[q], g, S::PX, S::TY + 2)) use_tma = 0;
    }
  }
  if (use_tma)
    kgo<MomentumTile<TI, TYV, OPT, 1>, S::NT, 512 / S::NT>(L, k_momentum_tile<TI, TYV, OPT, 1>,
        tile::grid_of<TYV>(g, kz), dim3(S::TX, S::TY), mom_smem<TI, TYV, 1>(), g, ph, sc, kz, u, v, w, psi, psio, fx,
        fy, fz, p, po, kappa, s, sp, duo, dvo, dwo, uo, vo, wo, maps, L.wrap);
  else
    kgo<MomentumTile<TI, TYV, OPT, 0>, S::NT, 512 / S::NT>(L, k_momentum_tile<TI, TYV, OPT, 0>,
        tile::grid_of<TYV>(g, kz), dim3(S::TX, S::TY), mom_smem<TI, TYV, 0>(), g, ph, sc, kz, u, v, w, psi, psio, fx,
        fy, fz, p, po, kappa, s, sp, duo, dvo, dwo, uo, vo, wo, maps, L.wrap);
}

template <typename TI, int TYV>
static void momentum_opt(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* u,
                         const double* v, const double* w, const double* psi, const double* psio, const TI* fx,
                         const TI* fy, const TI* fz, const double* p, const double* po, const TI* kappa,
                         const double* s, const SurfSplit* sp, TI* duo, TI* dvo, TI* dwo, double* uo, double* vo,
                         double* wo) {
  const SurfSplit none{};
  const SurfSplit& q = sp ? *sp : none;
  const int opt = (s ? kMomBuoy : 0) | (sp ? kMomBal : 0);
  if (opt == kMomBuoy)
    momentum_go<TI, TYV, kMomBuoy>(L, g, ph, sc, u, v, w, psi, psio, fx, fy, fz, p, po, kappa, s, q, duo, dvo, dwo,
                                   uo, vo, wo);
  else if (opt == kMomBal)
    momentum_go<TI, TYV, kMomBal>(L, g, ph, sc, u, v, w, psi, psio, fx, fy, fz, p, po, kappa, s, q, duo, dvo, dwo,
                                  uo, vo, wo);
  else if (opt == (kMomBuoy | kMomBal))
    momentum_go<TI, TYV, kMomBuoy | kMomBal>(L, g, ph, sc, u, v, w, psi, psio, fx, fy, fz, p, po, kappa, s, q, duo,
                                             dvo, dwo, uo, vo, wo);
  else
    momentum_go<TI, TYV, 0>(L, g, ph, sc, u, v, w, psi, psio, fx, fy, fz, p, po, kappa, s, q, duo, dvo, dwo, uo, vo,
                            wo);
}

template <typename TI>
void launch_momentum_t(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* u,
                       const double* v, const double* w, const double* psi, const double* psio, const TI* fx,
                       const TI* fy, const TI* fz, const double* p, const double* po, const TI* kappa,
                       const double* s, const SurfSplit* sp, TI* duo, TI* dvo, TI* dwo, double* uo, double* vo,
                       double* wo) {
  if (tile::rows_of(g) == 2)
    momentum_opt<TI, 2>(L, g, ph, sc, u, v, w, psi, psio, fx, fy, fz, p, po, kappa, s, sp, duo, dvo, dwo, uo, vo, wo);
  else
    momentum_opt<TI, 4>(L, g, ph, sc, u, v, w, psi, psio, fx, fy, fz, p, po, kappa, s, sp, duo, dvo, dwo, uo, vo, wo);
}

template void launch_momentum_t<double>(const Launch&, const Geo&, const Phys&, const DevScalars*, const double*,
                                        const double*, const double*, const double*, const double*, const double*,
                                        const double*, const double*, const double*, const double*, const double*,
                                        const double*, const SurfSplit*, double*, double*, double*, double*, double*,
                                        double*);
template void launch_momentum_t<float>(const Launch&, const Geo&, const Phys&, const DevScalars*, const double*,
                                       const double*, const double*, const double*, const double*, const float*,
                                       const float*, const float*, const double*, const double*, const float*,
                                       const double*, const SurfSplit*, float*, float*, float*, double*, double*,
                                       double*);

// the momentum tiles use more than the default 48 KB of dynamic shared memory
template <typename TI, int TYV, int OPT>
static void mom_attr() {
  cudaFuncSetAttribute(k_momentum_tile<TI, TYV, OPT, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)mom_smem<TI, TYV, 0>());
  cudaFuncSetAttribute(k_momentum_tile<TI, TYV, OPT, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)mom_smem<TI, TYV, 1>());
}
template <typename TI, int TYV>
static void mom_attrs() {
  mom_attr<TI, TYV, 0>();
  mom_attr<TI, TYV, kMomBuoy>();
  mom_attr<TI, TYV, kMomBal>();
  mom_attr<TI, TYV, kMomBuoy | kMomBal>();
}
void momentum_set_attributes() {
  mom_attrs<double, 4>();
  mom_attrs<float, 4>();
  mom_attrs<double, 2>();
  mom_attrs<float, 2>();
}

}  // namespace cansfz
