// z-marching tile kernels of the phase-field stage:
//
//   k_youngs_tile  cmpt_norm_curv_youngs, src/two_fluid.f90:60-175
//   k_acdi_tile    acdi_transport_pf, src/acdi.f90:64-225, with rk_2fl's
//                  update and clip fused in (src/rk.f90:234-248)
//
// Both are templated on the intermediate type TI: double in the FP64 drop-in,
// float in the mixed form (state fields u, v, w, psi stay FP64 in both).
//
// Youngs: the reference evaluates, for every cell, the gradient at its eight
// vertices and normalises each one (8 square roots and divisions per cell);
// each vertex is shared by eight cells.  Here a vertex plane k+1/2 of the
// tile is computed once into shared memory and each cell gathers its eight
// vertices.  The vertex gradient is evaluated in the form the reference uses
// for the (+x,+y,+z) vertex of its lower cell, so a vertex that the
// reference evaluates from another cell may differ in the last bit (sums of
// the same four terms in another order).  The vertex plane of level k+1 and
// the cells of level k are evaluated in the same pass (three vertex planes,
// four cell planes in the ring), so each level needs one barrier.
//
// ACDI: each face flux (advective part and regularisation part) is shared by
// the two cells on either side.  Each thread evaluates its cell's +x, +y and
// +z faces together (x and y into shared memory, the z face carried in
// registers to the next level as its k-1/2 face); one extra warp evaluates
// the tile's 40 -x and -y boundary faces meanwhile, so that no cell warp
// takes a fourth face evaluation per level.  The face velocities of level
// k+1 and the AB2 history of level k are loaded before level k's faces are
// evaluated, so that the face arithmetic hides their latency.  Every face
// expression is the reference's with the two cells' roles swapped only inside sums and
// products of two terms, so the results are bitwise those of the per-cell
// form.
#include "batch.cuh"
#include "k_tiles.cuh"

namespace cansfz {

#define HALTED(sc) ((sc) != nullptr && (sc)->halted)

namespace {

template <typename T>
__device__ __forceinline__ T sqr(T x) { return x * x; }

template <int TYV>
int tile_kz(const Geo& g, int batched) {
  using S = tile::Shape<TYV>;
  // in an ensemble the other cases keep the GPU busy: 32 levels per block
  // spend 6% on the two extra planes each block loads (25% at 8 levels)
  if (batched) return g.nz < 32 ? g.nz : 32;
  // about six waves of four resident blocks on each of 148 SMs, so the last
  // partial wave costs little; at least 8 levels per block (each block loads
  // two planes and evaluates one face/vertex plane beyond its own levels)
  const long long xy = (long long)((g.nx + S::TX - 1) / S::TX) * ((g.ny + S::TY - 1) / S::TY);
  long long kz = (xy * g.nz) / (148LL * 24);
  if (kz < 8) kz = 8;
  if (kz > 64) kz = 64;
  return (int)kz;
}

}  // namespace

// ---------------------------------------------------------------------------
// Youngs normals and curvature
// ---------------------------------------------------------------------------
template <typename TI, int TYV>
struct YoungsTile {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const DevScalars* __restrict__ sc, int kz,
      const TI* __restrict__ phi, TI* __restrict__ normx, TI* __restrict__ normy, TI* __restrict__ normz,
      TI* __restrict__ kappa) {
    using namespace tile;
    using SH = Shape<TYV>;
    constexpr int TX = SH::TX, TY = SH::TY, NT = SH::NT, PX = SH::PX, PXY = SH::PXY;
    (void)TY;
    typedef TI T;
    constexpr int VX = TX + 1, VY = TY + 1, VXY = VX * VY;  // vertices of the tile's cells in one plane
    // cell planes m-1 .. m+2 around the level m being gathered (m+3 in
    // flight), and three vertex planes: the two the cells of level m gather
    // from and the one evaluated for level m+1 in the same pass
    constexpr int NCP = 4, NVP = 3;
    __shared__ T pl[NCP][PXY];
    __shared__ T vn[NVP][3][VXY];
    if (HALTED(sc)) return;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
    const int i0 = bk.x * TX + 1, j0 = bk.y * TY + 1;
    const int kb = bk.z * kz + 1, ke = min(kb + kz - 1, g.nz);

    // cell plane kk (kb-1 <= kk <= ke+1) into its ring slot; an empty group
    // past the top keeps the wait counts uniform
    auto issue = [&](int kk) {
      if (kk <= ke + 1) {
        T* dst = pl[kk % NCP];
        for (int q = tid; q < PXY; q += NT) {
          int h;
          const bool ok = plane_cell<PX>(g, i0, j0, kk, q, &h);
          cp_async(dst + q, phi + (ok ? h : 0), ok);
        }
      }
      cp_commit();
    };
    // vertex plane kk+1/2 from cell planes kk and kk+1
    auto vertices = [&](int kk) {
      const T* lo = pl[kk % NCP];
      const T* hi = pl[(kk + 1) % NCP];
      T* ox = vn[(kk + NVP) % NVP][0];
      T* oy = vn[(kk + NVP) % NVP][1];
      T* oz = vn[(kk + NVP) % NVP][2];
      const T d1 = (T)g.dxi, d2 = (T)g.dyi, dz = (T)g.dzci[kk];
      for (int q = tid; q < VXY; q += NT) {
        const int a = q % VX, b = q / VX, s = a + PX * b;
        const T ccc = lo[s], pcc = lo[s + 1], cpc = lo[s + PX], ppc = lo[s + PX + 1];
        const T ccp = hi[s], pcp = hi[s + 1], cpp = hi[s + PX], ppp = hi[s + PX + 1];
        const T mx = T(0.25) * ((pcc + ppc + pcp + ppp) - (ccc + cpc + ccp + cpp)) * d1;
        const T my = T(0.25) * ((cpc + ppc + cpp + ppp) - (ccc + pcc + ccp + pcp)) * d2;
        const T mz = T(0.25) * ((ccp + pcp + cpp + ppp) - (ccc + pcc + cpc + ppc)) * dz;
        const T inv = recip_rn(sqrt(sqr(mx) + sqr(my) + sqr(mz)) + T(CANSFZ_EPS));
        ox[q] = mx * inv;
        oy[q] = my * inv;
        oz[q] = mz * inv;
      }
    };

    issue(kb - 1);
    issue(kb);
    issue(kb + 1);
    issue(kb + 2);
    cp_wait<1>();
    __syncthreads();  // planes kb-1, kb, kb+1 are in
    vertices(kb - 1);
    vertices(kb);
    __syncthreads();  // plane kb-1's slot is refilled at the first level

    const int i = i0 + tx, j = j0 + ty;
    const bool act = i <= g.nx && j <= g.ny;
    const T d1 = (T)g.dxi, d2 = (T)g.dyi;
    for (int k = kb; k <= ke; ++k) {
      // plane k+3 goes into the slot of plane k-1, last read for vertex plane
      // k-1/2 before the previous barrier
      issue(k + 3);
      cp_wait<1>();
      __syncthreads();  // plane k+2 is in; vertex planes k-1/2 and k+1/2 are complete
      // one pass: vertex plane k+3/2 (for level k+1) and the cells of level k,
      // which read the other two vertex planes
      if (k + 1 <= ke) vertices(k + 1);
      if (act) {
        const T* lo = vn[(k - 1 + NVP) % NVP][0];
        const T* hi = vn[k % NVP][0];
        const int vm = tx + VX * ty;  // the (-x,-y) vertex of the cell
        // vertex q: 0 (+,+,+) 1 (+,-,+) 2 (+,+,-) 3 (+,-,-) 4 (-,+,+) 5 (-,-,+) 6 (-,+,-) 7 (-,-,-)
        const int off[8] = {VX + 1, 1, VX + 1, 1, VX, 0, VX, 0};
        T mx[8], my[8], mz[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const T* src = (q == 2 || q == 3 || q == 6 || q == 7) ? lo : hi;
          mx[q] = src[vm + off[q]];
          my[q] = src[VXY + vm + off[q]];
          mz[q] = src[2 * VXY + vm + off[q]];
        }
        const T norm_x = T(.125) * (mx[0] + mx[1] + mx[2] + mx[3] + mx[4] + mx[5] + mx[6] + mx[7]);
        const T norm_y = T(.125) * (my[0] + my[1] + my[2] + my[3] + my[4] + my[5] + my[6] + my[7]);
        const T norm_z = T(.125) * (mz[0] + mz[1] + mz[2] + mz[3] + mz[4] + mz[5] + mz[6] + mz[7]);
        const T inv = recip_rn(sqrt(sqr(norm_x) + sqr(norm_y) + sqr(norm_z)) + T(CANSFZ_EPS));
        const int c = g.h(i, j, k);
        normx[c] = norm_x * inv;
        normy[c] = norm_y * inv;
        normz[c] = norm_z * inv;
        kappa[c] = -(T(0.25) * ((mx[0] + mx[1] + mx[2] + mx[3]) - (mx[4] + mx[5] + mx[6] + mx[7])) * d1 +
                     T(0.25) * ((my[0] + my[2] + my[4] + my[6]) - (my[1] + my[3] + my[5] + my[7])) * d2 +
                     T(0.25) * ((mz[0] + mz[1] + mz[4] + mz[5]) - (mz[2] + mz[3] + mz[6] + mz[7])) * (T)g.dzfi[k]);
      }
    }
  }
};
template <typename TI, int TYV>
__global__ void __launch_bounds__(tile::Shape<TYV>::NT) k_youngs_tile(Geo g, const DevScalars* __restrict__ sc, int kz,
                                                          const TI* __restrict__ phi, TI* __restrict__ normx,
                                                          TI* __restrict__ normy, TI* __restrict__ normz,
                                                          TI* __restrict__ kappa) {
  YoungsTile<TI, TYV>::run(blk_here(), g, sc, kz, phi, normx, normy, normz, kappa);
}

// ---------------------------------------------------------------------------
// ACDI transport
// ---------------------------------------------------------------------------
namespace {

template <typename T>
struct AcdiCoef {
  T gs, gam, qg, is;  // gam*seps, gam, gam/4, 1/seps
};

// The advective flux `up` and the regularisation flux `rg` (diffusion minus
// sharpening) through the face between cells L and R along `dir`; dli is the
// inverse distance of the two cell centres.  src/acdi.f90:110-203 for the
// +face of cell L.
template <typename T, bool SDF>
__device__ __forceinline__ void acdi_face(const AcdiCoef<T>& cf, int dir, T dli, T psiL, T psiR, T vel, T nxL,
                                          T nyL, T nzL, T nxR, T nyR, T nzR, T phiL, T phiR, T* up, T* rg) {
  *up = T(0.5) * (psiR + psiL) * vel;
  const T dpsi = cf.gs * (psiR - psiL) * dli;
  const T nxf = T(0.5) * (nxR + nxL), nyf = T(0.5) * (nyR + nyL), nzf = T(0.5) * (nzR + nzL);
  const T nn = dir == 0 ? nxf : (dir == 1 ? nyf : nzf);
  const T rn = nn / (sqrt(sqr(nxf) + sqr(nyf) + sqr(nzf)) + T(CANSFZ_EPS));
  T sharp;
  if (SDF) {
    sharp = cf.qg * ((T(1.) - sqr(tanh(T(0.25) * (phiR + phiL) * cf.is))) * rn);
  } else {
    const T pf = T(0.5) * (psiR + psiL);
    sharp = cf.gam * pf * (T(1.) - pf) * rn;
  }
  *rg = dpsi - sharp;
}

template <typename TI, bool SDF, int TYV>
constexpr size_t acdi_smem() {
  using namespace tile;
  using SH = Shape<TYV>;
  constexpr int TX = SH::TX, TY = SH::TY, PXY = SH::PXY, NSLOT = SH::NSLOT;
  constexpr int NF = (TX + 1) * TY + TX * (TY + 1);
  return sizeof(double) * NSLOT * PXY + sizeof(TI) * (NSLOT * 3 * PXY + (SDF ? NSLOT * PXY : 0) + 2 * NF);
}

}  // namespace

// UPD: psi_out = clip(psi + f1*d + f2*d_old); `dpsidt` holds d_old on entry
// and d on exit.  Without UPD, dpsidt receives d.
template <typename TI, bool SDF, bool UPD, int TYV>
struct AcdiTile {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const DevScalars* __restrict__ sc, int kz,
      const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ w,
      const TI* __restrict__ nx_, const TI* __restrict__ ny_, const TI* __restrict__ nz_,
      const TI* __restrict__ phi, const double* __restrict__ psi, TI* __restrict__ dpsidt, TI* __restrict__ fx,
      TI* __restrict__ fy, TI* __restrict__ fz, double* __restrict__ psi_out) {
    using namespace tile;
    using SH = Shape<TYV>;
    constexpr int TX = SH::TX, TY = SH::TY, PX = SH::PX, PXY = SH::PXY, NSLOT = SH::NSLOT;
    constexpr int NTA = TX * (TY + 1);  // TY rows of cell threads and one warp for the tile's boundary faces
    typedef TI T;
    constexpr int NFX = (TX + 1) * TY, NFY = TX * (TY + 1), NF = NFX + NFY;
    extern __shared__ __align__(16) unsigned char smem[];
    double* s_psi = reinterpret_cast<double*>(smem);                 // [NSLOT][PXY]
    T* s_n = reinterpret_cast<T*>(s_psi + NSLOT * PXY);               // [NSLOT][3][PXY]
    T* s_phi = s_n + NSLOT * 3 * PXY;                                 // [NSLOT][PXY], SDF only
    T* f_up = s_phi + (SDF ? NSLOT * PXY : 0);                        // [NF]
    T* f_rg = f_up + NF;                                              // [NF]
    if (HALTED(sc)) return;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
    const int i0 = bk.x * TX + 1, j0 = bk.y * TY + 1;
    const int kb = bk.z * kz + 1, ke = min(kb + kz - 1, g.nz);
    const int sx = g.sx;
    AcdiCoef<T> cf;
    cf.gam = (T)sc->gam;
    const T seps = (T)sc->seps;
    cf.gs = cf.gam * seps;
    cf.qg = T(0.25) * cf.gam;
    cf.is = T(1.) / seps;
    const T dxi = (T)g.dxi, dyi = (T)g.dyi;
    const bool first2 = sc->first_rk2fl;

    auto issue = [&](int kk) {
      const int s = kk % NSLOT;
      for (int q = tid; q < PXY; q += NTA) {
        int h;
        const bool ok = plane_cell<PX>(g, i0, j0, kk, q, &h);
        const int hh = ok ? h : 0;
        cp_async(s_psi + s * PXY + q, psi + hh, ok);
        cp_async(s_n + (s * 3 + 0) * PXY + q, nx_ + hh, ok);
        cp_async(s_n + (s * 3 + 1) * PXY + q, ny_ + hh, ok);
        cp_async(s_n + (s * 3 + 2) * PXY + q, nz_ + hh, ok);
        if (SDF) cp_async(s_phi + s * PXY + q, phi + hh, ok);
      }
      cp_commit();
    };
    // face between plane elements qa (slot sa) and qb (slot sb)
    auto face = [&](int dir, T dli, int sa, int qa, int sb, int qb, T vel, T* up, T* rg) {
      const T* na = s_n + sa * 3 * PXY;
      const T* nb = s_n + sb * 3 * PXY;
      const T pa = SDF ? s_phi[sa * PXY + qa] : T(0), pb = SDF ? s_phi[sb * PXY + qb] : T(0);
      acdi_face<T, SDF>(cf, dir, dli, (T)s_psi[sa * PXY + qa], (T)s_psi[sb * PXY + qb], vel, na[qa],
                        na[PXY + qa], na[2 * PXY + qa], nb[qb], nb[PXY + qb], nb[2 * PXY + qb], pa, pb, up, rg);
    };

    const int i = i0 + tx, j = j0 + ty;
    const bool act = ty < TY && i <= g.nx && j <= g.ny;
    const int qc = (tx + 1) + PX * (ty + 1);  // the thread's own cell in a plane

    issue(kb - 1);
    issue(kb);
    issue(kb + 1);
    cp_wait<1>();
    __syncthreads();
    T up_zm = T(0), rg_zm = T(0);
    if (act)
      face(2, (T)g.dzci[kb - 1], (kb - 1) % NSLOT, qc, kb % NSLOT, qc, (T)__ldg(w + g.h(i, j, kb - 1)), &up_zm,
           &rg_zm);
    __syncthreads();  // plane kb-1's slot is refilled next

    T vx_n = T(0), vy_n = T(0), vz_n = T(0);
    if (act) {
      const int c = g.h(i, j, kb);
      vx_n = (T)__ldg(u + c); vy_n = (T)__ldg(v + c); vz_n = (T)__ldg(w + c);
    }
    for (int k = kb; k <= ke; ++k) {
      if (k + 2 <= ke + 1) issue(k + 2);
      else cp_commit();
      cp_wait<1>();
      __syncthreads();  // plane k+1 is in; every thread is done with level k-1
      const int s0 = k % NSLOT, s1 = (k + 1) % NSLOT;
      T up_zp = T(0), rg_zp = T(0);
      T dO_pre = T(0);
      if (act) {
        // the cell's own +x, +y and +z faces: three independent evaluations in
        // one block of code, so that their dependency chains overlap
        const int c = g.h(i, j, k);
        const T vx = vx_n, vy = vy_n, vz = vz_n;
        if (k < ke) {
          vx_n = (T)__ldg(u + c + g.sxy); vy_n = (T)__ldg(v + c + g.sxy); vz_n = (T)__ldg(w + c + g.sxy);
        }
        if (UPD && !first2) dO_pre = dpsidt[g.t(i, j, k)];
        T upx, rgx, upy, rgy;
        face(0, dxi, s0, qc, s0, qc + 1, vx, &upx, &rgx);
        face(1, dyi, s0, qc, s0, qc + PX, vy, &upy, &rgy);
        face(2, (T)g.dzci[k], s0, qc, s1, qc, vz, &up_zp, &rg_zp);
        const int fxp = ty * (TX + 1) + tx + 1, fyp = NFX + (ty + 1) * TX + tx;
        f_up[fxp] = upx;
        f_rg[fxp] = rgx;
        f_up[fyp] = upy;
        f_rg[fyp] = rgy;
      }
      // the tile's -x faces (x-face 0 of each row) and -y faces (y-face 0 of
      // each column), by the extra warp while the cell warps evaluate their
      // own three faces
      if (ty == TY) {
        for (int e = tx; e < TY + TX; e += TX) {
          if (e < TY) {
            if (j0 + e <= g.ny) {
              const int q = PX * (e + 1), f = e * (TX + 1);
              face(0, dxi, s0, q, s0, q + 1, (T)__ldg(u + g.h(i0 - 1, j0 + e, k)), &f_up[f], &f_rg[f]);
            }
          } else {
            const int a = e - TY;
            if (i0 + a <= g.nx) {
              const int q = a + 1, f = NFX + a;
              face(1, dyi, s0, q, s0, q + PX, (T)__ldg(v + g.h(i0 + a, j0 - 1, k)), &f_up[f], &f_rg[f]);
            }
          }
        }
      }
      const double psi_c = act ? s_psi[s0 * PXY + qc] : 0.;  // read before the barrier: the slot is refilled next level
      __syncthreads();
      if (act) {
        const int fxm = ty * (TX + 1) + tx, fym = NFX + ty * TX + tx;
        const T upxm = f_up[fxm], upxp = f_up[fxm + 1], rgxm = f_rg[fxm], rgxp = f_rg[fxm + 1];
        const T upym = f_up[fym], upyp = f_up[fym + TX], rgym = f_rg[fym], rgyp = f_rg[fym + TX];
        const T dzfi_c = (T)g.dzfi[k];
        const T adv = dxi * (upxp - upxm) + dyi * (upyp - upym) + dzfi_c * (up_zp - up_zm);
        const T rglr = (rgxp - rgxm) * dxi + (rgyp - rgym) * dyi + (rg_zp - rg_zm) * dzfi_c;
        const T d = -adv + rglr;
        const int c = g.h(i, j, k), t = g.t(i, j, k);
        if (UPD) {
          const T dO = first2 ? d : dO_pre;
          psi_out[c] = fmin(fmax(0., psi_c + sc->f1 * (double)d + sc->f2 * (double)dO), 1.);
        }
        dpsidt[t] = d;
        fx[c] = upxp - rgxp;
        fy[c] = upyp - rgyp;
        fz[c] = up_zp - rg_zp;
      }
      up_zm = up_zp;
      rg_zm = rg_zp;
    }
    (void)sx;
  }
};
template <typename TI, bool SDF, bool UPD, int TYV>
__global__ void __launch_bounds__(tile::Shape<TYV>::TX * (tile::Shape<TYV>::TY + 1)) k_acdi_tile(Geo g, const DevScalars* __restrict__ sc, int kz,
    const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ w,
    const TI* __restrict__ nx_, const TI* __restrict__ ny_, const TI* __restrict__ nz_,
    const TI* __restrict__ phi, const double* __restrict__ psi, TI* __restrict__ dpsidt,
    TI* __restrict__ fx, TI* __restrict__ fy, TI* __restrict__ fz, double* __restrict__ psi_out) {
  AcdiTile<TI, SDF, UPD, TYV>::run(blk_here(), g, sc, kz, u, v, w, nx_, ny_, nz_, phi, psi, dpsidt, fx, fy, fz,
      psi_out);
}

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
// that the stencil arithmetic hides their latency; holding them takes up to
// 128 registers; the kernel runs on 32x4 tiles (128 threads), four blocks per
// SM, so that a block's two barriers per level couple four warps, not eight.
// The expressions are those of the per-point kernels (same operand order).
// The whole update is evaluated in FP64.  TI is the storage type of the phase
// fluxes, the curvature and the AB2 histories: double in the drop-in, float
// in the mixed form (an FP32 RHS was 3% faster and left a 1e-6 pressure
// error; with the RHS in FP64 the mixed form's error is 5e-9).
// BUOY adds the Boussinesq buoyancy of the scalar s (_SCALAR with
// _BOUSSINESQ_BUOYANCY, src/mom.f90:1017-1024) after the pressure terms.
// ---------------------------------------------------------------------------
namespace {
template <typename TI, int TYV>
constexpr size_t mom_smem() {
  using namespace tile;
  using SH = Shape<TYV>;
  constexpr int PXY = SH::PXY, NSLOT = SH::NSLOT;
  return (size_t)NSLOT * PXY * (4 * sizeof(double) + 3 * sizeof(TI));
}
}  // namespace

template <typename TI, int TYV, bool BUOY>
struct MomentumTile {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const Phys& ph,
      const DevScalars* __restrict__ sc, int kz, const double* __restrict__ u, const double* __restrict__ v,
      const double* __restrict__ w, const double* __restrict__ psi, const double* __restrict__ psio,
      const TI* __restrict__ fx, const TI* __restrict__ fy, const TI* __restrict__ fz, const double* __restrict__ p,
      const double* __restrict__ po, const TI* __restrict__ kappa, const double* __restrict__ s,
      TI* __restrict__ duo, TI* __restrict__ dvo, TI* __restrict__ dwo, double* __restrict__ uo,
      double* __restrict__ vo, double* __restrict__ wo) {
    using namespace tile;
    using SH = Shape<TYV>;
    constexpr int TX = SH::TX, TY = SH::TY, NT = SH::NT, PX = SH::PX, PXY = SH::PXY, NSLOT = SH::NSLOT;
    (void)TY;
    typedef double T;  // the RHS in FP64 for both storage types
    extern __shared__ __align__(16) unsigned char smem[];
    double* s_u = reinterpret_cast<double*>(smem);  // each [NSLOT][PXY]
    double* s_v = s_u + NSLOT * PXY;
    double* s_w = s_v + NSLOT * PXY;
    double* s_c = s_w + NSLOT * PXY;
    TI* s_fx = reinterpret_cast<TI*>(s_c + NSLOT * PXY);
    TI* s_fy = s_fx + NSLOT * PXY;
    TI* s_fz = s_fy + NSLOT * PXY;
    if (HALTED(sc)) return;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + TX * ty;
    const int i0 = bk.x * TX + 1, j0 = bk.y * TY + 1;
    const int kb = bk.z * kz + 1, ke = min(kb + kz - 1, g.nz);
    const int sx = g.sx, sxy = g.sxy;

    auto issue = [&](int kk) {
      const int o = (kk % NSLOT) * PXY;
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
    for (int k = kb; k <= ke; ++k) {
      if (k + 2 <= ke + 1) issue(k + 2);
      else cp_commit();
      cp_wait<1>();
      __syncthreads();  // planes k and k+1 are in; every thread is done with level k-1
      if (act) {
        const int o0 = (k % NSLOT) * PXY + qc, o1 = ((k + 1) % NSLOT) * PXY + qc;
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
        const double pso_x = __ldg(psio + c + 1), pso_y = __ldg(psio + c + sx), pso_z = __ldg(psio + c + sxy);
        const double p_x = __ldg(p + c + 1), p_y = __ldg(p + c + sx), p_z = __ldg(p + c + sxy);
        const double po_x = __ldg(po + c + 1), po_y = __ldg(po + c + sx), po_z = __ldg(po + c + sxy);
        const double k_x = (double)__ldg(kappa + c + 1), k_y = (double)__ldg(kappa + c + sx),
                     k_z = (double)__ldg(kappa + c + sxy);
        const double hu0 = first ? 0. : (double)duo[t], hv0 = first ? 0. : (double)dvo[t],
                     hw0 = first ? 0. : (double)dwo[t];
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
        sdu = sdu + skappaxp * (ps_x - ps_c) * dxid;
        sdv = sdv + skappayp * (ps_y - ps_c) * dyid;
        sdw = sdw + skappazp * (ps_z - ps_c) * dzcid;
        const double dpdx_e = (q_pcc - q_ccc) * dxid, dpdy_e = (q_cpc - q_ccc) * dyid, dpdz_e = (q_ccp - q_ccc) * dzcid;
        sdu = sdu - (dpdx_e + rhoxp * ph.irho0 * (dpdx - dpdx_e));
        sdv = sdv - (dpdy_e + rhoyp * ph.irho0 * (dpdy - dpdy_e));
        sdw = sdw - (dpdz_e + rhozp * ph.irho0 * (dpdz - dpdz_e));
        if (BUOY) {
          const double s_c = __ldg(s + c), s_x = __ldg(s + c + 1), s_y = __ldg(s + c + sx), s_z = __ldg(s + c + sxy);
          const double factorxp = ph.rhobeta + ph.drhobeta * psixp;
          const double factoryp = ph.rhobeta + ph.drhobeta * psiyp;
          const double factorzp = ph.rhobeta + ph.drhobeta * psizp;
          sdu = sdu - ph.gacc[0] * factorxp * 0.5 * (s_x + s_c);
          sdv = sdv - ph.gacc[1] * factoryp * 0.5 * (s_y + s_c);
          sdw = sdw - ph.gacc[2] * factorzp * 0.5 * (s_z + s_c);
        }
        uo[c] = un + f12 * sdu * irx;
        vo[c] = vn + f12 * sdv * iry;
        wo[c] = wn + f12 * sdw * irz;
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
      __syncthreads();  // plane k's slot is refilled at the next level
    }
    (void)sxy;
  }
};
template <typename TI, int TYV, bool BUOY>
__global__ void __launch_bounds__(tile::Shape<TYV>::NT, 512 / tile::Shape<TYV>::NT) k_momentum_tile(Geo g, Phys ph,
    const DevScalars* __restrict__ sc, int kz, const double* __restrict__ u, const double* __restrict__ v,
    const double* __restrict__ w, const double* __restrict__ psi, const double* __restrict__ psio,
    const TI* __restrict__ fx, const TI* __restrict__ fy, const TI* __restrict__ fz, const double* __restrict__ p,
    const double* __restrict__ po, const TI* __restrict__ kappa, const double* __restrict__ s, TI* __restrict__ duo,
    TI* __restrict__ dvo, TI* __restrict__ dwo, double* __restrict__ uo, double* __restrict__ vo,
    double* __restrict__ wo) {
  MomentumTile<TI, TYV, BUOY>::run(blk_here(), g, ph, sc, kz, u, v, w, psi, psio, fx, fy, fz, p, po, kappa, s, duo,
      dvo, dwo, uo, vo, wo);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <typename TI, int TYV>
static void youngs_go(const Launch& L, const Geo& g, const DevScalars* sc, const TI* phi, TI* nx, TI* ny, TI* nz,
                      TI* kappa) {
  using S = tile::Shape<TYV>;
  const int kz = tile_kz<TYV>(g, L.batched);
  kgo<YoungsTile<TI, TYV>, S::NT, 3>(L, k_youngs_tile<TI, TYV>, tile::grid_of<TYV>(g, kz), dim3(S::TX, S::TY), 0, g,
                                     sc, kz, phi, nx, ny, nz, kappa);
}

template <typename TI>
void launch_youngs_t(const Launch& L, const Geo& g, const DevScalars* sc, const TI* phi, TI* nx, TI* ny, TI* nz,
                     TI* kappa) {
  if (tile::rows_of(g) == 2) youngs_go<TI, 2>(L, g, sc, phi, nx, ny, nz, kappa);
  else youngs_go<TI, 8>(L, g, sc, phi, nx, ny, nz, kappa);
}

template <typename TI, bool SDF, bool UPD, int TYV>
static void acdi_go(const Launch& L, const Geo& g, const DevScalars* sc, const double* u, const double* v,
                    const double* w, const TI* nx, const TI* ny, const TI* nz, const TI* phi, const double* psi,
                    double* psi_out, TI* hist, TI* fx, TI* fy, TI* fz) {
  using S = tile::Shape<TYV>;
  const int kz = tile_kz<TYV>(g, L.batched);
  kgo<AcdiTile<TI, SDF, UPD, TYV>, S::TX * (S::TY + 1), 3>(L, k_acdi_tile<TI, SDF, UPD, TYV>,
                                             tile::grid_of<TYV>(g, kz),
                                             dim3(S::TX, S::TY + 1), acdi_smem<TI, SDF, TYV>(), g, sc, kz, u, v, w, nx,
                                             ny, nz, phi, psi, hist, fx, fy, fz, psi_out);
}

template <typename TI, int TYV>
static void acdi_pick(const Launch& L, const Geo& g, const DevScalars* sc, bool sdf, bool upd, const double* u,
                      const double* v, const double* w, const TI* nx, const TI* ny, const TI* nz, const TI* phi,
                      const double* psi, double* psi_out, TI* hist, TI* fx, TI* fy, TI* fz) {
  if (sdf && upd) acdi_go<TI, true, true, TYV>(L, g, sc, u, v, w, nx, ny, nz, phi, psi, psi_out, hist, fx, fy, fz);
  else if (sdf) acdi_go<TI, true, false, TYV>(L, g, sc, u, v, w, nx, ny, nz, phi, psi, psi_out, hist, fx, fy, fz);
  else if (upd) acdi_go<TI, false, true, TYV>(L, g, sc, u, v, w, nx, ny, nz, phi, psi, psi_out, hist, fx, fy, fz);
  else acdi_go<TI, false, false, TYV>(L, g, sc, u, v, w, nx, ny, nz, phi, psi, psi_out, hist, fx, fy, fz);
}

template <typename TI>
void launch_acdi_t(const Launch& L, const Geo& g, const DevScalars* sc, bool sdf, bool upd, const double* u,
                   const double* v, const double* w, const TI* nx, const TI* ny, const TI* nz, const TI* phi,
                   const double* psi, double* psi_out, TI* hist, TI* fx, TI* fy, TI* fz) {
  if (tile::rows_of(g) == 2)
    acdi_pick<TI, 2>(L, g, sc, sdf, upd, u, v, w, nx, ny, nz, phi, psi, psi_out, hist, fx, fy, fz);
  else
    acdi_pick<TI, 8>(L, g, sc, sdf, upd, u, v, w, nx, ny, nz, phi, psi, psi_out, hist, fx, fy, fz);
}

template <typename TI, int TYV, bool BUOY>
static void momentum_go(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* u,
                        const double* v, const double* w, const double* psi, const double* psio, const TI* fx,
                        const TI* fy, const TI* fz, const double* p, const double* po, const TI* kappa,
                        const double* s, TI* duo, TI* dvo, TI* dwo, double* uo, double* vo, double* wo) {
  using S = tile::Shape<TYV>;
  const int kz = tile_kz<TYV>(g, L.batched);
  kgo<MomentumTile<TI, TYV, BUOY>, S::NT, 512 / S::NT>(L, k_momentum_tile<TI, TYV, BUOY>, tile::grid_of<TYV>(g, kz),
                                       dim3(S::TX, S::TY), mom_smem<TI, TYV>(), g, ph, sc, kz, u, v, w, psi, psio, fx,
                                       fy, fz, p, po, kappa, s, duo, dvo, dwo, uo, vo, wo);
}

template <typename TI>
void launch_momentum_t(const Launch& L, const Geo& g, const Phys& ph, const DevScalars* sc, const double* u,
                       const double* v, const double* w, const double* psi, const double* psio, const TI* fx,
                       const TI* fy, const TI* fz, const double* p, const double* po, const TI* kappa,
                       const double* s, TI* duo, TI* dvo, TI* dwo, double* uo, double* vo, double* wo) {
  const bool two = tile::rows_of(g) == 2;
  if (s && two)
    momentum_go<TI, 2, true>(L, g, ph, sc, u, v, w, psi, psio, fx, fy, fz, p, po, kappa, s, duo, dvo, dwo, uo, vo, wo);
  else if (s)
    momentum_go<TI, 4, true>(L, g, ph, sc, u, v, w, psi, psio, fx, fy, fz, p, po, kappa, s, duo, dvo, dwo, uo, vo, wo);
  else if (two)
    momentum_go<TI, 2, false>(L, g, ph, sc, u, v, w, psi, psio, fx, fy, fz, p, po, kappa, s, duo, dvo, dwo, uo, vo,
                              wo);
  else
    momentum_go<TI, 4, false>(L, g, ph, sc, u, v, w, psi, psio, fx, fy, fz, p, po, kappa, s, duo, dvo, dwo, uo, vo,
                              wo);
}

template void launch_momentum_t<double>(const Launch&, const Geo&, const Phys&, const DevScalars*, const double*,
                                        const double*, const double*, const double*, const double*, const double*,
                                        const double*, const double*, const double*, const double*, const double*,
                                        const double*, double*, double*, double*, double*, double*, double*);
template void launch_momentum_t<float>(const Launch&, const Geo&, const Phys&, const DevScalars*, const double*,
                                       const double*, const double*, const double*, const double*, const float*,
                                       const float*, const float*, const double*, const double*, const float*,
                                       const double*, float*, float*, float*, double*, double*, double*);
template void launch_youngs_t<double>(const Launch&, const Geo&, const DevScalars*, const double*, double*, double*,
                                      double*, double*);
template void launch_youngs_t<float>(const Launch&, const Geo&, const DevScalars*, const float*, float*, float*,
                                     float*, float*);
template void launch_acdi_t<double>(const Launch&, const Geo&, const DevScalars*, bool, bool, const double*,
                                    const double*, const double*, const double*, const double*, const double*,
                                    const double*, const double*, double*, double*, double*, double*, double*);
template void launch_acdi_t<float>(const Launch&, const Geo&, const DevScalars*, bool, bool, const double*,
                                   const double*, const double*, const float*, const float*, const float*,
                                   const float*, const double*, double*, float*, float*, float*, float*);

// the ACDI and momentum tiles use more than the default 48 KB of dynamic shared memory
template <typename TI, bool SDF, bool UPD, int TYV>
static void acdi_attr() {
  cudaFuncSetAttribute(k_acdi_tile<TI, SDF, UPD, TYV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)acdi_smem<TI, SDF, TYV>());
}
template <typename TI, int TYV>
static void mom_attrs() {
  cudaFuncSetAttribute(k_momentum_tile<TI, TYV, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)mom_smem<TI, TYV>());
  cudaFuncSetAttribute(k_momentum_tile<TI, TYV, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)mom_smem<TI, TYV>());
}
template <typename TI, int TYV>
static void tile_attrs() {
  acdi_attr<TI, true, true, TYV>();
  acdi_attr<TI, true, false, TYV>();
  acdi_attr<TI, false, true, TYV>();
  acdi_attr<TI, false, false, TYV>();
}
void tiles_set_attributes() {
  mom_attrs<double, 4>();
  mom_attrs<float, 4>();
  mom_attrs<double, 2>();
  mom_attrs<float, 2>();
  tile_attrs<double, 8>();
  tile_attrs<float, 8>();
  tile_attrs<double, 2>();
  tile_attrs<float, 2>();
}

}  // namespace cansfz
