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
// the same four terms in another order).  A cell's normal sums its eight
// vertices as the two half sums its curvature takes the difference of (the
// reference sums them in order 1..8: the normal may differ in the last bit).  The vertex plane of level k+1 and
// the cells of level k are evaluated in the same pass (three vertex planes,
// four cell planes in the ring), so each level needs one barrier.  A vertex
// plane has (TX+1)(TY+1) vertices, TX+TY+1 more than the tile's cells; a
// ninth warp takes those, so that per level every thread evaluates at most
// two normalisations (one vertex and one cell, or two vertices) and no cell
// warp waits at the barrier for a third.
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

// 1/(sqrt(s) + eps) for s >= 0, the normalisation factor of the face
// normal in the ACDI regularisation flux (src/acdi.f90:150-190).  With r = 1/sqrt(s),
// 1/(sqrt(s) + eps) = r/(1 + eps*r) = r*(1 - eps*r + (eps*r)^2 - ...); where
// eps*r < 2^-26 the first two terms are exact to below 2^-52 relative, so
// r - (eps*r)*r is within an ulp or two of the direct form; one rsqrt takes
// the place of a square root and a division.  Elsewhere (|grad| below ~1e-8,
// zero included) the direct form.
template <typename T>
__device__ __forceinline__ T inv_norm_eps(T s) {
  const T r = rsqrt(s);
  const T er = T(CANSFZ_EPS) * r;
  if (er < T(1.4901161193847656e-8)) return r - er * r;
  return T(1) / (sqrt(s) + T(CANSFZ_EPS));
}

}  // namespace

// ---------------------------------------------------------------------------
// Youngs normals and curvature
// ---------------------------------------------------------------------------
template <typename TI, int TYV>
struct YoungsTile {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const DevScalars* __restrict__ sc, int kz,
      const TI* __restrict__ phi, TI* __restrict__ normx, TI* __restrict__ normy, TI* __restrict__ normz,
      TI* __restrict__ kappa, int wrap) {
    using namespace tile;
    using SH = Shape<TYV>;
    constexpr int TX = SH::TX, TY = SH::TY, NT = SH::NT, PX = SH::PX, PXY = SH::PXY;
    typedef TI T;
    constexpr int VX = TX + 1, VY = TY + 1, VXY = VX * VY;  // vertices of the tile's cells in one plane
    // threads: TY cell rows plus the vertex warp; each thread's first vertex
    // is its own index, and the vertex warp's lanes 0..TY take the rest
    constexpr int NTT = NT + TX;
    static_assert(NTT <= VXY && VXY - NTT <= TX, "one vertex per thread plus the vertex warp's second");
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
        for (int q = tid; q < PXY; q += NTT) {
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
      auto vertex = [&](int q) {
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
      };
      vertex(tid);  // tid < NTT <= VXY
      if (tid >= NT && tid - NT + NTT < VXY) vertex(tid - NT + NTT);
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
    const bool act = ty < TY && i <= g.nx && j <= g.ny;
    const T d1 = (T)g.dxi, d2 = (T)g.dyi;
    const int wox = wrap_ox(g, wrap, i), woy = wrap_oy(g, wrap, j);  // the column's x and y images
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
        // the half sums over the +/- vertices of each direction serve both
        // the curvature (their difference) and the cell normal (their sum)
        const T xp = mx[0] + mx[1] + mx[2] + mx[3], xm = mx[4] + mx[5] + mx[6] + mx[7];
        const T yp = my[0] + my[2] + my[4] + my[6], ym = my[1] + my[3] + my[5] + my[7];
        const T zp = mz[0] + mz[1] + mz[4] + mz[5], zm = mz[2] + mz[3] + mz[6] + mz[7];
        const T norm_x = T(.125) * (xp + xm);
        const T norm_y = T(.125) * (yp + ym);
        const T norm_z = T(.125) * (zp + zm);
        const T inv = recip_rn(sqrt(sqr(norm_x) + sqr(norm_y) + sqr(norm_z)) + T(CANSFZ_EPS));
        const int c = g.h(i, j, k);
        const T ox = norm_x * inv, oy = norm_y * inv, oz = norm_z * inv;
        const T kap = -(T(0.25) * (xp - xm) * d1 + T(0.25) * (yp - ym) * d2 + T(0.25) * (zp - zm) * (T)g.dzfi[k]);
        normx[c] = ox;
        normy[c] = oy;
        normz[c] = oz;
        kappa[c] = kap;
        store_images(c, wox, woy, wrap_oz(g, wrap, k), [&](int h) {
          normx[h] = ox;
          normy[h] = oy;
          normz[h] = oz;
          kappa[h] = kap;
        });
      }
    }
  }
};
template <typename TI, int TYV>
__global__ void __launch_bounds__(tile::Shape<TYV>::NT + tile::Shape<TYV>::TX, 4) k_youngs_tile(Geo g, const DevScalars* __restrict__ sc, int kz,
                                                          const TI* __restrict__ phi, TI* __restrict__ normx,
                                                          TI* __restrict__ normy, TI* __restrict__ normz,
                                                          TI* __restrict__ kappa, int wrap) {
  YoungsTile<TI, TYV>::run(blk_here(), g, sc, kz, phi, normx, normy, normz, kappa, wrap);
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
  const T rn = nn * inv_norm_eps(sqr(nxf) + sqr(nyf) + sqr(nzf));
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
      TI* __restrict__ fy, TI* __restrict__ fz, double* __restrict__ psi_out, int wrap) {
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
        double pn = 0.;
        if (UPD) {
          const T dO = first2 ? d : dO_pre;
          pn = fmin(fmax(0., psi_c + sc->f1 * (double)d + sc->f2 * (double)dO), 1.);
          psi_out[c] = pn;
        }
        dpsidt[t] = d;
        const T ex = upxp - rgxp, ey = upyp - rgyp, ez = up_zp - rg_zp;
        fx[c] = ex;
        fy[c] = ey;
        fz[c] = ez;
        store_wraps(g, wrap, i, j, k, [&](int h) {
          if (UPD) psi_out[h] = pn;
          fx[h] = ex;
          fy[h] = ey;
          fz[h] = ez;
        });
      }
      up_zm = up_zp;
      rg_zm = rg_zp;
    }
    (void)sx;
  }
};
template <typename TI, bool SDF, bool UPD, int TYV>
__global__ void __launch_bounds__(tile::Shape<TYV>::TX * (tile::Shape<TYV>::TY + 1), 3) k_acdi_tile(Geo g, const DevScalars* __restrict__ sc, int kz,
    const double* __restrict__ u, const double* __restrict__ v, const double* __restrict__ w,
    const TI* __restrict__ nx_, const TI* __restrict__ ny_, const TI* __restrict__ nz_,
    const TI* __restrict__ phi, const double* __restrict__ psi, TI* __restrict__ dpsidt,
    TI* __restrict__ fx, TI* __restrict__ fy, TI* __restrict__ fz, double* __restrict__ psi_out, int wrap) {
  AcdiTile<TI, SDF, UPD, TYV>::run(blk_here(), g, sc, kz, u, v, w, nx_, ny_, nz_, phi, psi, dpsidt, fx, fy, fz,
      psi_out, wrap);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <typename TI, int TYV>
static void youngs_go(const Launch& L, const Geo& g, const DevScalars* sc, const TI* phi, TI* nx, TI* ny, TI* nz,
                      TI* kappa) {
  using S = tile::Shape<TYV>;
  const int kz = tile::kz_of<TYV>(g, L.batched, L.nsm, L.phase_slots > 0 ? L.phase_slots : 24);
  kgo<YoungsTile<TI, TYV>, S::NT + S::TX, 4>(L, k_youngs_tile<TI, TYV>, tile::grid_of<TYV>(g, kz),
                                              dim3(S::TX, S::TY + 1), 0, g, sc, kz, phi, nx, ny, nz, kappa, L.wrap);
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
  const int kz = tile::kz_of<TYV>(g, L.batched, L.nsm, L.phase_slots > 0 ? L.phase_slots : 24);
  kgo<AcdiTile<TI, SDF, UPD, TYV>, S::TX * (S::TY + 1), 3>(L, k_acdi_tile<TI, SDF, UPD, TYV>,
                                             tile::grid_of<TYV>(g, kz),
                                             dim3(S::TX, S::TY + 1), acdi_smem<TI, SDF, TYV>(), g, sc, kz, u, v, w, nx,
                                             ny, nz, phi, psi, hist, fx, fy, fz, psi_out, L.wrap);
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

// the ACDI tiles use more than the default 48 KB of dynamic shared memory
template <typename TI, bool SDF, bool UPD, int TYV>
static void acdi_attr() {
  cudaFuncSetAttribute(k_acdi_tile<TI, SDF, UPD, TYV>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)acdi_smem<TI, SDF, TYV>());
}
template <typename TI, int TYV>
static void tile_attrs() {
  acdi_attr<TI, true, true, TYV>();
  acdi_attr<TI, true, false, TYV>();
  acdi_attr<TI, false, true, TYV>();
  acdi_attr<TI, false, false, TYV>();
}
void tiles_set_attributes() {
  tile_attrs<double, 8>();
  tile_attrs<float, 8>();
  tile_attrs<double, 2>();
  tile_attrs<float, 2>();
}

}  // namespace cansfz
