// Ghost-layer fills of boundp / bounduvw (src/bound.f90:15-124) on a 1x1
// pencil.  The reference's order decides the corner and edge ghosts:
//   1. updthalo: periodic self-exchange along y, then z (src/bound.f90:398-475)
//   2. set_bc on the x faces (x is the pencil axis, always bounded)
//   3. set_bc on the y faces when y is not periodic
//   4. set_bc on the z faces when z is not periodic
// Each stage is one launch over every field of a BcGroup; within a stage a
// thread owns one point of the face plane and applies face 0 then face 1,
// exactly as set_bc (src/bound.f90:126-293) writes them.  A field whose
// producing kernel already wrote its periodic images (BcField::wrapped)
// skips the periodic copies of those directions; the stages of its
// non-periodic faces run as before and read those images.
#include "batch.cuh"

namespace cansfz {

enum { ST_PER = 0, ST_X = 1, ST_Y = 2, ST_Z = 3 };

// set_bc for one line along idir through the plane point: q(m) addresses the
// element at index m (0..n+1) of that line.
template <typename E, typename Q>
__device__ __forceinline__ void set_bc_line(const BcFace& f, int ib, int n, E* __restrict__ p, Q q) {
  if (f.type == BC_NONE) return;
  if (f.type == BC_P) {
    // p(0) = p(n); p(n+1) = p(1)
    p[q(0)] = p[q(n)];
    p[q(n + 1)] = p[q(1)];
    return;
  }
  const E factor = (E)f.factor, sgn = (E)f.sgn;
  if (f.centered) {
    if (ib == 0) p[q(0)] = factor + sgn * p[q(1)];
    else p[q(n + 1)] = factor + sgn * p[q(n)];
  } else if (f.type == BC_D) {
    if (ib == 0) p[q(0)] = factor;
    else { p[q(n + 1)] = p[q(n - 1)]; p[q(n)] = factor; }
  } else {  // non-centered N
    if (ib == 0) p[q(0)] = E(1.) * factor + p[q(1)];
    else { p[q(n + 1)] = p[q(n)]; p[q(n)] = E(1.) * factor + p[q(n - 1)]; }
  }
}

template <int STAGE, typename E>
__device__ __forceinline__ void bc_stage_point(const Geo& g, const BcField& F, E* __restrict__ p, int q) {
  const int NX = g.nx + 2, NY = g.ny + 2, NZ = g.nz + 2;
  if (STAGE == ST_PER) {
    const bool py = F.halo_periodic[1] && !(F.wrapped & 2), pz = F.halo_periodic[2] && !(F.wrapped & 4);
    const int nyp = py ? 2 * NX * NZ : 0, nzp = pz ? 2 * NX * NY : 0;
    int i, j, k;
    if (q < nyp) {
      i = q % NX; const int r = q / NX; k = r % NZ; j = (r / NZ) ? g.ny + 1 : 0;
    } else if (q < nyp + nzp) {
      const int s = q - nyp;
      i = s % NX; const int r = s / NX; j = r % NY; k = (r / NY) ? g.nz + 1 : 0;
    } else {
      return;
    }
    int js = j, ks = k;
    if (py) { if (j == 0) js = g.ny; else if (j == g.ny + 1) js = 1; }
    if (pz) { if (k == 0) ks = g.nz; else if (k == g.nz + 1) ks = 1; }
    p[g.h(i, j, k)] = p[g.h(i, js, ks)];
  } else if (STAGE == ST_X) {
    if (q >= NY * NZ || (F.wrapped & 1)) return;
    const int j = q % NY, k = q / NY;
    const int base = g.sx * j + g.sxy * k;
    auto at = [=](int m) { return base + m; };
    set_bc_line(F.face[0][0], 0, g.nx, p, at);
    set_bc_line(F.face[0][1], 1, g.nx, p, at);
  } else if (STAGE == ST_Y) {
    if (q >= NX * NZ) return;
    const int i = q % NX, k = q / NX;
    const int base = i + g.sxy * k, sx = g.sx;
    auto at = [=](int m) { return base + sx * m; };
    set_bc_line(F.face[1][0], 0, g.ny, p, at);
    set_bc_line(F.face[1][1], 1, g.ny, p, at);
  } else {
    if (q >= NX * NY) return;
    const int i = q % NX, j = q / NX;
    const int base = i + g.sx * j, sxy = g.sxy;
    auto at = [=](int m) { return base + sxy * m; };
    set_bc_line(F.face[2][0], 0, g.nz, p, at);
    set_bc_line(F.face[2][1], 1, g.nz, p, at);
  }
}

template <int STAGE>
struct BcStage {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const BcGroup& grp,
      const DevScalars* __restrict__ sc) {
    if (sc != nullptr && sc->halted) return;
    const int fi = bk.y;
    if (fi >= grp.nf) return;
    const BcField& F = grp.f[fi];
    const int q = bk.x * blockDim.x + threadIdx.x;
    if (F.f32) bc_stage_point<STAGE, float>(g, F, static_cast<float*>(F.p), q);
    else bc_stage_point<STAGE, double>(g, F, static_cast<double*>(F.p), q);
  }
};
template <int STAGE>
__global__ void k_bc_stage(Geo g, BcGroup grp, const DevScalars* __restrict__ sc) {
  BcStage<STAGE>::run(blk_here(), g, grp, sc);
}

void launch_bc_group(const Launch& L, const Geo& g, const BcGroup& grp, const DevScalars* sc) {
  if (grp.nf <= 0) return;
  bool any_per = false, any_x = false, any_y = false, any_z = false;
  for (int f = 0; f < grp.nf; ++f) {
    const BcField& F = grp.f[f];
    any_per |= (F.halo_periodic[1] && !(F.wrapped & 2)) || (F.halo_periodic[2] && !(F.wrapped & 4));
    any_x |= (F.face[0][0].type != BC_NONE || F.face[0][1].type != BC_NONE) && !(F.wrapped & 1);
    any_y |= F.face[1][0].type != BC_NONE || F.face[1][1].type != BC_NONE;
    any_z |= F.face[2][0].type != BC_NONE || F.face[2][1].type != BC_NONE;
  }
  const int NX = g.nx + 2, NY = g.ny + 2, NZ = g.nz + 2;
  const int tb = 256;
  if (any_per) {
    const int n = 2 * NX * NZ + 2 * NX * NY;
    kgo<BcStage<ST_PER>, 256, 1>(L, k_bc_stage<ST_PER>, dim3((n + tb - 1) / tb, grp.nf), tb, 0, g, grp, sc);
  }
  if (any_x) kgo<BcStage<ST_X>, 256, 1>(L, k_bc_stage<ST_X>, dim3((NY * NZ + tb - 1) / tb, grp.nf), tb, 0, g, grp, sc);
  if (any_y) kgo<BcStage<ST_Y>, 256, 1>(L, k_bc_stage<ST_Y>, dim3((NX * NZ + tb - 1) / tb, grp.nf), tb, 0, g, grp, sc);
  if (any_z) kgo<BcStage<ST_Z>, 256, 1>(L, k_bc_stage<ST_Z>, dim3((NX * NY + tb - 1) / tb, grp.nf), tb, 0, g, grp, sc);
}

// updt_rhs_b, src/bound.f90:341-396 (c_or_f = 'c', so q = 0): add the BC
// planes rhsb?(:,:,0:1) to the boundary-adjacent RHS planes.
__global__ void k_updt_rhs_b(Geo g, int bx0, int bx1, int by0, int by1, int bz0, int bz1,
                             const double* __restrict__ rx, const double* __restrict__ ry,
                             const double* __restrict__ rz, double* __restrict__ p) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  const int nx = g.nx, ny = g.ny, nz = g.nz;
  // the six planes are added in the reference's order; each thread owns one
  // point of one plane and the planes only overlap on their edges, so the
  // edge cells receive their contributions in launch order below.
  if (blockIdx.y == 0 && q < ny * nz) {
    const int j = q % ny + 1, k = q / ny + 1;
    if (bx0) p[g.h(1, j, k)] += rx[(j - 1) + ny * (k - 1)];
    if (bx1) p[g.h(nx, j, k)] += rx[(j - 1) + ny * ((k - 1) + nz)];
  } else if (blockIdx.y == 1 && q < nx * nz) {
    const int i = q % nx + 1, k = q / nx + 1;
    if (by0) p[g.h(i, 1, k)] += ry[(i - 1) + nx * (k - 1)];
    if (by1) p[g.h(i, ny, k)] += ry[(i - 1) + nx * ((k - 1) + nz)];
  } else if (blockIdx.y == 2 && q < nx * ny) {
    const int i = q % nx + 1, j = q / nx + 1;
    if (bz0) p[g.h(i, j, 1)] += rz[(i - 1) + nx * (j - 1)];
    if (bz1) p[g.h(i, j, nz)] += rz[(i - 1) + nx * ((j - 1) + ny)];
  }
}

void launch_updt_rhs_b(const Launch& L, const Geo& g, const int is_bound[3][2], const double* rhsbx,
                       const double* rhsby, const double* rhsbz, double* p) {
  const int tb = 256;
  const int n0 = g.ny * g.nz, n1 = g.nx * g.nz, n2 = g.nx * g.ny;
  // x, y, z planes one launch each so that edge cells add in the reference order
  k_updt_rhs_b<<<dim3((n0 + tb - 1) / tb, 1), tb, 0, L.st>>>(g, is_bound[0][0], is_bound[0][1], 0, 0, 0, 0, rhsbx,
                                                            rhsby, rhsbz, p);
  k_updt_rhs_b<<<dim3((n1 + tb - 1) / tb, 2), tb, 0, L.st>>>(g, 0, 0, is_bound[1][0], is_bound[1][1], 0, 0, rhsbx,
                                                            rhsby, rhsbz, p);
  k_updt_rhs_b<<<dim3((n2 + tb - 1) / tb, 3), tb, 0, L.st>>>(g, 0, 0, 0, 0, is_bound[2][0], is_bound[2][1], rhsbx,
                                                            rhsby, rhsbz, p);
}

}  // namespace cansfz
