// Shared pieces of the z-marching tile kernels (k_tiles.cu).
//
// A block owns TX x TY columns of cells and walks KZ levels in z.  The cell
// planes it needs (with a one-cell halo in x and y) are staged in shared
// memory through a three-slot ring filled by cp.async (8- or 4-byte
// element copies, zero-filled outside the array), one plane ahead of the
// level being computed.  Quantities shared by neighbouring cells (vertex
// gradients of the Youngs normals, face fluxes of the transport) are then
// computed once per vertex or face instead of once per cell that uses them.
#pragma once

#include "cansfz_internal.cuh"

namespace cansfz {
namespace tile {

// Tile shape: 32 x TYV columns.  TYV = 8 for 3-D grids; TYV = 2 for the
// reference's 2-D convention (ny = 2), where an 8-row tile would leave three
// quarters of its threads idle.
template <int TYV>
struct Shape {
  static constexpr int TX = 32, TY = TYV, NT = TX * TY;
  static constexpr int PX = TX + 2, PY = TY + 2, PXY = PX * PY;  // a plane of cells with a one-cell halo
  static constexpr int NSLOT = 3;                                // ring of planes k-1, k, k+1 (k+2 in flight)
};

__device__ __forceinline__ void cp_async(void* sdst, const double* gsrc, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gsrc), "r"(valid ? 8 : 0));
}
__device__ __forceinline__ void cp_async(void* sdst, const float* gsrc, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gsrc), "r"(valid ? 4 : 0));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Position of plane-slot element q (0 <= q < PXY) in the halo layout; false
// when the cell lies outside the array (beyond ghost nx+1 or ny+1).
template <int PX>
__device__ __forceinline__ bool plane_cell(const Geo& g, int i0, int j0, int kk, int q, int* h) {
  const int a = q % PX, b = q / PX;
  const int ii = i0 - 1 + a, jj = j0 - 1 + b;
  *h = g.h(ii, jj, kk);
  return ii <= g.nx + 1 && jj <= g.ny + 1;
}

template <int TYV>
inline dim3 grid_of(const Geo& g, int kz) {
  using S = Shape<TYV>;
  return dim3((g.nx + S::TX - 1) / S::TX, (g.ny + S::TY - 1) / S::TY, (g.nz + kz - 1) / kz);
}

// the tile shape of a grid: 2 rows for ny <= 2, else 8
inline int rows_of(const Geo& g) { return g.ny <= 2 ? 2 : 8; }

// z levels per block; `slots`: blocks per SM that the split aims at (the
// ACDI and Youngs tiles 24, the momentum tile 48, measured at 256^3)
template <int TYV>
inline int kz_of(const Geo& g, int batched, int nsm, int slots = 24) {
  using S = Shape<TYV>;
  // in an ensemble the other cases keep the GPU busy: 32 levels per block
  // spend 6% on the two extra planes each block loads (25% at 8 levels)
  if (batched) return g.nz < 32 ? g.nz : 32;
  // several waves of resident blocks on each of the device's SMs (148 on a
  // B200), so the last partial wave costs little; at least 8 levels per
  // block (each block loads two planes and evaluates one face/vertex plane
  // beyond its own levels)
  const long long xy = (long long)((g.nx + S::TX - 1) / S::TX) * ((g.ny + S::TY - 1) / S::TY);
  long long kz = (xy * g.nz) / ((long long)(nsm > 0 ? nsm : 148) * slots);
  if (kz < 8) kz = 8;
  if (kz > 64) kz = 64;
  return (int)kz;
}

}  // namespace tile
}  // namespace cansfz
