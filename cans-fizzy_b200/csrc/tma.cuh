// Tensor-memory-accelerator (TMA) plane loads and mbarriers for the
// z-marching tile kernels (sm_100a).
//
// A halo-layout FP64 field a(0:nx+1, 0:ny+1, 0:nz+1) is described once per
// launch by a 3-D tensor map (dims nx+2, ny+2, nz+2; byte strides 8*sx and
// 8*sxy).  One thread of a block loads a whole tile plane (the block's 32 x TY
// cells plus the one-cell halo: 34 x (TY+2) values) with one
// cp.async.bulk.tensor per field; the copies complete on an mbarrier of the
// plane's ring slot, on which every thread of the block waits.  Points beyond
// the array (beyond index nx+1 or ny+1) read as zero, as the element-wise
// copies they replace did.  The plane's x origin i0-1 = 32*bx is a multiple of
// 2 doubles (16 bytes), the alignment a tiled copy needs.  Copies read this
// GPU's memory only and use no cluster multicast.
#pragma once

#include <cuda.h>

#include "cansfz_internal.cuh"

namespace cansfz {

// the tensor maps of one launch's staged fields (kernel parameter, or an
// entry of a batched launch's argument table; 64-byte aligned either way)
struct alignas(64) HaloMaps {
  CUtensorMap m[11];
};

// host: encode the map of a halo-layout FP64 field with a box of bx x by x 1
// values; false when the driver entry point is missing or the encoding fails
bool make_halo_map(CUtensorMap* m, const void* base, const Geo& g, int bx, int by);

#ifdef __CUDACC__
namespace tma {

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(su32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void bar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void bar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(su32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(su32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for the completion of phase `parity`: false after ~0.5 s
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!bar_try(bar, parity))
    if (clock64() - t0 > (1LL << 30)) return false;
  return true;
}
// one box of a 3-D tensor map at element coordinates (x, y, z) into shared
// memory at dst (16-byte aligned), completing on bar
__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];\n" ::"r"(su32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(su32(bar))
      : "memory");
}

}  // namespace tma
#endif

}  // namespace cansfz
