// Horizontal batching of same-shape cases (the ensemble's case groups).
//
// Every step kernel's body is a static `run(const Blk&, args...)` of a small
// struct F; the named __global__ kernel calls it with its own block index.
// The batched form k_batch<F> runs the same body for several cases in one
// launch: the cases' argument lists lie in a device table, and grid z is
// the case's own grid z times the number of cases, so block
// (x, y, c*zper + z) runs block (x, y, z) of case c with case c's
// arguments.  The body sees exactly the arguments and block index of its
// single-case launch, so a batched launch computes bit for bit what the
// cases' own launches compute.
//
// Launch sites go through kgo(): with no recorder it launches the named
// kernel; with a recorder (Launch::rec) it stores the launch (batched kernel,
// grid, block, shared memory, argument bytes) instead.  The ensemble records
// one step of every case, groups cases whose records agree launch for launch,
// uploads the groups' argument tables and replays each group as batched
// launches.
#pragma once

#include <cstring>
#include <type_traits>
#include <utility>
#include <vector>

#include "cansfz_internal.cuh"

namespace cansfz {

// the block's position in its case's grid, and that grid's size
struct Blk {
  int x, y, z;
  int nx, ny, nz;
};
__device__ __forceinline__ Blk blk_here() {
  return Blk{(int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z, (int)gridDim.x, (int)gridDim.y, (int)gridDim.z};
}

// a flat, trivially copyable argument list
template <int I, class T>
struct PackLeaf {
  T v;
};
template <class S, class... A>
struct PackImpl;
template <int... I, class... A>
struct PackImpl<std::integer_sequence<int, I...>, A...> : PackLeaf<I, A>... {};
template <class... A>
using Pack = PackImpl<std::make_integer_sequence<int, sizeof...(A)>, A...>;

template <class F, int... I, class... A>
__device__ __forceinline__ void run_pack(const Blk& b, const PackImpl<std::integer_sequence<int, I...>, A...>& p) {
  F::run(b, static_cast<const PackLeaf<I, A>&>(p).v...);
}
template <int... I, class... A, class... V>
inline void fill_pack(PackImpl<std::integer_sequence<int, I...>, A...>& p, V&&... v) {
  ((static_cast<PackLeaf<I, A>&>(p).v = static_cast<A>(v)), ...);
}

// the argument types of F::run after the block index (structs that run
// takes by reference are stored by value)
template <class R>
struct RunArgs;
template <class... A>
struct RunArgs<void (*)(const Blk&, A...)> {
  using type = Pack<std::decay_t<A>...>;
};

template <class F, int NT, int MINB, class P>
__global__ void __launch_bounds__(NT, MINB) k_batch(const P* __restrict__ tab, int zper) {
  const int c = (int)blockIdx.z / zper;
  const Blk b{(int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z - c * zper, (int)gridDim.x, (int)gridDim.y, zper};
  run_pack<F>(b, tab[c]);
}

// ---------------------------------------------------------------------------
// host side: recorded launches
// ---------------------------------------------------------------------------
struct RecEntry {
  const void* key;  // the batched kernel (same key: same kernel and template arguments)
  dim3 grid, block;
  size_t smem;
  std::vector<unsigned char> args;
  // batched launch of n entries like this one whose argument lists lie at
  // `tab` (device memory, n * args.size() bytes, in case order)
  int (*launch)(const RecEntry& e, int n, const void* tab, cudaStream_t st);
  // opt the batched kernel into the entry's dynamic shared memory (outside capture)
  int (*prepare)(const RecEntry& e);
  bool same_launch(const RecEntry& o) const {
    return key == o.key && grid.x == o.grid.x && grid.y == o.grid.y && grid.z == o.grid.z &&
           block.x == o.block.x && block.y == o.block.y && block.z == o.block.z && smem == o.smem &&
           args.size() == o.args.size();
  }
};
struct Recorder {
  std::vector<RecEntry> e;
};

template <class F, int NT, int MINB, class P>
int batch_prepare(const RecEntry& e) {
  if (e.smem <= 48 * 1024) return 0;
  return cudaFuncSetAttribute(k_batch<F, NT, MINB, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)e.smem) == cudaSuccess ? 0 : 1;
}

template <class F, int NT, int MINB, class P>
int batch_launch(const RecEntry& e, int n, const void* tab, cudaStream_t st) {
  const int per = (int)(65535 / e.grid.z);  // grid z limit
  if (per < 1) return 1;
  const P* t = static_cast<const P*>(tab);
  for (int c0 = 0; c0 < n; c0 += per) {
    const int m = n - c0 < per ? n - c0 : per;
    k_batch<F, NT, MINB, P><<<dim3(e.grid.x, e.grid.y, e.grid.z * m), e.block, e.smem, st>>>(t + c0, (int)e.grid.z);
    if (cudaGetLastError() != cudaSuccess) return 1;
  }
  return 0;
}

// Launch F's named kernel `k` with `v...`, or record the launch when the
// Launch carries a recorder.  NT, MINB: the kernel's launch bounds.
template <class F, int NT, int MINB, class K, class... V>
inline void kgo(const Launch& L, K k, dim3 grid, dim3 block, size_t smem, V&&... v) {
  using P = typename RunArgs<decltype(&F::run)>::type;
  static_assert(alignof(P) <= 128, "argument tables align their entries to at most 128 bytes");
  if (L.rec) {
    P p;
    fill_pack(p, std::forward<V>(v)...);
    RecEntry e;
    e.key = reinterpret_cast<const void*>(k_batch<F, NT, MINB, P>);
    e.grid = grid;
    e.block = block;
    e.smem = smem;
    e.args.resize(sizeof(P));
    std::memcpy(e.args.data(), static_cast<const void*>(&p), sizeof(P));
    e.launch = &batch_launch<F, NT, MINB, P>;
    e.prepare = &batch_prepare<F, NT, MINB, P>;
    L.rec->e.push_back(std::move(e));
    return;
  }
  k<<<grid, block, smem, L.st>>>(std::forward<V>(v)...);
}

}  // namespace cansfz
