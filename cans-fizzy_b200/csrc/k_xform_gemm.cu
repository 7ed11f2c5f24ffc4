// Line transforms of the mixed form's FP32 spectral solve as dense GEMMs on
// the fifth-generation tensor cores (tcgen05, sm_100a).
//
// A real transform of length n along x or y is the product of the lines with
// an n x n matrix F (out[j] = sum_k F[j][k] in[k]): the periodic kind's
// packed real DFT (r0, r_{n/2}, r1, i1, ...) and its inverse, DCT-II/III and
// DST-II/III, the kinds and orders that the shared-memory FFTs of
// k_poisson.cu produce (src/fft.f90:244-269,491-567 and FFTW's r2r
// definitions, which the reference calls).  A dense matrix moves the same
// bytes as an FFT and needs no stage barriers; its 2n flops per point go to
// the tensor pipe.
//
// Precision: split BF16 with FP32 accumulation.  Every operand v is held as
// v_hi = bf16(v) and v_lo = bf16(v - v_hi); each product is
// A_hi B_hi + A_hi B_lo + A_lo B_hi (the A_lo B_lo term and the bits below
// v_lo are dropped), which leaves a relative error of ~2^-16 per transform.
// The mixed form's FP64-residual refinement (k_residual, 1-3 sweeps) wins
// the accuracy back; the FP32 spectral buffer and z solve are unchanged.
//
// Kernel structure (two persistent CTAs of 8 warps per SM, 128 lines per tile):
//   * the tile's 128 lines x n samples stream through shared memory in chunks
//     of 64 samples, one stage per CTA: while one CTA's chunk is on the
//     tensor cores the other CTA of the SM loads and splits its next one.  Each thread loads 32 samples of one
//     line (the next chunk's load is in flight while the tensor cores work on
//     the current one), splits them and stores them in the canonical K-major
//     layout of the MMA (8-row x 16-byte core matrices, no swizzle);
//   * the matching 64-column chunk of F (hi and lo, precomputed on the host
//     in the same layout) arrives by two bulk copies (cp.async.bulk) that
//     complete on an mbarrier;
//   * one thread issues 3 x 4 tcgen05.mma (M = 128, N = n, K = 16) per chunk
//     into an FP32 accumulator of n TMEM columns and commits them to the
//     stage's mbarrier, which frees the stage for the next chunk;
//   * after the last chunk, every warp reads 32 TMEM lanes (32 lines), half
//     of the columns, with tcgen05.ld and writes the outputs.
// Every mbarrier wait is bounded (about half a second); a wait that runs
// out marks the step scalars CANSFZ_ERR_TIMEOUT and halted, waits (bounded)
// for the CTA's copies and MMAs in flight, frees its TMEM and returns.
//
// The bulk copies read only this GPU's memory and use no cluster multicast.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "cansfz_internal.cuh"

namespace cansfz {

namespace {

constexpr int GM = 128;   // lines per tile (MMA M)
constexpr int GKC = 64;   // samples per K chunk
constexpr int GST = 1;    // stages per CTA (two CTAs share an SM and alternate)
constexpr int GTHREADS = 256;

__device__ __forceinline__ uint32_t su32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for the completion of phase `parity`: false after ~0.5 s
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try(bar, parity))
    if (clock64() - t0 > (1LL << 30)) return false;
  return true;
}
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// shared-memory matrix descriptor: K-major, no swizzle; LBO = byte distance
// of the core matrices adjacent in K, SBO = of those adjacent in M/N
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr & 0x3FFFF) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         (1ull << 46);  // descriptor version of sm_100
}
// instruction descriptor: BF16 x BF16 -> FP32, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}
__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
}

#define X32R(v)                                                                                                   \
  "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),    \
      "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),     \
      "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),    \
      "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
// 32 lanes x 32 consecutive FP32 columns: thread i of the warp gets lane
// (warp's quarter + i), columns col..col+31
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
      : X32R(v)
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

// the split of 8 consecutive samples of one line into the hi and lo core
// rows (16 bytes each) at byte offset `off` of the A stage
template <typename V>
__device__ __forceinline__ void split_store(unsigned char* ahi, unsigned char* alo, uint32_t off, const V (&v)[8]) {
  uint32_t h[4], l[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const __nv_bfloat16 h0 = __float2bfloat16_rn((float)v[2 * q]);
    const __nv_bfloat16 h1 = __float2bfloat16_rn((float)v[2 * q + 1]);
    const __nv_bfloat16 l0 = __float2bfloat16_rn((float)(v[2 * q] - (V)__bfloat162float(h0)));
    const __nv_bfloat16 l1 = __float2bfloat16_rn((float)(v[2 * q + 1] - (V)__bfloat162float(h1)));
    h[q] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
    l[q] = (uint32_t)__bfloat16_as_ushort(l0) | ((uint32_t)__bfloat16_as_ushort(l1) << 16);
  }
  *reinterpret_cast<uint4*>(ahi + off) = make_uint4(h[0], h[1], h[2], h[3]);
  *reinterpret_cast<uint4*>(alo + off) = make_uint4(l[0], l[1], l[2], l[3]);
}

}  // namespace

// MODE 0: x forward, lines (j,k) of an FP64 halo field -> FP32 spectral rows
// MODE 1: y pass, lines (x,z) of the FP32 spectral buffer, samples at stride
//         nx, in place
// MODE 2: x backward, FP32 spectral rows -> FP64 halo field, dst = normfft*v
//         (ADD: dst += normfft*v, a refinement correction)
struct GemmXform {
  const void* src;
  void* dst;
  const uint16_t* bmat;  // [n/64 chunks][hi, lo][n rows][64] in the core layout
  int n, nlines, ntiles;
  Geo g;
  double normfft;
};

// the 32 samples (four core rows) of one line that a thread stages per chunk
template <int MODE>
struct LineVals {
  using T = typename std::conditional<MODE == 0, double, float>::type;
  T v[32];
};

template <int MODE>
__device__ __forceinline__ void load_line(const GemmXform& p, bool live, size_t base, int l, int k0,
                                          LineVals<MODE>& x) {
  if (MODE == 0) {
    const double* sp = static_cast<const double*>(p.src) + base + k0;
#pragma unroll
    for (int q = 0; q < 32; ++q) x.v[q] = live ? __ldg(sp + q) : 0.;
  } else if (MODE == 1) {
    const float* sp = static_cast<const float*>(p.src) + base + (size_t)k0 * p.g.nx;
#pragma unroll
    for (int q = 0; q < 32; ++q) x.v[q] = live ? sp[(size_t)q * p.g.nx] : 0.f;
  } else {
    const float4* sp = reinterpret_cast<const float4*>(static_cast<const float*>(p.src) + (size_t)l * p.n + k0);
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 f = live ? sp[q] : make_float4(0.f, 0.f, 0.f, 0.f);
      x.v[4 * q] = f.x; x.v[4 * q + 1] = f.y; x.v[4 * q + 2] = f.z; x.v[4 * q + 3] = f.w;
    }
  }
}

template <int MODE, bool ADD>
__global__ void __launch_bounds__(GTHREADS, 2) k_xform_gemm(GemmXform p, DevScalars* sc) {
  if (sc != nullptr && sc->halted) return;
  extern __shared__ __align__(1024) unsigned char smem[];
  const int n = p.n, nkc = n / GKC;
  const uint32_t a_bytes = GM * GKC * 2, b_bytes = (uint32_t)n * GKC * 2;
  const uint32_t stage_bytes = 2 * a_bytes + 2 * b_bytes;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + GST * stage_bytes);  // full[2], done[2], acc, fin
  uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 8);
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t bfull[2] = {su32(bars + 0), su32(bars + 1)};
  const uint32_t bdone[2] = {su32(bars + 2), su32(bars + 3)};
  const uint32_t bacc = su32(bars + 4), bfin = su32(bars + 5);
  if (tid == 0) {
    for (int q = 0; q < 6; ++q) mbar_init(su32(bars + q), 1);
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  const uint32_t ncols = n <= 32 ? 32 : (n <= 64 ? 64 : (n <= 128 ? 128 : 256));
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(su32(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_before();
  __syncthreads();
  tc_after();
  const uint32_t tmem = *tslot;
  const uint32_t idesc = idesc_bf16(GM, n);
  const uint32_t lbo = 128, sbo = (GKC / 8) * 128;
  uint32_t ph_full[2] = {0, 0}, ph_done[2] = {0, 0}, ph_acc = 0;
  int used[2] = {0, 0}, inflight[2] = {0, 0};
  bool fail = false, issued = false;
  int gch = 0;
  // thread t stages half h = t / 128 (32 samples) of line r = t % 128 of the tile
  const int r = tid & (GM - 1), hh = tid / GM;
  const uint32_t arow = (uint32_t)((r >> 3) * (GKC / 8)) * 128 + (uint32_t)(r & 7) * 16 + (uint32_t)hh * 4 * 128;
  // the epilogue: warp w reads TMEM lanes 32*(w%4).. (its lines), columns of half w/4
  const int er = (warp & 3) * 32 + (tid & 31), ecol0 = (warp >> 2) * (n / 2);
  auto line_of = [&](int tile, int rr, bool& live, size_t& base) {
    const int l = tile * GM + rr;
    live = l < p.nlines;
    if (MODE == 0 || MODE == 2) {
      const int j = live ? l % p.g.ny : 0, k = live ? l / p.g.ny : 0;
      base = (size_t)p.g.h(1, j + 1, k + 1);
    } else {
      const int x = live ? l % p.g.nx : 0, z = live ? l / p.g.nx : 0;
      base = (size_t)z * p.g.nx * p.g.ny + x;
    }
    return l;
  };
  LineVals<MODE> x;
  bool live;
  size_t base;
  int l = line_of(blockIdx.x, r, live, base);
  if (blockIdx.x < p.ntiles) load_line<MODE>(p, live, base, l, hh * 32, x);  // first chunk in flight

  for (int tile = blockIdx.x; tile < p.ntiles; tile += gridDim.x) {
    for (int kc = 0; kc < nkc; ++kc, ++gch) {
      const int s = gch % GST;
      if (used[s]) {
        if (!mbar_wait(bdone[s], ph_done[s])) fail = true;
        ph_done[s] ^= 1;
      }
      used[s] = 1;
      if (__syncthreads_or(fail)) goto cleanup;
      unsigned char* st = smem + s * stage_bytes;
      unsigned char* ahi = st;
      unsigned char* alo = st + a_bytes;
      unsigned char* bhi = st + 2 * a_bytes;
      unsigned char* blo = bhi + b_bytes;
      if (tid == 0) {
        mbar_expect_tx(bfull[s], 2 * b_bytes);
        const unsigned char* bsrc = reinterpret_cast<const unsigned char*>(p.bmat) + (size_t)kc * 2 * b_bytes;
        bulk_g2s(su32(bhi), bsrc, b_bytes, bfull[s]);
        bulk_g2s(su32(blo), bsrc + b_bytes, b_bytes, bfull[s]);
        inflight[s] = 1;
      }
#pragma unroll
      for (int g = 0; g < 4; ++g) {
        typename LineVals<MODE>::T v8[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v8[q] = x.v[8 * g + q];
        split_store(ahi, alo, arow + (uint32_t)g * 128, v8);
      }
      fence_async_smem();
      __syncthreads();
      // the next chunk's samples (or the next tile's first) load while the
      // tensor cores work on this one
      {
        const bool last = kc == nkc - 1;
        const int nt = last ? tile + (int)gridDim.x : tile;
        if (nt < p.ntiles) {
          if (last) l = line_of(nt, r, live, base);
          load_line<MODE>(p, live, base, l, (last ? 0 : (kc + 1) * GKC) + hh * 32, x);
        }
      }
      if (tid == 0) {
        if (!mbar_wait(bfull[s], ph_full[s])) {
          fail = true;
        } else {
          inflight[s] = 0;
          ph_full[s] ^= 1;
          tc_after();
#pragma unroll
          for (int kk = 0; kk < GKC / 16; ++kk) {
            const uint32_t ko = (uint32_t)kk * 2 * 128;
            const uint64_t dah = sdesc(su32(ahi) + ko, lbo, sbo), dal = sdesc(su32(alo) + ko, lbo, sbo);
            const uint64_t dbh = sdesc(su32(bhi) + ko, lbo, sbo), dbl = sdesc(su32(blo) + ko, lbo, sbo);
            mma_bf16(tmem, dah, dbh, idesc, (kc | kk) != 0 ? 1u : 0u);
            mma_bf16(tmem, dah, dbl, idesc, 1u);
            mma_bf16(tmem, dal, dbh, idesc, 1u);
          }
          issued = true;
          mma_commit(bdone[s]);
          if (kc == nkc - 1) mma_commit(bacc);
        }
      }
    }
    // the tile's accumulator: each warp reads its 32 lanes, half the columns
    if (!mbar_wait(bacc, ph_acc)) fail = true;
    ph_acc ^= 1;
    if (__syncthreads_or(fail)) goto cleanup;
    tc_after();
    {
      bool elive;
      size_t ebase;
      const int el = line_of(tile, er, elive, ebase);
      // x passes: a line's outputs are contiguous, so each warp turns its
      // 32 lines x 32 columns around in shared memory (the stages are idle
      // now) and writes line by line, 32 consecutive columns per store
      float* tb = reinterpret_cast<float*>(smem) + warp * (32 * 33);
      const int lane = tid & 31;
      for (int c0 = ecol0; c0 < ecol0 + n / 2; c0 += 32) {
        uint32_t v[32];
        tmem_ld32(tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)c0, v);
        if (MODE == 1) {
          if (!elive) continue;
          float* dp = static_cast<float*>(p.dst) + ebase + (size_t)c0 * p.g.nx;
#pragma unroll
          for (int q = 0; q < 32; ++q) dp[(size_t)q * p.g.nx] = __uint_as_float(v[q]);
        } else {
#pragma unroll
          for (int q = 0; q < 32; ++q) tb[lane * 33 + q] = __uint_as_float(v[q]);
          __syncwarp();
          const int lr0 = (warp & 3) * 32;
          for (int i = 0; i < 32; ++i) {
            bool li;
            size_t bi;
            const int ll = line_of(tile, lr0 + i, li, bi);
            if (!li) continue;
            const float val = tb[i * 33 + lane];
            if (MODE == 0) {
              static_cast<float*>(p.dst)[(size_t)ll * n + c0 + lane] = val;
            } else {
              double* dp = static_cast<double*>(p.dst) + bi + c0 + lane;
              const double xv = (double)val * p.normfft;
              *dp = ADD ? *dp + xv : xv;
            }
          }
          __syncwarp();
        }
      }
      (void)el;
    }
    tc_before();
    __syncthreads();
  }
cleanup:
  if (tid == 0) {
    // the CTA's bulk copies and MMAs in flight complete before it exits
    for (int s = 0; s < 2; ++s)
      if (inflight[s]) {
        mbar_wait(bfull[s], ph_full[s]);
        inflight[s] = 0;
      }
    if (issued) {
      mma_commit(bfin);
      mbar_wait(bfin, 0);
    }
    if (fail && sc != nullptr) {
      atomicCAS(&sc->status, CANSFZ_OK, CANSFZ_ERR_TIMEOUT);
      sc->halted = 1;
    }
  }
  tc_before();
  __syncthreads();
  tc_after();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(ncols) : "memory");
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// F[j][k] of one transform (out[j] = sum_k F[j][k] in[k]) in the orders of the
// FFT kernels: kind 0 the packed real DFT (r0, r_{n/2}, r1, i1, ...; FFTW's
// R2HC values) and its unnormalised inverse (HC2R); kind 1 REDFT10 / REDFT01;
// kind 2 RODFT10 / RODFT01 (FFTW's definitions; dir > 0 forward)
double xform_coef(int kind, int dir, int n, int j, int k) {
  const double pi = 3.14159265358979323846264338327950288;
  if (kind == 0) {
    const int h = n / 2;
    if (dir > 0) {
      const int m = j == 0 ? 0 : (j == 1 ? h : j / 2);
      const bool im = j > 1 && (j & 1);
      const double ang = 2. * pi * (double)(((long long)m * k) % n) / (double)n;
      return im ? -std::sin(ang) : std::cos(ang);
    }
    if (k == 0) return 1.;
    if (k == 1) return (j & 1) ? -1. : 1.;
    const int m = k / 2;
    const double ang = 2. * pi * (double)(((long long)m * j) % n) / (double)n;
    return (k & 1) ? -2. * std::sin(ang) : 2. * std::cos(ang);
  }
  if (kind == 1) {
    if (dir > 0) return 2. * std::cos(pi * (double)j * (2. * k + 1.) / (2. * n));
    return k == 0 ? 1. : 2. * std::cos(pi * (double)k * (2. * j + 1.) / (2. * n));
  }
  if (dir > 0) return 2. * std::sin(pi * (double)(j + 1) * (2. * k + 1.) / (2. * n));
  if (k == n - 1) return (j & 1) ? -1. : 1.;
  return 2. * std::sin(pi * (double)(k + 1) * (2. * j + 1.) / (2. * n));
}

namespace {
// round-to-nearest-even of an FP32 value to its upper 16 bits (bf16)
uint16_t bf16_bits(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
float bf16_value(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}
}  // namespace

// the transform's matrix as the kernel's B operand: for each 64-sample chunk
// the hi then the lo part of F[0..n)[chunk], n rows x 64 in core matrices of
// 8 rows x 8 bf16 (rows of a core matrix 16 bytes apart, core matrices
// along K 128 bytes apart, 8-row groups (64/8)*128 bytes apart)
std::vector<uint16_t> xform_bmat(int kind, int dir, int n) {
  const int nkc = n / GKC;
  std::vector<uint16_t> out((size_t)nkc * 2 * n * GKC);
  for (int kc = 0; kc < nkc; ++kc)
    for (int j = 0; j < n; ++j)
      for (int kk = 0; kk < GKC; ++kk) {
        const double f = xform_coef(kind, dir, n, j, kc * GKC + kk);
        const uint16_t hi = bf16_bits((float)f);
        const uint16_t lo = bf16_bits((float)(f - (double)bf16_value(hi)));
        const size_t core = (size_t)((j >> 3) * (GKC / 8) + (kk >> 3)) * 64 + (size_t)(j & 7) * 8 + (kk & 7);
        out[(size_t)kc * 2 * n * GKC + core] = hi;
        out[(size_t)kc * 2 * n * GKC + (size_t)n * GKC + core] = lo;
      }
  return out;
}

bool xform_gemm_length(int n) { return n == 64 || n == 128 || n == 256; }

size_t xform_gemm_smem(int n) { return (size_t)GST * (2 * GM * GKC * 2 + 2 * (size_t)n * GKC * 2) + 8 * 8 + 16; }

template <int MODE, bool ADD>
static int set_attr_one(int n) {
  return cudaFuncSetAttribute(k_xform_gemm<MODE, ADD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)xform_gemm_smem(n)) == cudaSuccess ? 0 : 1;
}
int xform_gemm_set_attributes() {
  return set_attr_one<0, false>(256) | set_attr_one<1, false>(256) | set_attr_one<2, false>(256) |
         set_attr_one<2, true>(256);
}

// one pass: mode 0 x forward (src: FP64 halo field, dst: FP32 rows), 1 y
// (src = dst: FP32 spectral buffer), 2 x backward (src: FP32 rows, dst: FP64
// halo field, `add`: accumulate)
void launch_xform_gemm(const Launch& L, const Geo& g, int mode, bool add, const uint16_t* bmat, int n,
                       const void* src, void* dst, double normfft, DevScalars* sc) {
  GemmXform p{};
  p.src = src;
  p.dst = dst;
  p.bmat = bmat;
  p.n = n;
  p.nlines = mode == 1 ? g.nx * g.nz : g.ny * g.nz;
  p.ntiles = (p.nlines + GM - 1) / GM;
  p.g = g;
  p.normfft = normfft;
  const int nsm = 2 * (L.nsm > 0 ? L.nsm : 148);  // two CTAs per SM
  const dim3 grid(p.ntiles < nsm ? p.ntiles : nsm);
  const size_t smem = xform_gemm_smem(n);
  if (mode == 0) k_xform_gemm<0, false><<<grid, GTHREADS, smem, L.st>>>(p, sc);
  else if (mode == 1) k_xform_gemm<1, false><<<grid, GTHREADS, smem, L.st>>>(p, sc);
  else if (add) k_xform_gemm<2, true><<<grid, GTHREADS, smem, L.st>>>(p, sc);
  else k_xform_gemm<2, false><<<grid, GTHREADS, smem, L.st>>>(p, sc);
}

}  // namespace cansfz

extern "C" int cansfz_xform_matrix(int kind, int dir, int n, double* F) {
  if (!F || kind < 0 || kind > 2 || dir == 0 || n < 2 || (kind == 0 && (n & 1))) return CANSFZ_ERR_ARG;
  for (int j = 0; j < n; ++j)
    for (int k = 0; k < n; ++k) F[(size_t)j * n + k] = cansfz::xform_coef(kind, dir, n, j, k);
  return CANSFZ_OK;
}
