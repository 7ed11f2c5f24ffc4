// Allocation-free Poisson solve: cansfz_solver_static.
//
// Some callers cannot allocate device memory while they run the solver.
//
// * A driver whose device memory is owned by another runtime hands out
//   only buffers carved from that runtime's pool. An OpenACC data region is
//   one example; a memory-budgeted host application is another.
// * Code that must not trigger the implicit device-wide synchronisation a
//   cudaMalloc/cudaFree can cause, such as a solve issued from a callback or
//   between asynchronous stages that must stay overlapped.
//
// For them this file keeps the solver's scratch in file-scope device arrays
// of a fixed maximum size: the spectral work buffer and the twiddle tables.
// Every GPU that loads the library holds these arrays until the process
// exits (16 MiB + 64 KiB per device).  The caller passes the inputs and the
// output: the right-hand side (in place in p), the eigenvalues and the z
// coefficients.  No cudaMalloc, cudaFree or allocating library routine is
// called.
//
// Set-up: the first call on a device (that device current) resolves the
// device addresses of the arrays with cudaGetSymbolAddress and opts the
// transform kernels into their shared-memory size.  Make that first call
// before any stream capture on the device.  All calls share the arrays and
// keep the last call's contents; calls whose kernels overlap on the GPU
// (different streams, no ordering between them) race on them.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "cansfz_internal.cuh"

namespace {

constexpr size_t kMaxCells = (size_t)128 * 128 * 128;  // 2,097,152 cells of FP64 scratch: 16 MiB
constexpr int kMaxLine = 1024;                          // longest x or y transform
// longest z column: the z solve keeps one FP64 pivot checkpoint per 16
// levels for each of its 64 columns in shared memory (32 bytes per level),
// which must fit the 48 KiB a kernel gets without opting in
constexpr int kMaxZ = 1536;

static __device__ __align__(256) double g_scratch[kMaxCells];
static __device__ __align__(256) double2 g_tw[2][kMaxLine / 2];
static __device__ __align__(256) double2 g_tw2[2][kMaxLine / 2 + 1];
static __device__ __align__(256) double2 g_twc[2][kMaxLine + 1];

struct DeviceSyms {
  bool ready = false;
  double* scratch = nullptr;
  double2* tw = nullptr;
  double2* tw2 = nullptr;
  double2* twc = nullptr;
};
constexpr int kMaxDevices = 64;
DeviceSyms g_syms[kMaxDevices];
std::mutex g_mu;

// once per device, with that device current
int setup_device(int dev) {
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceSyms& s = g_syms[dev];
  if (s.ready) return CANSFZ_OK;
  if (cudaGetSymbolAddress((void**)&s.scratch, g_scratch) != cudaSuccess) return CANSFZ_ERR_CUDA;
  if (cudaGetSymbolAddress((void**)&s.tw, g_tw) != cudaSuccess) return CANSFZ_ERR_CUDA;
  if (cudaGetSymbolAddress((void**)&s.tw2, g_tw2) != cudaSuccess) return CANSFZ_ERR_CUDA;
  if (cudaGetSymbolAddress((void**)&s.twc, g_twc) != cudaSuccess) return CANSFZ_ERR_CUDA;
  cansfz::poisson_set_attributes();
  if (cudaPeekAtLastError() != cudaSuccess) return CANSFZ_ERR_CUDA;
  s.ready = true;
  return CANSFZ_OK;
}

// twiddles of one line transform (d = 0: x, 1: y) written into the static tables
__global__ void k_twiddles(int d, int n, double2* tw, double2* tw2, double2* twc) {
  const int m = n / 2;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q <= n; q += gridDim.x * blockDim.x) {
    double s, c;
    if (q < m) {
      sincospi(-2.0 * q / m, &s, &c);
      tw[d * (kMaxLine / 2) + q] = make_double2(c, s);
    }
    if (q <= m) {
      sincospi(-2.0 * q / n, &s, &c);
      tw2[d * (kMaxLine / 2 + 1) + q] = make_double2(c, s);
    }
    sincospi(-(double)q / (2.0 * n), &s, &c);
    twc[d * (kMaxLine + 1) + q] = make_double2(c, s);
  }
}

int kind_of(const char c[2]) {
  if (c[0] == 'P' && c[1] == 'P') return 0;
  if (c[0] == 'N' && c[1] == 'N') return 1;
  if (c[0] == 'D' && c[1] == 'D') return 2;
  return -1;
}

bool radix_plan(int m, int radix[FFT_MAXSTAGES], int* nst) {
  int k = 0;
  while (m % 4 == 0 && m > 4) { radix[k++] = 4; m /= 4; }
  for (int r : {4, 2, 3, 5, 7}) while (m % r == 0 && k < FFT_MAXSTAGES) { radix[k++] = r; m /= r; }
  *nst = k;
  return m == 1;
}

}  // namespace

extern "C" int cansfz_solver_static(const int n[3], const char cbc[3][2], double normfft, const double* lambdaxy,
                                    const double* a, const double* b, const double* c, double* p, void* stream) {
  if (!n || !cbc || !lambdaxy || !a || !b || !c || !p) return CANSFZ_ERR_ARG;
  const int nx = n[0], ny = n[1], nz = n[2];
  if (nx < 2 || ny < 2 || nz < 2 || (nx & 1) || (ny & 1)) return CANSFZ_ERR_ARG;
  // sizes beyond the static scratch, or beyond what the kernels launch
  // with, are rejected before anything is launched
  if ((size_t)nx * ny * nz > kMaxCells || nx > kMaxLine || ny > kMaxLine || nz > kMaxZ) return CANSFZ_ERR_ARG;
  const int kx = kind_of(cbc[0]), ky = kind_of(cbc[1]);
  if (kx < 0 || ky < 0) return CANSFZ_ERR_UNSUPPORTED;
  if (cbc[2][0] == 'P' || cbc[2][1] == 'P') return CANSFZ_ERR_UNSUPPORTED;  // periodic z needs a second buffer
  // an error left pending by the caller's earlier work is reported before
  // this call launches anything (and left pending for the caller)
  if (cudaPeekAtLastError() != cudaSuccess) return CANSFZ_ERR_CUDA;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return CANSFZ_ERR_CUDA;
  if (int rc = setup_device(dev)) return rc;
  const DeviceSyms& s = g_syms[dev];
  cudaStream_t st = (cudaStream_t)stream;

  cansfz::PoissonPlan pl{};
  cansfz::LinePlan* lps[2] = {&pl.px, &pl.py};
  const int ns[2] = {nx, ny}, kinds[2] = {kx, ky};
  for (int d = 0; d < 2; ++d) {
    cansfz::LinePlan& lp = *lps[d];
    lp.n = ns[d];
    lp.kind = kinds[d];
    lp.m = ns[d] / 2;
    if (!radix_plan(lp.m, lp.radix, &lp.nst)) return CANSFZ_ERR_UNSUPPORTED;
    lp.tw = s.tw + d * (kMaxLine / 2);
    lp.tw2 = s.tw2 + d * (kMaxLine / 2 + 1);
    lp.twc = s.twc + d * (kMaxLine + 1);
    k_twiddles<<<4, 256, 0, st>>>(d, ns[d], s.tw, s.tw2, s.twc);
    if (cudaGetLastError() != cudaSuccess) return CANSFZ_ERR_CUDA;
  }
  pl.lam = lambdaxy;
  pl.a = a;
  pl.b = b;
  pl.c = c;
  pl.normfft = normfft;
  pl.zper = 0;
  pl.work = s.scratch;

  cansfz::Geo g{};
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.sx = nx + 2; g.sxy = (nx + 2) * (ny + 2);
  cansfz::Launch L{st, 0, 0};
  cansfz::launch_poisson(L, g, pl, nullptr, p);
  return cudaGetLastError() == cudaSuccess ? CANSFZ_OK : CANSFZ_ERR_CUDA;
}
