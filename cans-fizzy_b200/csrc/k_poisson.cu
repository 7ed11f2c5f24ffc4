// Constant-coefficient Poisson solve of solver_gpu (src/solver_gpu.f90:31-163)
// on one GPU, 1x1 pencil.  No transposes: the x lines are contiguous rows,
// the y lines are read as column tiles of TL consecutive x positions, and the
// z tridiagonal systems are solved one column per thread.
//
//   x: real transform of each row    (R2HC packed / DCT-II / DST-II)
//   y: real transform of each column (same kinds, per BC)
//   z: Thomas per (x,y) mode with b + lambda_x + lambda_y (gaussel_gpu,
//      src/solver_gpu.f90:165-230), Sherman-Morrison for periodic z
//      (gaussel_periodic_gpu, :232-370)
//   y, x: inverse transforms; x inverse scales by normfft and writes (or,
//      for a refinement correction, adds to) the interior of a halo field.
//
// Line transforms: a complex FFT of length m = n/2 (the real sequence packed
// as z_j = x_2j + i x_2j+1), Stockham auto-sort, radix 4/2/3 (generic radix
// via the twiddle table), in shared memory laid out position-major /
// line-minor so that consecutive threads touch consecutive lines.  The
// periodic kind stores the spectrum as (r0, r_{n/2}, r1, i1, r2, i2, ...);
// the eigenvalues are permuted to that order on the host.  The cosine and
// sine kinds follow Makhoul's reordering (as src/fft.f90:320-658 does).
//
// Every transform kernel is a template on the precision T of the spectral
// data: T = double is the drop-in FP64 solve; T = float is the spectral
// solve of the mixed form, whose accuracy an FP64 residual refinement wins
// back (launch_poisson_mixed).
#include "batch.cuh"

namespace cansfz {

#define HALTED(sc) ((sc) != nullptr && (sc)->halted)

template <typename T> struct CT;
template <> struct CT<double> { using t = double2; };
template <> struct CT<float> { using t = float2; };
template <typename T> using cx = typename CT<T>::t;

template <typename T> __device__ __forceinline__ cx<T> mk(T a, T b) { cx<T> r; r.x = a; r.y = b; return r; }
template <typename T> __device__ __forceinline__ cx<T> cmul(cx<T> a, cx<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T> __device__ __forceinline__ cx<T> cadd(cx<T> a, cx<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ cx<T> csub(cx<T> a, cx<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T> __device__ __forceinline__ cx<T> cconj(cx<T> a) { return mk<T>(a.x, -a.y); }
template <typename T> __device__ __forceinline__ cx<T> mul_i(cx<T> a) { return mk<T>(-a.y, a.x); }  // i*a

// twiddle tables in the transform precision
template <typename T> __device__ __forceinline__ cx<T> TW(const LinePlan& pl, int q);
template <> __device__ __forceinline__ double2 TW<double>(const LinePlan& pl, int q) { return __ldg(&pl.tw[q]); }
template <> __device__ __forceinline__ float2 TW<float>(const LinePlan& pl, int q) { return __ldg(&pl.twf[q]); }
template <typename T> __device__ __forceinline__ cx<T> TW2(const LinePlan& pl, int q);
template <> __device__ __forceinline__ double2 TW2<double>(const LinePlan& pl, int q) { return __ldg(&pl.tw2[q]); }
template <> __device__ __forceinline__ float2 TW2<float>(const LinePlan& pl, int q) { return __ldg(&pl.tw2f[q]); }
template <typename T> __device__ __forceinline__ cx<T> TWC(const LinePlan& pl, int q);
template <> __device__ __forceinline__ double2 TWC<double>(const LinePlan& pl, int q) { return __ldg(&pl.twc[q]); }
template <> __device__ __forceinline__ float2 TWC<float>(const LinePlan& pl, int q) { return __ldg(&pl.twcf[q]); }

template <typename T>
struct Bufs {
  T* re[2];
  T* im[2];
  int LP;  // line pitch in shared memory (odd: conflict-free strided access)
};

template <typename T> __device__ __forceinline__ cx<T> ld2(const Bufs<T>& B, int b, int pos, int line) {
  const int q = pos * B.LP + line;
  return mk<T>(B.re[b][q], B.im[b][q]);
}
template <typename T> __device__ __forceinline__ void st2(const Bufs<T>& B, int b, int pos, int line, cx<T> v) {
  const int q = pos * B.LP + line;
  B.re[b][q] = v.x;
  B.im[b][q] = v.y;
}
// raw real position s of a line stored as complex pairs (s even: re, odd: im)
template <typename T> __device__ __forceinline__ T ldr(const Bufs<T>& B, int b, int s, int line) {
  const int q = (s >> 1) * B.LP + line;
  return (s & 1) ? B.im[b][q] : B.re[b][q];
}
template <typename T> __device__ __forceinline__ void str(const Bufs<T>& B, int b, int s, int line, T v) {
  const int q = (s >> 1) * B.LP + line;
  if (s & 1) B.im[b][q] = v; else B.re[b][q] = v;
}

// complex FFT (sign -1 forward, +1 backward) of length pl.m on L lines held
// in buffer `in`; returns the buffer index holding the result.
// MC > 0: the complex length is the compile-time constant MC and LC the
// compile-time lines per CTA; the radix plan is the host's (radix 4 while
// the rest is a multiple of 4 above 4, then 4, 2, 3, 5, 7 in turn), so every
// stage's radix, length and stride -- and with them every index division
// below -- fold into constants.
__host__ __device__ constexpr int plan_radix(int m, int st) {
  int k = 0;
  while (m % 4 == 0 && m > 4) {
    if (k == st) return 4;
    m /= 4;
    ++k;
  }
  const int rs[5] = {4, 2, 3, 5, 7};
  for (int q = 0; q < 5; ++q)
    while (m % rs[q] == 0) {
      if (k == st) return rs[q];
      m /= rs[q];
      ++k;
    }
  return 1;
}
__host__ __device__ constexpr int plan_nst(int m) {
  int k = 0;
  while (plan_radix(m, k) > 1) ++k;
  return k;
}

// one Stockham stage of radix r on L lines: buffer cur -> cur^1
template <typename T>
__device__ __forceinline__ void fft_stage(const LinePlan& pl, const Bufs<T>& B, int cur, int L, int sign, int m,
                                          int r, int len, int s) {
    const int mm = len / r;
    const int tstep = m / len;  // exp(-2 pi i p u / len) = tw[p*u*tstep]
    const int nb = m / r;       // butterflies per line (= mm * s)
    const int nxt = cur ^ 1;
    for (int it = threadIdx.x; it < L * nb; it += blockDim.x) {
      const int line = it % L, b = it / L;
      const int p = b / s, q = b - p * s;
      auto put = [&](int u, cx<T> y) {
        if (u > 0 && p > 0) {
          cx<T> wp = TW<T>(pl, (p * u * tstep) % m);
          if (sign > 0) wp = cconj<T>(wp);
          y = cmul<T>(y, wp);
        }
        st2<T>(B, nxt, q + s * (r * p + u), line, y);
      };
      if (r == 2) {
        const cx<T> a0 = ld2<T>(B, cur, q + s * p, line), a1 = ld2<T>(B, cur, q + s * (p + mm), line);
        put(0, cadd<T>(a0, a1));
        put(1, csub<T>(a0, a1));
      } else if (r == 4) {
        const cx<T> a0 = ld2<T>(B, cur, q + s * p, line), a1 = ld2<T>(B, cur, q + s * (p + mm), line);
        const cx<T> a2 = ld2<T>(B, cur, q + s * (p + 2 * mm), line), a3 = ld2<T>(B, cur, q + s * (p + 3 * mm), line);
        const cx<T> t0 = cadd<T>(a0, a2), t1 = csub<T>(a0, a2), t2 = cadd<T>(a1, a3), t3 = csub<T>(a1, a3);
        // W4 = exp(sign * i pi / 2) = sign * i
        const cx<T> it3 = sign < 0 ? mk<T>(t3.y, -t3.x) : mk<T>(-t3.y, t3.x);  // W4 * t3
        put(0, cadd<T>(t0, t2));
        put(1, cadd<T>(t1, it3));
        put(2, csub<T>(t0, t2));
        put(3, csub<T>(t1, it3));
      } else if (r == 3) {
        const cx<T> a0 = ld2<T>(B, cur, q + s * p, line), a1 = ld2<T>(B, cur, q + s * (p + mm), line);
        const cx<T> a2 = ld2<T>(B, cur, q + s * (p + 2 * mm), line);
        const cx<T> t1 = cadd<T>(a1, a2), t2 = csub<T>(a1, a2);
        const T c3 = (T)0.86602540378443864676 * (T)(-sign);  // -sign*sqrt(3)/2
        const cx<T> base = mk<T>(a0.x - (T)0.5 * t1.x, a0.y - (T)0.5 * t1.y);
        const cx<T> rot = mk<T>(c3 * t2.y, -c3 * t2.x);  // -i * c3 * t2
        put(0, cadd<T>(a0, t1));
        put(1, cadd<T>(base, rot));
        put(2, csub<T>(base, rot));
      } else {
        // generic radix (5, 7): direct r-point DFT with the twiddle table
        for (int u = 0; u < r; ++u) {
          cx<T> acc = mk<T>(0, 0);
          for (int v = 0; v < r; ++v) {
            cx<T> wv = TW<T>(pl, ((v * u) % r) * (m / r));
            if (sign > 0) wv = cconj<T>(wv);
            acc = cadd<T>(acc, cmul<T>(ld2<T>(B, cur, q + s * (p + v * mm), line), wv));
          }
          put(u, acc);
        }
      }
    }
}

template <typename T, int MC, int ST, int NST, int LEN, int S>
__device__ __forceinline__ void fft_stages_c(const LinePlan& pl, const Bufs<T>& B, int& cur, int L, int sign) {
  if constexpr (ST < NST) {
    constexpr int r = plan_radix(MC, ST);
    fft_stage<T>(pl, B, cur, L, sign, MC, r, LEN, S);
    __syncthreads();
    cur ^= 1;
    fft_stages_c<T, MC, ST + 1, NST, LEN / r, S * r>(pl, B, cur, L, sign);
  }
}

template <typename T, int MC, int LC>
__device__ int fft_lines(const LinePlan& pl, const Bufs<T>& B, int in, int Lrt, int sign) {
  const int L = LC ? LC : Lrt;
  int cur = in;
  if constexpr (MC > 0) {
    fft_stages_c<T, MC, 0, plan_nst(MC), MC, 1>(pl, B, cur, L, sign);
  } else {
    const int m = pl.m;
    int len = m, s = 1;
    for (int st = 0; st < pl.nst; ++st) {
      const int r = pl.radix[st];
      fft_stage<T>(pl, B, cur, L, sign, m, r, len, s);
      __syncthreads();
      cur ^= 1;
      len /= r;
      s *= r;
    }
  }
  return cur;
}

// post-processing of a forward real transform: X_k, k = 0..m, from Z
template <typename T>
__device__ __forceinline__ cx<T> real_fwd_X(const LinePlan& pl, const Bufs<T>& B, int zb, int k, int line, int m) {
  const cx<T> zk = ld2<T>(B, zb, k % m, line);
  const cx<T> zc = cconj<T>(ld2<T>(B, zb, (m - k) % m, line));
  const cx<T> w = TW2<T>(pl, k);
  const cx<T> sum = mk<T>((T)0.5 * (zk.x + zc.x), (T)0.5 * (zk.y + zc.y));
  const cx<T> dif = csub<T>(zk, zc);
  const cx<T> wd = cmul<T>(w, dif);
  // -i/2 * wd = (0.5*wd.y, -0.5*wd.x)
  return mk<T>(sum.x + (T)0.5 * wd.y, sum.y - (T)0.5 * wd.x);
}

// Z_k = (X_k + conj X_{m-k}) + i (X_k - conj X_{m-k}) conj(W^k), k = 0..m-1
template <typename T>
__device__ __forceinline__ cx<T> real_bwd_Z(const LinePlan& pl, cx<T> xk, cx<T> xmk, int k) {
  const cx<T> xc = cconj<T>(xmk);
  const cx<T> w = cconj<T>(TW2<T>(pl, k));
  return cadd<T>(cadd<T>(xk, xc), mul_i<T>(cmul<T>(csub<T>(xk, xc), w)));
}

// packed spectrum of the periodic kind: complex index k -> X_k with
// X_0 = (r0, 0), X_m = (r_m, 0) both held in complex slot 0
template <typename T>
__device__ __forceinline__ cx<T> packed_X(const Bufs<T>& B, int b, int k, int m, int line) {
  if (k == 0) return mk<T>(B.re[b][line], 0);
  if (k == m) return mk<T>(B.im[b][line], 0);
  return ld2<T>(B, b, k, line);
}

// ---------------------------------------------------------------------------
// the four line transforms on L lines already in shared memory
// ---------------------------------------------------------------------------
// forward: input real line in buffer 0 as pairs (x_2j, x_2j+1) (after the
// kind's input reordering); output real line written through `out(line, s, v)`
template <typename T, bool LF, int MC, int LC, typename OUT>
__device__ void line_forward(const LinePlan& pl, const Bufs<T>& B, int Lrt, OUT out) {
  const int m = MC ? MC : pl.m, n = MC ? 2 * MC : pl.n;
  const int L = LC ? LC : Lrt;
  const int zb = fft_lines<T, MC, LC>(pl, B, 0, L, -1);
  if (pl.kind == 0) {
    for (int it = threadIdx.x; it < L * m; it += blockDim.x) {
      const int line = LF ? it % L : it / m, k = LF ? it / L : it - line * m;
      const cx<T> X = real_fwd_X<T>(pl, B, zb, k, line, m);
      if (k == 0) {
        const cx<T> Xm = real_fwd_X<T>(pl, B, zb, m, line, m);
        out(line, 0, X.x);
        out(line, 1, Xm.x);
      } else {
        out(line, 2 * k, X.x);
        out(line, 2 * k + 1, X.y);
      }
    }
  } else {
    const bool dst = pl.kind == 2;
    for (int it = threadIdx.x; it < L * (m + 1); it += blockDim.x) {
      const int line = LF ? it % L : it / (m + 1), k = LF ? it / L : it - line * (m + 1);
      const cx<T> V = real_fwd_X<T>(pl, B, zb, k, line, m);
      const cx<T> wk = TWC<T>(pl, k);
      const T yk = (T)2 * (wk.x * V.x - wk.y * V.y);
      if (k < n) out(line, dst ? n - 1 - k : k, yk);
      if (k > 0 && k < m) {
        const cx<T> wn = TWC<T>(pl, n - k);
        const T ynk = (T)2 * (wn.x * V.x + wn.y * V.y);  // Re(w_{n-k} conj(V_k))
        out(line, dst ? k - 1 : n - k, ynk);
      }
    }
  }
}

// backward: input real line (packed spectrum or natural DCT/DST coefficients)
// in buffer 1 as pairs; output real line through `out(line, i, v)`
template <typename T, bool LF, int MC, int LC, typename OUT>
__device__ void line_backward(const LinePlan& pl, const Bufs<T>& B, int Lrt, OUT out) {
  const int m = MC ? MC : pl.m, n = MC ? 2 * MC : pl.n;
  const int L = LC ? LC : Lrt;
  if (pl.kind == 0) {
    for (int it = threadIdx.x; it < L * m; it += blockDim.x) {
      const int line = it % L, k = it / L;
      st2<T>(B, 0, k, line,
             real_bwd_Z<T>(pl, packed_X<T>(B, 1, k, m, line), packed_X<T>(B, 1, m - k, m, line), k));
    }
  } else {
    const bool dst = pl.kind == 2;
    // X_k of the DCT-III (for the sine kind: the reversed input)
    auto X = [&](int k, int line) -> T {
      if (k >= n) return (T)0;
      return ldr<T>(B, 1, dst ? n - 1 - k : k, line);
    };
    auto V = [&](int k, int line) -> cx<T> {  // e^{i pi k/(2n)} (X_k - i X_{n-k})
      const cx<T> w = cconj<T>(TWC<T>(pl, k));
      return cmul<T>(w, mk<T>(X(k, line), -X(n - k, line)));
    };
    for (int it = threadIdx.x; it < L * m; it += blockDim.x) {
      const int line = it % L, k = it / L;
      st2<T>(B, 0, k, line, real_bwd_Z<T>(pl, V(k, line), V(m - k, line), k));
    }
  }
  __syncthreads();
  const int zb = fft_lines<T, MC, LC>(pl, B, 0, L, +1);
  if (pl.kind == 0) {
    for (int it = threadIdx.x; it < L * n; it += blockDim.x) {
      const int line = LF ? it % L : it / n, i = LF ? it / L : it - line * n;
      out(line, i, ldr<T>(B, zb, i, line));
    }
  } else {
    const bool dst = pl.kind == 2;
    for (int it = threadIdx.x; it < L * n; it += blockDim.x) {
      const int line = LF ? it % L : it / n, i = LF ? it / L : it - line * n;
      const int pos = (i & 1) ? n - 1 - (i >> 1) : (i >> 1);
      T v = ldr<T>(B, zb, pos, line);
      if (dst && (i & 1)) v = -v;
      out(line, i, v);
    }
  }
}

// input position of real sample i for the forward kinds (Makhoul reorder)
__device__ __forceinline__ int fwd_pos(int kind, int n, int i) {
  if (kind == 0) return i;
  return (i & 1) ? n - 1 - (i >> 1) : (i >> 1);
}

template <typename T>
__device__ __forceinline__ Bufs<T> smem_bufs(T* sm, int m, int L) {
  Bufs<T> B;
  B.LP = L | 1;
  const int sz = m * B.LP;
  B.re[0] = sm;
  B.im[0] = sm + sz;
  B.re[1] = sm + 2 * sz;
  B.im[1] = sm + 3 * sz;
  return B;
}

// ---------------------------------------------------------------------------
// x transforms.  Lines = rows (j,k), L per CTA.
// Forward input: the interior of a halo-layout FP64 field, or (FUSED) the
// fillps right-hand side rho0*div(u)/dt computed on the fly in FP64
// (src/fillps.f90:39-50).
// ---------------------------------------------------------------------------
// the most lines an x-transform CTA holds (lines_per_cta with x_maxL)
constexpr int kXLinesMax = 16;

template <typename T, bool FUSED, int MC, int LC>
struct FftXFwd {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const LinePlan& pl,
      const DevScalars* __restrict__ sc, const double* __restrict__ src, const double* __restrict__ u,
      const double* __restrict__ v, const double* __restrict__ w, const Phys& ph, T* __restrict__ work, int Lrt) {
    if (HALTED(sc)) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* sm = reinterpret_cast<T*>(smraw);
    const int n = MC ? 2 * MC : pl.n, m = MC ? MC : pl.m;
    const int L = LC ? LC : Lrt;
    const Bufs<T> B = smem_bufs<T>(sm, m < 1 ? 1 : m, L);
    const int nlines = g.ny * g.nz;
    const int l0 = bk.x * L;
    const double dti = FUSED ? sc->dti : 0.;
    const double dtidxi = dti * g.dxi, dtidyi = dti * g.dyi;
    // per line: the halo index of its point i = 0 (-1 past the last line)
    // and dti*dzfi(k), so that the per-point work needs no division by ny
    __shared__ int lbase[kXLinesMax];
    __shared__ double ldz[kXLinesMax];
    if (threadIdx.x < L) {
      const int gl = l0 + threadIdx.x, k = gl / g.ny + 1;
      lbase[threadIdx.x] = gl < nlines ? g.h(0, gl % g.ny + 1, k) : -1;
      ldz[threadIdx.x] = gl < nlines ? dti * g.dzfi[k] : 0.;
    }
    __syncthreads();
    auto get = [&](int it) -> double {
      const int line = it / n, i = it - line * n;
      const int cb = lbase[line];
      double x = 0.;
      if (cb >= 0) {
        const int c = cb + i + 1;
        if (FUSED) {
          x = ph.rho0 * ((__ldg(w + c) - __ldg(w + c - g.sxy)) * ldz[line] +
                         (__ldg(v + c) - __ldg(v + c - g.sx)) * dtidyi + (__ldg(u + c) - __ldg(u + c - 1)) * dtidxi);
        } else {
          x = __ldg(src + c);
        }
      }
      return x;
    };
    auto put = [&](int it, double x) {
      const int line = it / n, i = it - line * n;
      T xv = (T)x;
      if (pl.kind == 2 && (i & 1)) xv = -xv;  // sine kind: negate odd samples
      str<T>(B, 0, fwd_pos(pl.kind, n, i), line, xv);
    };
    constexpr int NB = (LC > 0 && MC > 0) ? (LC * 2 * MC + 255) / 256 : 0;
    if (NB > 0 && NB <= 16) {
      double r[NB > 0 ? NB : 1];
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        const int it = threadIdx.x + 256 * q;
        r[q] = it < L * n ? get(it) : 0.;
      }
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        const int it = threadIdx.x + 256 * q;
        if (it < L * n) put(it, r[q]);
      }
    } else {
      for (int it = threadIdx.x; it < L * n; it += blockDim.x) put(it, get(it));
    }
    __syncthreads();
    line_forward<T, false, MC, LC>(pl, B, L, [&](int line, int s, T val) {
      const int gl = l0 + line;
      if (gl < nlines) work[(size_t)gl * n + s] = val;
    });
  }
};
template <typename T, bool FUSED, int MC, int LC>
__global__ void __launch_bounds__(256) k_fft_x_fwd(Geo g, LinePlan pl, const DevScalars* __restrict__ sc,
    const double* __restrict__ src, const double* __restrict__ u, const double* __restrict__ v,
    const double* __restrict__ w, Phys ph, T* __restrict__ work, int Lrt) {
  FftXFwd<T, FUSED, MC, LC>::run(blk_here(), g, pl, sc, src, u, v, w, ph, work, Lrt);
}

// ADD: dst += normfft * x (refinement correction) instead of dst = normfft * x
// wrap: periodic images of dst written as well (store_wraps; not with ADD)
template <typename T, bool ADD, int MC, int LC>
struct FftXBwd {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const LinePlan& pl,
      const DevScalars* __restrict__ sc, const T* __restrict__ work, double normfft, double* __restrict__ dst,
      int Lrt, int wrap) {
    if (HALTED(sc)) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* sm = reinterpret_cast<T*>(smraw);
    const int n = MC ? 2 * MC : pl.n, m = MC ? MC : pl.m;
    const int L = LC ? LC : Lrt;
    const Bufs<T> B = smem_bufs<T>(sm, m < 1 ? 1 : m, L);
    const int nlines = g.ny * g.nz;
    const int l0 = bk.x * L;
    // per line: the halo index of its point i = 0 (-1 past the last line)
    // and the offsets of its y and z images
    __shared__ int lbase[kXLinesMax], loy[kXLinesMax], loz[kXLinesMax];
    if (threadIdx.x < L) {
      const int gl = l0 + threadIdx.x, j = gl % g.ny + 1, k = gl / g.ny + 1;
      lbase[threadIdx.x] = gl < nlines ? g.h(0, j, k) : -1;
      loy[threadIdx.x] = ADD ? 0 : wrap_oy(g, wrap, j);
      loz[threadIdx.x] = ADD ? 0 : wrap_oz(g, wrap, k);
    }
    constexpr int NB = (LC > 0 && MC > 0) ? (LC * 2 * MC + 255) / 256 : 0;
    if (NB > 0 && NB <= 32) {
      T r[NB > 0 ? NB : 1];
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        const int it = threadIdx.x + 256 * q;
        const int line = it / n, gl = l0 + line;
        r[q] = (it < L * n && gl < nlines) ? work[(size_t)gl * n + (it - line * n)] : (T)0;
      }
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        const int it = threadIdx.x + 256 * q;
        const int line = it / n;
        if (it < L * n) str<T>(B, 1, it - line * n, line, r[q]);
      }
    } else {
      for (int it = threadIdx.x; it < L * n; it += blockDim.x) {
        const int line = it / n, s = it - line * n;
        const int gl = l0 + line;
        str<T>(B, 1, s, line, gl < nlines ? work[(size_t)gl * n + s] : (T)0);
      }
    }
    __syncthreads();
    line_backward<T, false, MC, LC>(pl, B, L, [&](int line, int i, T val) {
      const int cb = lbase[line];
      if (cb >= 0) {
        const int c = cb + i + 1;
        if (ADD) {
          dst[c] = dst[c] + (double)val * normfft;
        } else {
          const double o = (double)val * normfft;
          dst[c] = o;
          store_images(c, ADD ? 0 : wrap_ox(g, wrap, i + 1), loy[line], loz[line], [&](int h) { dst[h] = o; });
        }
      }
    });
  }
};
template <typename T, bool ADD, int MC, int LC>
__global__ void __launch_bounds__(256) k_fft_x_bwd(Geo g, LinePlan pl, const DevScalars* __restrict__ sc,
    const T* __restrict__ work, double normfft, double* __restrict__ dst, int Lrt, int wrap) {
  FftXBwd<T, ADD, MC, LC>::run(blk_here(), g, pl, sc, work, normfft, dst, Lrt, wrap);
}

// ---------------------------------------------------------------------------
// x transforms of the periodic kind with one warp per line, for m = 32 R
// complex points (R = 2 or 4: real lines of 128 or 256 points).  A lane
// holds R points of the line in registers; the complex FFT is an R-point DFT
// in each lane, a twiddle, and 32-point DFTs across the lanes by radix-2
// decimation in frequency with shuffles, so a line needs no block-wide
// barrier; the real-to-complex pre- and post-processing pair k with m - k
// through a 2 KiB per-warp shared-memory line (FP64), synchronised by the
// warp alone.  The same transform as the shared-memory Stockham kernels in
// another summation order (differences at round-off).
// ---------------------------------------------------------------------------
constexpr int kWarpLines = 4;  // lines per warp
template <typename T>
__device__ __forceinline__ cx<T> shfl_xor_c(cx<T> v, int m) {
  return mk<T>(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
template <typename T>
__device__ __forceinline__ cx<T> shfl_c(cx<T> v, int src) {
  return mk<T>(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// complex FFT of length M = 32 R with sign SIGN (-1 forward, +1 backward) of
// the line z held as v[q] = z_{lane + 32 q}.  With k = r + R s:
//   Z_k = sum_l W_32^{l s} W_M^{l r} sum_q z_{l + 32 q} W_R^{q r}
// (W_n = exp(SIGN 2 pi i / n)).  On return v[r] = Z_{r + R brev5(lane)}.
template <typename T, int R, int SIGN>
__device__ __forceinline__ void warp_fft(const LinePlan& pl, cx<T> (&v)[R], int lane) {
  constexpr int M = 32 * R;
  if (R == 2) {
    const cx<T> a = v[0], b = v[1 % R];
    v[0] = cadd<T>(a, b);
    v[1 % R] = csub<T>(a, b);
  } else if (R == 4) {
    const cx<T> t0 = cadd<T>(v[0], v[2 % R]), t1 = csub<T>(v[0], v[2 % R]);
    const cx<T> t2 = cadd<T>(v[1 % R], v[3 % R]), t3 = csub<T>(v[1 % R], v[3 % R]);
    const cx<T> it3 = SIGN < 0 ? mk<T>(t3.y, -t3.x) : mk<T>(-t3.y, t3.x);  // W4 * t3
    v[0] = cadd<T>(t0, t2);
    v[1 % R] = cadd<T>(t1, it3);
    v[2 % R] = csub<T>(t0, t2);
    v[3 % R] = csub<T>(t1, it3);
  }
#pragma unroll
  for (int r = 1; r < R; ++r) {
    if (lane > 0) {
      cx<T> w = TW<T>(pl, lane * r);  // W_M^{lane r}, lane r < M
      if (SIGN > 0) w = cconj<T>(w);
      v[r] = cmul<T>(v[r], w);
    }
  }
#pragma unroll
  for (int h = 16; h >= 1; h >>= 1) {
    // pairs (i, i + h) of each block of 2h lanes: the upper lane takes
    // x_i + x_{i+h}, the lower one (x_i - x_{i+h}) W_{2h}^{i mod h}
    const bool lo = (lane & h) != 0;
    const int e = (lane & (h - 1)) * (M / (2 * h));  // W_{2h}^t = W_M^{t M / (2h)}
    cx<T> w = mk<T>(1, 0);
    if (lo && e > 0) {
      w = TW<T>(pl, e);
      if (SIGN > 0) w = cconj<T>(w);
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const cx<T> p = shfl_xor_c<T>(v[r], h);
      if (lo) {
        const cx<T> d = csub<T>(p, v[r]);
        v[r] = e > 0 ? cmul<T>(d, w) : d;
      } else {
        v[r] = cadd<T>(v[r], p);
      }
    }
  }
}

// X_k of a forward real transform from Z_k and Z_{m-k} (as real_fwd_X)
template <typename T>
__device__ __forceinline__ cx<T> real_fwd_Xc(const LinePlan& pl, cx<T> zk, cx<T> zmk, int k) {
  const cx<T> zc = cconj<T>(zmk);
  const cx<T> w = TW2<T>(pl, k);
  const cx<T> sum = mk<T>((T)0.5 * (zk.x + zc.x), (T)0.5 * (zk.y + zc.y));
  const cx<T> dif = csub<T>(zk, zc);
  const cx<T> wd = cmul<T>(w, dif);
  return mk<T>(sum.x + (T)0.5 * wd.y, sum.y - (T)0.5 * wd.x);
}

template <typename T, bool FUSED, int R>
struct FftXFwdW {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const LinePlan& pl,
      const DevScalars* __restrict__ sc, const double* __restrict__ src, const double* __restrict__ u,
      const double* __restrict__ v, const double* __restrict__ w, const Phys& ph, T* __restrict__ work) {
    if (HALTED(sc)) return;
    constexpr int M = 32 * R, N = 2 * M;
    __shared__ cx<T> sz[8][M];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, brl = (int)(__brev((unsigned)lane) >> 27);
    const int nlines = g.ny * g.nz;
    const double dti = FUSED ? sc->dti : 0.;
    const double dtidxi = dti * g.dxi, dtidyi = dti * g.dyi;
    for (int t = 0; t < kWarpLines; ++t) {
      const int gl = (bk.x * 8 + warp) * kWarpLines + t;
      if (gl >= nlines) break;  // the same for the whole warp
      const int jj = gl % g.ny + 1, kk = gl / g.ny + 1;
      const int cb = g.h(1, jj, kk);
      const double dzk = FUSED ? dti * g.dzfi[kk] : 0.;
      auto get = [&](int c) -> double {
        if (FUSED)
          return ph.rho0 * ((__ldg(w + c) - __ldg(w + c - g.sxy)) * dzk + (__ldg(v + c) - __ldg(v + c - g.sx)) * dtidyi +
                            (__ldg(u + c) - __ldg(u + c - 1)) * dtidxi);
        return __ldg(src + c);
      };
      cx<T> z[R];
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int c = cb + 2 * (lane + 32 * q);
        z[q] = mk<T>((T)get(c), (T)get(c + 1));
      }
      warp_fft<T, R, -1>(pl, z, lane);
#pragma unroll
      for (int r = 0; r < R; ++r) sz[warp][r + R * brl] = z[r];
      __syncwarp();
      cx<T>* out = reinterpret_cast<cx<T>*>(work + (size_t)gl * N);
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int k = lane + 32 * q;
        const cx<T> X = real_fwd_Xc<T>(pl, sz[warp][k], sz[warp][(M - k) % M], k);
        if (k == 0) {
          const cx<T> Xm = real_fwd_Xc<T>(pl, sz[warp][0], sz[warp][0], M);
          out[0] = mk<T>(X.x, Xm.x);  // packed: r_0, r_m
        } else {
          out[k] = X;
        }
      }
      __syncwarp();
    }
  }
};
template <typename T, bool FUSED, int R>
__global__ void __launch_bounds__(256) k_fft_x_fwd_w(Geo g, LinePlan pl, const DevScalars* __restrict__ sc,
    const double* __restrict__ src, const double* __restrict__ u, const double* __restrict__ v,
    const double* __restrict__ w, Phys ph, T* __restrict__ work) {
  FftXFwdW<T, FUSED, R>::run(blk_here(), g, pl, sc, src, u, v, w, ph, work);
}

template <typename T, bool ADD, int R>
struct FftXBwdW {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const LinePlan& pl,
      const DevScalars* __restrict__ sc, const T* __restrict__ work, double normfft, double* __restrict__ dst,
      int wrap) {
    if (HALTED(sc)) return;
    constexpr int M = 32 * R, N = 2 * M;
    __shared__ cx<T> sz[8][M];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, brl = (int)(__brev((unsigned)lane) >> 27);
    const int nlines = g.ny * g.nz;
    for (int t = 0; t < kWarpLines; ++t) {
      const int gl = (bk.x * 8 + warp) * kWarpLines + t;
      if (gl >= nlines) break;  // the same for the whole warp
      // the packed spectrum (r_0, r_m, r_1, i_1, ...): X_k = slot k, 1 <= k < m
      const cx<T>* row = reinterpret_cast<const cx<T>*>(work + (size_t)gl * N);
      cx<T> P[R], G[R], Z[R];
#pragma unroll
      for (int q = 0; q < R; ++q) P[q] = row[lane + 32 * q];
      // X_{m-k} for k = lane + 32 q: slot 32 (R-1-q) + (32 - lane) of lane 32 - lane,
      // for lane 0 slot 32 (R - q) of its own
      const int srcl = (32 - lane) & 31;
#pragma unroll
      for (int q = 0; q < R; ++q) G[q] = shfl_c<T>(P[q], srcl);
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int k = lane + 32 * q;
        cx<T> xk = P[q], xmk = G[R - 1 - q];
        if (lane == 0) {
          if (q == 0) {
            xk = mk<T>(P[0].x, (T)0);
            xmk = mk<T>(P[0].y, (T)0);
          } else {
            xmk = G[(R - q) % R];
          }
        }
        Z[q] = real_bwd_Z<T>(pl, xk, xmk, k);
      }
      warp_fft<T, R, +1>(pl, Z, lane);
#pragma unroll
      for (int r = 0; r < R; ++r) sz[warp][r + R * brl] = Z[r];
      __syncwarp();
      const int jj = gl % g.ny + 1, kk = gl / g.ny + 1;
      const int cb = g.h(1, jj, kk);
      const int oy = ADD ? 0 : wrap_oy(g, wrap, jj), oz = ADD ? 0 : wrap_oz(g, wrap, kk);
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int j = lane + 32 * q;
        const cx<T> zj = sz[warp][j];
        const int c = cb + 2 * j;  // x_{2j} at i = 2j + 1, x_{2j+1} at i = 2j + 2
        if (ADD) {
          dst[c] = dst[c] + (double)zj.x * normfft;
          dst[c + 1] = dst[c + 1] + (double)zj.y * normfft;
        } else {
          const double o0 = (double)zj.x * normfft, o1 = (double)zj.y * normfft;
          dst[c] = o0;
          dst[c + 1] = o1;
          store_images(c, wrap_ox(g, wrap, 2 * j + 1), oy, oz, [&](int h) { dst[h] = o0; });
          store_images(c + 1, wrap_ox(g, wrap, 2 * j + 2), oy, oz, [&](int h) { dst[h] = o1; });
        }
      }
      __syncwarp();
    }
  }
};
template <typename T, bool ADD, int R>
__global__ void __launch_bounds__(256) k_fft_x_bwd_w(Geo g, LinePlan pl, const DevScalars* __restrict__ sc,
    const T* __restrict__ work, double normfft, double* __restrict__ dst, int wrap) {
  FftXBwdW<T, ADD, R>::run(blk_here(), g, pl, sc, work, normfft, dst, wrap);
}

// ---------------------------------------------------------------------------
// y transforms, in place on the spectral buffer.  Lines = L consecutive x
// positions of one z plane; the tile is read and written row by row.
// ---------------------------------------------------------------------------
template <typename T, int DIR, int MC, int LC>
struct FftY {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const LinePlan& pl,
      const DevScalars* __restrict__ sc, T* __restrict__ work, int Lrt) {
    if (HALTED(sc)) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* sm = reinterpret_cast<T*>(smraw);
    const int n = MC ? 2 * MC : pl.n, m = MC ? MC : pl.m, nx = g.nx;
    const int L = LC ? LC : Lrt;
    const Bufs<T> B = smem_bufs<T>(sm, m < 1 ? 1 : m, L);
    const int i0 = bk.x * L, k = bk.y;
    T* plane = work + (size_t)k * nx * n;
    auto put = [&](int it, T x) {
      const int line = it % L, j = it / L;
      if (DIR > 0) {
        if (pl.kind == 2 && (j & 1)) x = -x;
        str<T>(B, 0, fwd_pos(pl.kind, n, j), line, x);
      } else {
        str<T>(B, 1, j, line, x);
      }
    };
    auto get = [&](int it) -> T {
      const int line = it % L, j = it / L;
      const int i = i0 + line;
      return i < nx ? plane[(size_t)j * nx + i] : (T)0;
    };
    constexpr int NB = (LC > 0 && MC > 0) ? (LC * 2 * MC + 255) / 256 : 0;
    if (NB > 0 && NB <= 32) {
      // the tile's loads issued together, then the shared-memory stores
      T r[NB > 0 ? NB : 1];
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        const int it = threadIdx.x + 256 * q;
        r[q] = it < L * n ? get(it) : (T)0;
      }
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        const int it = threadIdx.x + 256 * q;
        if (it < L * n) put(it, r[q]);
      }
    } else {
      for (int it = threadIdx.x; it < L * n; it += blockDim.x) put(it, get(it));
    }
    __syncthreads();
    auto out = [&](int line, int j, T val) {
      const int i = i0 + line;
      if (i < nx) plane[(size_t)j * nx + i] = val;
    };
    if (DIR > 0) line_forward<T, true, MC, LC>(pl, B, L, out);
    else line_backward<T, true, MC, LC>(pl, B, L, out);
  }
};
template <typename T, int DIR, int MC, int LC>
__global__ void __launch_bounds__(256) k_fft_y(Geo g, LinePlan pl, const DevScalars* __restrict__ sc,
                                               T* __restrict__ work, int Lrt) {
  FftY<T, DIR, MC, LC>::run(blk_here(), g, pl, sc, work, Lrt);
}

// ---------------------------------------------------------------------------
// y transforms of the periodic kind in two register passes (complex lengths
// m = A*B of 32, 64 and 128).  With j = j2 + B j1 and k = k1 + A k2,
//   Z_{k1 + A k2} = sum_j2 W_B^{j2 k2} W_m^{j2 k1} sum_j1 z_{j2 + B j1} W_A^{j1 k1}
// (W_n = exp(-2 pi i / n) forward, its conjugate backward): an A-point DFT
// per (line, j2), a twiddle, then a B-point DFT per (line, k1), each in one
// thread's registers.  The two passes meet once in shared memory, so a
// transform takes one block barrier; the lines' samples go from HBM into
// registers (and back) directly, the threads of a warp covering 16 or 32
// consecutive x positions of a row, so every access is a whole 128-byte
// row segment.  The real-sequence step pairs Z_k with Z_{m-k}: one thread
// of the second forward pass (of the first backward pass) owns the columns
// k1 and A - k1 (or 0 and A/2), which hold every such pair, so the pairing
// stays in registers.
// ---------------------------------------------------------------------------
// v * exp(S 2 pi i E / 16), 0 <= E < 8 (E a constant after unrolling)
template <typename T, int S>
__device__ __forceinline__ cx<T> rot16(cx<T> v, int E) {
  // cos and sin of 2 pi E / 16
  constexpr double C1 = 0.92387953251128675613, S1 = 0.38268343236508977173, H = 0.70710678118654752440;
  if (E == 0) return v;
  if (E == 4) return S < 0 ? mk<T>(v.y, -v.x) : mk<T>(-v.y, v.x);  // times S i
  const double c = E == 1 ? C1 : E == 2 ? H : E == 3 ? S1 : E == 5 ? -S1 : E == 6 ? -H : -C1;
  const double s = (E == 1 || E == 7) ? S1 : (E == 2 || E == 6) ? H : C1;
  const T wc = (T)c, ws = (T)(S * s);
  return mk<T>(v.x * wc - v.y * ws, v.x * ws + v.y * wc);
}

// N-point DFT (N = 2, 4, 8, 16; sign S) of v[0], v[ST], ..., v[(N-1) ST]
// into o[0..N-1], radix-2 decimation in time, unrolled into registers
template <typename T, int N, int S, int ST>
struct RegDft {
  static __device__ __forceinline__ void run(const cx<T>* v, cx<T>* o) {
    if constexpr (N == 2) {
      o[0] = cadd<T>(v[0], v[ST]);
      o[1] = csub<T>(v[0], v[ST]);
    } else {
      cx<T> e[N / 2], d[N / 2];
      RegDft<T, N / 2, S, 2 * ST>::run(v, e);
      RegDft<T, N / 2, S, 2 * ST>::run(v + ST, d);
#pragma unroll
      for (int k = 0; k < N / 2; ++k) {
        const cx<T> t = rot16<T, S>(d[k], k * (16 / N));
        o[k] = cadd<T>(e[k], t);
        o[k + N / 2] = csub<T>(e[k], t);
      }
    }
  }
};

template <int M> struct Y2Shape;  // complex length -> (A, B, lines per CTA)
template <> struct Y2Shape<32> { static constexpr int A = 8, B = 4, L = 32; };
template <> struct Y2Shape<64> { static constexpr int A = 8, B = 8, L = 16; };
template <> struct Y2Shape<128> { static constexpr int A = 16, B = 8, L = 16; };
__host__ __device__ constexpr bool y2_length(int m) { return m == 32 || m == 64 || m == 128; }

template <typename T, int DIR, int MC>
struct FftY2 {
  static constexpr int A = Y2Shape<MC>::A, B = Y2Shape<MC>::B, L = Y2Shape<MC>::L, NT = B * L;
  static_assert(A % 2 == 0 && A / 2 <= B, "the pair pass fits in the B-pass threads");
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const LinePlan& pl,
      const DevScalars* __restrict__ sc, T* __restrict__ work) {
    if (HALTED(sc)) return;
    constexpr int M = MC;
    __shared__ cx<T> sb[M * L];  // [k1][j2][line]
    const int nx = g.nx;
    const int l = threadIdx.x % L, q = threadIdx.x / L;
    const int i = bk.x * L + l;
    const bool in = i < nx;
    // row r of this thread's line: col[r * nx]
    T* col = work + (size_t)bk.y * nx * (2 * M) + (in ? i : 0);
    auto row = [&](int r) -> T& { return col[(size_t)r * nx]; };
    // the pair pass: columns k1a = p and k1b = A - p (p > 0), or 0 and A/2
    const int p = q, k1a = p, k1b = p == 0 ? A / 2 : A - p;
    if (DIR > 0) {
      {  // A-point DFTs over j1, line l, j2 = q
        const int j2 = q;
        cx<T> z[A], y[A];
#pragma unroll
        for (int j1 = 0; j1 < A; ++j1) {
          const int r = 2 * (j2 + B * j1);
          z[j1] = in ? mk<T>(row(r), row(r + 1)) : mk<T>(0, 0);
        }
        RegDft<T, A, -1, 1>::run(z, y);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) {
          cx<T> v = y[k1];
          if (k1 > 0 && j2 > 0) v = cmul<T>(v, TW<T>(pl, j2 * k1));
          sb[(k1 * B + j2) * L + l] = v;
        }
      }
      __syncthreads();
      if (p < A / 2) {  // B-point DFTs over j2 for the columns k1a, k1b
        cx<T> a[B], b[B], za[B], zb[B];
#pragma unroll
        for (int j2 = 0; j2 < B; ++j2) {
          a[j2] = sb[(k1a * B + j2) * L + l];
          b[j2] = sb[(k1b * B + j2) * L + l];
        }
        RegDft<T, B, -1, 1>::run(a, za);  // Z_{k1a + A k2} = za[k2]
        RegDft<T, B, -1, 1>::run(b, zb);
        if (in) {
#pragma unroll
          for (int k2 = 0; k2 < B; ++k2) {
            // Z_{m-k}: m - (k1a + A k2) = k1b + A (B-1-k2) (p > 0) or A (B-k2) (p = 0)
            const int ka = k1a + A * k2, kb = k1b + A * k2;
            const cx<T> za_m = p > 0 ? zb[B - 1 - k2] : za[(B - k2) % B];
            const cx<T> zb_m = p > 0 ? za[B - 1 - k2] : zb[B - 1 - k2];
            const cx<T> Xa = real_fwd_Xc<T>(pl, za[k2], za_m, ka);
            const cx<T> Xb = real_fwd_Xc<T>(pl, zb[k2], zb_m, kb);
            if (ka == 0) {  // packed: r_0, r_m
              row(0) = Xa.x;
              row(1) = real_fwd_Xc<T>(pl, za[0], za[0], M).x;
            } else {
              row(2 * ka) = Xa.x;
              row(2 * ka + 1) = Xa.y;
            }
            row(2 * kb) = Xb.x;
            row(2 * kb + 1) = Xb.y;
          }
        }
      }
    } else {
      if (p < A / 2) {  // Z_k from the packed spectrum, B-point DFTs over k2
        cx<T> xa[B], xb[B];
        T xm = (T)0;  // X_m (real), packed beside X_0
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) {
          const int ka = k1a + A * k2, kb = k1b + A * k2;
          if (ka == 0) {
            xa[k2] = in ? mk<T>(row(0), (T)0) : mk<T>(0, 0);
            xm = in ? row(1) : (T)0;
          } else {
            xa[k2] = in ? mk<T>(row(2 * ka), row(2 * ka + 1)) : mk<T>(0, 0);
          }
          xb[k2] = in ? mk<T>(row(2 * kb), row(2 * kb + 1)) : mk<T>(0, 0);
        }
        cx<T> za[B], zb[B];
#pragma unroll
        for (int k2 = 0; k2 < B; ++k2) {
          const int ka = k1a + A * k2, kb = k1b + A * k2;
          const cx<T> xa_m = p > 0 ? xb[B - 1 - k2] : (k2 == 0 ? mk<T>(xm, (T)0) : xa[B - k2]);
          const cx<T> xb_m = p > 0 ? xa[B - 1 - k2] : xb[B - 1 - k2];
          za[k2] = real_bwd_Z<T>(pl, xa[k2], xa_m, ka);
          zb[k2] = real_bwd_Z<T>(pl, xb[k2], xb_m, kb);
        }
        cx<T> ua[B], ub[B];
        RegDft<T, B, +1, 1>::run(za, ua);
        RegDft<T, B, +1, 1>::run(zb, ub);
#pragma unroll
        for (int j2 = 0; j2 < B; ++j2) {
          cx<T> va = ua[j2], vb = ub[j2];
          if (j2 > 0) {
            if (k1a > 0) va = cmul<T>(va, cconj<T>(TW<T>(pl, j2 * k1a)));
            vb = cmul<T>(vb, cconj<T>(TW<T>(pl, j2 * k1b)));
          }
          sb[(k1a * B + j2) * L + l] = va;
          sb[(k1b * B + j2) * L + l] = vb;
        }
      }
      __syncthreads();
      {  // A-point DFTs over k1, line l, j2 = q: z_{j2 + B j1}
        const int j2 = q;
        cx<T> u[A], z[A];
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) u[k1] = sb[(k1 * B + j2) * L + l];
        RegDft<T, A, +1, 1>::run(u, z);
        if (in) {
#pragma unroll
          for (int j1 = 0; j1 < A; ++j1) {
            const int r = 2 * (j2 + B * j1);
            row(r) = z[j1].x;
            row(r + 1) = z[j1].y;
          }
        }
      }
    }
  }
};
// x transforms of the periodic kind in the same two register passes.  An x
// line is a contiguous row, so the threads of a line take consecutive j2
// (first forward pass) or consecutive column pairs (k1a, k1b) (pair pass),
// and a warp's accesses are whole row segments.  The two passes meet in
// shared memory laid out [line][k1][j2] with a k1 pitch of B + 1 complex
// values, which keeps the eight 16-byte accesses of a quarter warp on
// distinct banks in both passes.  Forward: the input is the interior of a
// halo-layout FP64 field, or (FUSED) fillps's right-hand side formed on the
// fly; the packed spectrum goes to the line's row of the spectral buffer.
// Backward: from that row into the halo-layout field, scaled by normfft,
// with its periodic images (or added to it, ADD).
template <typename T, bool FUSED, int MC>
struct FftX2Fwd {
  static constexpr int A = Y2Shape<MC>::A, B = Y2Shape<MC>::B, L = Y2Shape<MC>::L, NT = B * L, P = B + 1;
  static constexpr int LP = A * P + (B == 4 ? 4 : 0);  // line pitch: two lines per quarter warp when B = 4
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const LinePlan& pl,
      const DevScalars* __restrict__ sc, const double* __restrict__ src, const double* __restrict__ u,
      const double* __restrict__ v, const double* __restrict__ w, const Phys& ph, T* __restrict__ work) {
    if (HALTED(sc)) return;
    constexpr int M = MC, N = 2 * MC;
    __shared__ cx<T> sb[L * LP];  // [line][k1][j2]
    const int q = threadIdx.x % B, l = threadIdx.x / B;
    const int gl = bk.x * L + l;
    const bool in = gl < g.ny * g.nz;
    const int jj = in ? gl % g.ny + 1 : 1, kk = in ? gl / g.ny + 1 : 1;
    const int cb = g.h(1, jj, kk);
    const double dti = FUSED ? sc->dti : 0.;
    const double dtidxi = dti * g.dxi, dtidyi = dti * g.dyi, dzk = FUSED ? dti * g.dzfi[kk] : 0.;
    auto get = [&](int c) -> double {
      if (FUSED)
        return ph.rho0 * ((__ldg(w + c) - __ldg(w + c - g.sxy)) * dzk + (__ldg(v + c) - __ldg(v + c - g.sx)) * dtidyi +
                          (__ldg(u + c) - __ldg(u + c - 1)) * dtidxi);
      return __ldg(src + c);
    };
    cx<T>* sl = sb + l * LP;
    {  // A-point DFTs over j1, j2 = q
      const int j2 = q;
      cx<T> z[A], y[A];
#pragma unroll
      for (int j1 = 0; j1 < A; ++j1) {
        const int c = cb + 2 * (j2 + B * j1);
        z[j1] = in ? mk<T>((T)get(c), (T)get(c + 1)) : mk<T>(0, 0);
      }
      RegDft<T, A, -1, 1>::run(z, y);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) {
        cx<T> t = y[k1];
        if (k1 > 0 && j2 > 0) t = cmul<T>(t, TW<T>(pl, j2 * k1));
        sl[k1 * P + j2] = t;
      }
    }
    __syncthreads();
    const int p = q;
    if (p < A / 2 && in) {  // B-point DFTs over j2 for the columns k1a, k1b
      const int k1a = p, k1b = p == 0 ? A / 2 : A - p;
      cx<T> a[B], b[B], za[B], zb[B];
#pragma unroll
      for (int j2 = 0; j2 < B; ++j2) {
        a[j2] = sl[k1a * P + j2];
        b[j2] = sl[k1b * P + j2];
      }
      RegDft<T, B, -1, 1>::run(a, za);
      RegDft<T, B, -1, 1>::run(b, zb);
      cx<T>* out = reinterpret_cast<cx<T>*>(work + (size_t)gl * N);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) {
        const int ka = k1a + A * k2, kb = k1b + A * k2;
        const cx<T> za_m = p > 0 ? zb[B - 1 - k2] : za[(B - k2) % B];
        const cx<T> zb_m = p > 0 ? za[B - 1 - k2] : zb[B - 1 - k2];
        const cx<T> Xa = real_fwd_Xc<T>(pl, za[k2], za_m, ka);
        if (ka == 0) out[0] = mk<T>(Xa.x, real_fwd_Xc<T>(pl, za[0], za[0], M).x);  // packed: r_0, r_m
        else out[ka] = Xa;
        out[kb] = real_fwd_Xc<T>(pl, zb[k2], zb_m, kb);
      }
    }
  }
};
template <typename T, bool FUSED, int MC>
__global__ void __launch_bounds__(FftX2Fwd<T, FUSED, MC>::NT, 3) k_fft_x2_fwd(Geo g, LinePlan pl,
    const DevScalars* __restrict__ sc, const double* __restrict__ src, const double* __restrict__ u,
    const double* __restrict__ v, const double* __restrict__ w, Phys ph, T* __restrict__ work) {
  FftX2Fwd<T, FUSED, MC>::run(blk_here(), g, pl, sc, src, u, v, w, ph, work);
}

template <typename T, bool ADD, int MC>
struct FftX2Bwd {
  static constexpr int A = Y2Shape<MC>::A, B = Y2Shape<MC>::B, L = Y2Shape<MC>::L, NT = B * L, P = B + 1;
  static constexpr int LP = A * P + (B == 4 ? 4 : 0);
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const LinePlan& pl,
      const DevScalars* __restrict__ sc, const T* __restrict__ work, double normfft, double* __restrict__ dst,
      int wrap) {
    if (HALTED(sc)) return;
    constexpr int N = 2 * MC;
    __shared__ cx<T> sb[L * LP];  // [line][k1][j2]
    const int q = threadIdx.x % B, l = threadIdx.x / B;
    const int gl = bk.x * L + l;
    const bool in = gl < g.ny * g.nz;
    cx<T>* sl = sb + l * LP;
    const int p = q;
    if (p < A / 2 && in) {  // Z_k from the packed spectrum, B-point DFTs over k2
      const int k1a = p, k1b = p == 0 ? A / 2 : A - p;
      const cx<T>* row = reinterpret_cast<const cx<T>*>(work + (size_t)gl * N);
      cx<T> xa[B], xb[B];
      T xm = (T)0;
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) {
        const int ka = k1a + A * k2, kb = k1b + A * k2;
        const cx<T> ra = row[ka];
        if (ka == 0) {
          xa[k2] = mk<T>(ra.x, (T)0);
          xm = ra.y;
        } else {
          xa[k2] = ra;
        }
        xb[k2] = row[kb];
      }
      cx<T> za[B], zb[B];
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) {
        const int ka = k1a + A * k2, kb = k1b + A * k2;
        const cx<T> xa_m = p > 0 ? xb[B - 1 - k2] : (k2 == 0 ? mk<T>(xm, (T)0) : xa[B - k2]);
        const cx<T> xb_m = p > 0 ? xa[B - 1 - k2] : xb[B - 1 - k2];
        za[k2] = real_bwd_Z<T>(pl, xa[k2], xa_m, ka);
        zb[k2] = real_bwd_Z<T>(pl, xb[k2], xb_m, kb);
      }
      cx<T> ua[B], ub[B];
      RegDft<T, B, +1, 1>::run(za, ua);
      RegDft<T, B, +1, 1>::run(zb, ub);
#pragma unroll
      for (int j2 = 0; j2 < B; ++j2) {
        cx<T> va = ua[j2], vb = ub[j2];
        if (j2 > 0) {
          if (k1a > 0) va = cmul<T>(va, cconj<T>(TW<T>(pl, j2 * k1a)));
          vb = cmul<T>(vb, cconj<T>(TW<T>(pl, j2 * k1b)));
        }
        sl[k1a * P + j2] = va;
        sl[k1b * P + j2] = vb;
      }
    }
    __syncthreads();
    if (in) {  // A-point DFTs over k1, j2 = q: z_{j2 + B j1}
      const int j2 = q;
      cx<T> uu[A], z[A];
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) uu[k1] = sl[k1 * P + j2];
      RegDft<T, A, +1, 1>::run(uu, z);
      const int jj = gl % g.ny + 1, kk = gl / g.ny + 1;
      const int cb = g.h(1, jj, kk);
      const int oy = ADD ? 0 : wrap_oy(g, wrap, jj), oz = ADD ? 0 : wrap_oz(g, wrap, kk);
#pragma unroll
      for (int j1 = 0; j1 < A; ++j1) {
        const int j = j2 + B * j1;
        const int c = cb + 2 * j;  // x_{2j} at i = 2j + 1, x_{2j+1} at i = 2j + 2
        if (ADD) {
          dst[c] = dst[c] + (double)z[j1].x * normfft;
          dst[c + 1] = dst[c + 1] + (double)z[j1].y * normfft;
        } else {
          const double o0 = (double)z[j1].x * normfft, o1 = (double)z[j1].y * normfft;
          dst[c] = o0;
          dst[c + 1] = o1;
          store_images(c, wrap_ox(g, wrap, 2 * j + 1), oy, oz, [&](int h) { dst[h] = o0; });
          store_images(c + 1, wrap_ox(g, wrap, 2 * j + 2), oy, oz, [&](int h) { dst[h] = o1; });
        }
      }
    }
  }
};
template <typename T, bool ADD, int MC>
__global__ void __launch_bounds__(FftX2Bwd<T, ADD, MC>::NT, 4) k_fft_x2_bwd(Geo g, LinePlan pl,
    const DevScalars* __restrict__ sc, const T* __restrict__ work, double normfft, double* __restrict__ dst,
    int wrap) {
  FftX2Bwd<T, ADD, MC>::run(blk_here(), g, pl, sc, work, normfft, dst, wrap);
}

template <typename T, int DIR, int MC>
__global__ void __launch_bounds__(FftY2<T, DIR, MC>::NT, 3) k_fft_y2(Geo g, LinePlan pl,
                                                                   const DevScalars* __restrict__ sc,
                                                                   T* __restrict__ work) {
  FftY2<T, DIR, MC>::run(blk_here(), g, pl, sc, work);
}

// ---------------------------------------------------------------------------
// z: batched Thomas (dgtsv_homebrewed with the eps pivot shift, src/solver.f90:
// 151-177 / src/solver_gpu.f90:179-203).  One column per thread; the forward
// sweep writes p' in place and keeps d only at chunk ends (shared memory);
// the backward sweep recomputes d per chunk from those checkpoints with the
// same operations, so it equals the stored one bit for bit.  In FP64 the
// pivots use round-to-nearest intrinsics (no FMA contraction), as the
// reference's CPU build evaluates them.  In FP32 the eps shift vanishes, so
// the singular (0,0) column of an all-Neumann/periodic problem pins its last
// unknown to zero instead (any constant solves it).
// ---------------------------------------------------------------------------
#define ZCH 16

template <typename T> struct Rn;
template <> struct Rn<double> {
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  // 1/x correctly rounded: the same value as the division 1./x
  static __device__ __forceinline__ double rcp(double b) { return __drcp_rn(b); }
};
template <> struct Rn<float> {
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float rcp(float b) { return __frcp_rn(b); }
};

// 1./(b(l)+lambda - a(l)*d(l-1) + eps); `pin`: singular column, last row
template <typename T>
__device__ __forceinline__ T piv_inv(int l, int n, T bl, T lam, T al, T dprev, bool pin) {
  typedef Rn<T> R;
  if (pin && l == n - 1) return (T)0;
  if (l == 0) return R::rcp(R::add(R::add(bl, lam), (T)CANSFZ_EPS));
  return R::rcp(R::add(R::sub(R::add(bl, lam), R::mul(al, dprev)), (T)CANSFZ_EPS));
}

template <typename T>
__device__ void thomas_column(int n, const double* __restrict__ a, const double* __restrict__ b,
                              const double* __restrict__ c, T lam, T* __restrict__ col, size_t st,
                              T* __restrict__ dchk, int tpitch, bool pin) {
  typedef Rn<T> R;
  // forward elimination; the next chunk's loads are issued before this
  // chunk's elimination so that their latency overlaps the pivot chain
  T dprev = 0, pprev = 0;
  const int nch = (n + ZCH - 1) / ZCH;
  T pv[ZCH], nx[ZCH];
#pragma unroll
  for (int q = 0; q < ZCH; ++q) pv[q] = (q < n) ? col[(size_t)q * st] : (T)0;
  for (int ch = 0; ch < nch; ++ch) {
    const int k0 = ch * ZCH, k1 = k0 + ZCH;
#pragma unroll
    for (int q = 0; q < ZCH; ++q) nx[q] = (k1 + q < n) ? col[(size_t)(k1 + q) * st] : (T)0;
#pragma unroll
    for (int q = 0; q < ZCH; ++q) {
      const int l = k0 + q;
      if (l < n) {
        const T z = piv_inv<T>(l, n, (T)b[l], lam, (T)a[l], dprev, pin);
        const T d = R::mul((T)c[l], z);
        const T pn = (l == 0) ? R::mul(pv[q], z) : R::mul(R::sub(pv[q], R::mul((T)a[l], pprev)), z);
        dprev = d;
        pprev = pn;
        pv[q] = pn;
      }
    }
#pragma unroll
    for (int q = 0; q < ZCH; ++q)
      if (k0 + q < n) col[(size_t)(k0 + q) * st] = pv[q];
    dchk[ch * tpitch] = dprev;  // d at the last element of chunk ch
#pragma unroll
    for (int q = 0; q < ZCH; ++q) pv[q] = nx[q];
  }
  // backward substitution, chunk by chunk from the top; the chunk's loads are
  // issued before its pivots are recomputed from the checkpoint
  T pnext = 0;
  for (int ch = nch - 1; ch >= 0; --ch) {
    const int k0 = ch * ZCH;
    T dd[ZCH];
#pragma unroll
    for (int q = 0; q < ZCH; ++q) pv[q] = (k0 + q < n) ? col[(size_t)(k0 + q) * st] : (T)0;
    T dp = ch > 0 ? dchk[(ch - 1) * tpitch] : (T)0;
#pragma unroll
    for (int q = 0; q < ZCH; ++q) {
      const int l = k0 + q;
      T d = 0;
      if (l < n) d = R::mul((T)c[l], piv_inv<T>(l, n, (T)b[l], lam, (T)a[l], dp, pin));
      dd[q] = d;
      dp = d;
    }
#pragma unroll
    for (int q = ZCH - 1; q >= 0; --q) {
      const int l = k0 + q;
      if (l < n) {
        if (l < n - 1) pv[q] = R::sub(pv[q], R::mul(dd[q], pnext));
        pnext = pv[q];
      }
    }
#pragma unroll
    for (int q = 0; q < ZCH; ++q)
      if (k0 + q < n) col[(size_t)(k0 + q) * st] = pv[q];
  }
}

// The elimination factors of one column, z(l) = 1/pivot(l) and
// d(l) = c(l)*z(l), with the operations of the forward sweep above: they
// depend on the matrix and the column's eigenvalue only, so they are
// evaluated once per plan and the per-step solve reads them.
template <typename T>
struct ZFactors {
  static __device__ __forceinline__ void run(const Blk& bk, int ncol, int nz, const double* __restrict__ lam,
      const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c, int zsing,
      T* __restrict__ piv, T* __restrict__ df) {
    typedef Rn<T> R;
    const int col = bk.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const double lm = __ldg(lam + col);
    const bool pin = (sizeof(T) == 4) && zsing && lm == 0.;
    T dprev = 0;
    for (int l = 0; l < nz; ++l) {
      const T z = piv_inv<T>(l, nz, (T)b[l], (T)lm, (T)a[l], dprev, pin);
      const T d = R::mul((T)c[l], z);
      piv[(size_t)l * ncol + col] = z;
      df[(size_t)l * ncol + col] = d;
      dprev = d;
    }
  }
};
template <typename T>
__global__ void __launch_bounds__(128) k_z_factors(int ncol, int nz, const double* __restrict__ lam,
    const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c, int zsing,
    T* __restrict__ piv, T* __restrict__ df) {
  ZFactors<T>::run(blk_here(), ncol, nz, lam, a, b, c, zsing, piv, df);
}

// The solve of thomas_column with the factors read instead of evaluated:
// the same products and differences, so the same result bit for bit.  Each
// chunk's column values and factors are loaded one chunk ahead.
template <typename T>
__device__ void thomas_factored(int n, const double* __restrict__ a, const T* __restrict__ piv,
                                const T* __restrict__ df, T* __restrict__ col, size_t st) {
  typedef Rn<T> R;
  T pprev = 0;
  const int nch = (n + ZCH - 1) / ZCH;
  T pv[ZCH], zv[ZCH], nx[ZCH], nz_[ZCH];
#pragma unroll
  for (int q = 0; q < ZCH; ++q) {
    pv[q] = (q < n) ? col[(size_t)q * st] : (T)0;
    zv[q] = (q < n) ? piv[(size_t)q * st] : (T)0;
  }
  for (int ch = 0; ch < nch; ++ch) {
    const int k0 = ch * ZCH, k1 = k0 + ZCH;
#pragma unroll
    for (int q = 0; q < ZCH; ++q) {
      nx[q] = (k1 + q < n) ? col[(size_t)(k1 + q) * st] : (T)0;
      nz_[q] = (k1 + q < n) ? piv[(size_t)(k1 + q) * st] : (T)0;
    }
#pragma unroll
    for (int q = 0; q < ZCH; ++q) {
      const int l = k0 + q;
      if (l < n) {
        const T pn = (l == 0) ? R::mul(pv[q], zv[q]) : R::mul(R::sub(pv[q], R::mul((T)a[l], pprev)), zv[q]);
        pprev = pn;
        pv[q] = pn;
      }
    }
#pragma unroll
    for (int q = 0; q < ZCH; ++q) {
      if (k0 + q < n) col[(size_t)(k0 + q) * st] = pv[q];
      pv[q] = nx[q];
      zv[q] = nz_[q];
    }
  }
  // backward substitution from the top chunk down, the next lower chunk's
  // values and factors loaded ahead
  T pnext = 0;
  const int top = nch - 1;
#pragma unroll
  for (int q = 0; q < ZCH; ++q) {
    const int l = top * ZCH + q;
    pv[q] = (l < n) ? col[(size_t)l * st] : (T)0;
    zv[q] = (l < n) ? df[(size_t)l * st] : (T)0;
  }
  for (int ch = top; ch >= 0; --ch) {
    const int k0 = ch * ZCH, km = k0 - ZCH;
#pragma unroll
    for (int q = 0; q < ZCH; ++q) {
      nx[q] = (km >= 0) ? col[(size_t)(km + q) * st] : (T)0;
      nz_[q] = (km >= 0) ? df[(size_t)(km + q) * st] : (T)0;
    }
#pragma unroll
    for (int q = ZCH - 1; q >= 0; --q) {
      const int l = k0 + q;
      if (l < n) {
        if (l < n - 1) pv[q] = R::sub(pv[q], R::mul(zv[q], pnext));
        pnext = pv[q];
      }
    }
#pragma unroll
    for (int q = 0; q < ZCH; ++q) {
      if (k0 + q < n) col[(size_t)(k0 + q) * st] = pv[q];
      pv[q] = nx[q];
      zv[q] = nz_[q];
    }
  }
}

template <typename T>
struct ZSolveF {
  static __device__ __forceinline__ void run(const Blk& bk, int ncol, int nz, const double* __restrict__ a,
      const T* __restrict__ piv, const T* __restrict__ df, const DevScalars* __restrict__ sc,
      T* __restrict__ work) {
    if (HALTED(sc)) return;
    const int col = bk.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    thomas_factored<T>(nz, a, piv + col, df + col, work + col, (size_t)ncol);
  }
};
template <typename T>
__global__ void __launch_bounds__(128) k_zsolve_f(int ncol, int nz, const double* __restrict__ a,
    const T* __restrict__ piv, const T* __restrict__ df, const DevScalars* __restrict__ sc, T* __restrict__ work) {
  ZSolveF<T>::run(blk_here(), ncol, nz, a, piv, df, sc, work);
}

template <typename T>
struct ZSolve {
  static __device__ __forceinline__ void run(const Blk& bk, int ncol, int nz, const double* __restrict__ lam,
      const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
      const DevScalars* __restrict__ sc, T* __restrict__ work, int zsing) {
    if (HALTED(sc)) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* dchk = reinterpret_cast<T*>(smraw);  // [nch][blockDim]
    const int col = bk.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const double lm = __ldg(lam + col);
    const bool pin = (sizeof(T) == 4) && zsing && lm == 0.;
    thomas_column<T>(nz, a, b, c, (T)lm, work + col, (size_t)ncol, dchk + threadIdx.x, blockDim.x, pin);
  }
};
template <typename T>
__global__ void __launch_bounds__(128) k_zsolve(int ncol, int nz, const double* __restrict__ lam,
    const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
    const DevScalars* __restrict__ sc, T* __restrict__ work, int zsing) {
  ZSolve<T>::run(blk_here(), ncol, nz, lam, a, b, c, sc, work, zsing);
}

// ---------------------------------------------------------------------------
// z, partitioned: a tile of 32 columns with all nz levels in shared memory,
// the levels split into P = 8 chunks of CH levels, one warp per chunk and one
// lane per column.  The spectral buffer is read once and written once (the
// column solve above reads and writes each level twice), and 256 threads
// share each column's elimination instead of one.
//
//   A  each chunk eliminates its interior rows s+1..e-1 twice with running
//      scalars only: downwards with x_s as a parameter, which turns row e
//      into a row in (x_s, x_e, x_{e+1}), and upwards with x_e as a
//      parameter, which turns row s into a row in (x_{s-1}, x_s, x_e);
//   B  those 2P rows form a tridiagonal system in the chunks' end values
//      (x_s0, x_e0, x_s1, x_e1, ...), solved by Thomas in one warp;
//   C  with x_s and x_e known, each chunk solves its interior rows by Thomas
//      (forward sweep into shared memory, the c/pivot factors in registers,
//      back substitution).
//
// The order of elimination differs from gaussel's (src/solver.f90:151-177)
// only by round-off for these diagonally dominant systems (|b + lambda| >=
// |a| + |c|).  The one singular system, the (0,0) mode of an all-periodic/
// Neumann problem, whose eps-shifted pivot (src/solver.f90:163-167) fixes
// the solution's constant, is solved by one thread of block 0 in gaussel's
// own order (thomas_column's operations) from a copy of its right-hand
// side, while the rest of the grid runs.
// ---------------------------------------------------------------------------
constexpr int ZP_NC = 32;  // columns per tile
constexpr int ZP_P = 8;    // chunks (warps) per tile
// the chunk lengths built (nz = 8 * CH)
#define CANSFZ_FOR_ZCHUNKS(X) X(8) X(12) X(16) X(24) X(32)

__device__ __forceinline__ void cp16_cg(void* sdst, const void* gsrc) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gsrc));
}

template <typename T>
constexpr size_t zpart_smem(int nz) {
  return sizeof(T) * ((size_t)nz * ZP_NC + (size_t)8 * ZP_P * ZP_NC + (size_t)2 * ZP_P * ZP_NC + 2 * (size_t)nz);
}

template <typename T, int CH>
struct ZSolvePart {
  static __device__ __forceinline__ void run(const Blk& bk, int ncol, int nz, const double* __restrict__ lam,
      const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
      const DevScalars* __restrict__ sc, T* __restrict__ work, int zsing) {
    typedef Rn<T> R;
    if (HALTED(sc)) return;
    static_assert(CH >= 3, "a chunk needs an interior row");
    constexpr int NC = ZP_NC, P = ZP_P;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* tile = reinterpret_cast<T*>(smraw);        // [nz][NC]
    T* red = tile + (size_t)nz * NC;               // [2P][4][NC]: sub, diag, sup, rhs of the reduced rows
    T* xb = red + (size_t)8 * P * NC;              // [2P][NC]: x_s, x_e of every chunk
    T* s0 = xb + (size_t)2 * P * NC;               // [2][nz]: column 0 of block 0 (serial path)
    const int col0 = bk.x * NC;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int s = w * CH, e = s + CH - 1;
    // each warp stages its own chunk's rows (16-byte copies of rows of NC
    // consecutive columns) and starts on them without waiting for the others
    constexpr int PER = 16 / (int)sizeof(T), CPR = NC / PER;
    for (int q = lane; q < CH * CPR; q += 32) {
      const int l = s + q / CPR, cc = (q % CPR) * PER;
      cp16_cg(tile + (size_t)l * NC + cc, work + (size_t)l * ncol + col0 + cc);
    }
    asm volatile("cp.async.commit_group;\n" ::);
    const T lm = (T)__ldg(lam + col0 + lane);
    const bool serial0 = col0 == 0 && __ldg(lam) == 0.;
    asm volatile("cp.async.wait_group 0;\n" ::);
    __syncwarp();
    // ---- A: the chunk's two reduced rows.  The downward sweep's pivot
    // reciprocals are those of C's forward sweep (same rows, same first
    // pivot), so they are kept for it and C needs no reciprocal.
    T rp[CH - 2];
    {
      T D = 0, Y = 0, F = 0, U = 0, Z = 0, G = 0;
#pragma unroll
      for (int t = 0; t < CH - 2; ++t) {
        const int id = s + 1 + t, iu = e - 1 - t;
        const T ad = (T)__ldg(a + id), cd = (T)__ldg(c + id), bd = (T)__ldg(b + id) + lm;
        const T au = (T)__ldg(a + iu), cu = (T)__ldg(c + iu), bu = (T)__ldg(b + iu) + lm;
        const T dd = tile[id * NC + lane], du = tile[iu * NC + lane];
        const T rd = recip_rn(t == 0 ? bd : bd - ad * D);
        rp[t] = rd;
        Y = (t == 0 ? dd : dd - ad * Y) * rd;
        F = (t == 0 ? -ad : -ad * F) * rd;
        D = cd * rd;
        const T ru = recip_rn(t == 0 ? bu : bu - cu * U);
        Z = (t == 0 ? du : du - cu * Z) * ru;
        G = (t == 0 ? -cu : -cu * G) * ru;
        U = au * ru;
      }
      T* Rs = red + (size_t)(2 * w) * 4 * NC;
      T* Re = Rs + 4 * NC;
      const T as = (T)__ldg(a + s), bs = (T)__ldg(b + s) + lm, cs = (T)__ldg(c + s);
      const T ae = (T)__ldg(a + e), be = (T)__ldg(b + e) + lm, ce = (T)__ldg(c + e);
      Rs[0 * NC + lane] = w == 0 ? (T)0 : as;
      Rs[1 * NC + lane] = bs - cs * U;
      Rs[2 * NC + lane] = cs * G;
      Rs[3 * NC + lane] = tile[s * NC + lane] - cs * Z;
      Re[0 * NC + lane] = ae * F;
      Re[1 * NC + lane] = be - ae * D;
      Re[2 * NC + lane] = w == P - 1 ? (T)0 : ce;
      Re[3 * NC + lane] = tile[e * NC + lane] - ae * Y;
      if (serial0 && lane == 0)
        for (int l = s; l <= e; ++l) s0[l] = tile[(size_t)l * NC];  // column 0's right-hand side
    }
    __syncthreads();
    // ---- B: the reduced system of the 2P chunk-end values
    if (w == 0) {
      T Dp = 0, Yp = 0;
      for (int r = 0; r < 2 * P; ++r) {
        T* Rr = red + (size_t)r * 4 * NC;
        const T sub = Rr[0 * NC + lane], dg = Rr[1 * NC + lane], sup = Rr[2 * NC + lane], rhs = Rr[3 * NC + lane];
        const T rr = recip_rn(r == 0 ? dg : dg - sub * Dp);
        Dp = sup * rr;
        Yp = (r == 0 ? rhs : rhs - sub * Yp) * rr;
        Rr[0 * NC + lane] = Dp;
        Rr[1 * NC + lane] = Yp;
      }
      T x = Yp;
      xb[(2 * P - 1) * NC + lane] = x;
      for (int r = 2 * P - 2; r >= 0; --r) {
        const T* Rr = red + (size_t)r * 4 * NC;
        x = Rr[1 * NC + lane] - Rr[0 * NC + lane] * x;
        xb[r * NC + lane] = x;
      }
    }
    __syncthreads();
    // ---- C: the chunk's interior rows with x_s and x_e known, then its rows
    // out (column 0 of block 0 waits for the serial solve)
    {
      const T xs = xb[(2 * w) * NC + lane], xe = xb[(2 * w + 1) * NC + lane];
      T Y = 0;
#pragma unroll
      for (int t = 0; t < CH - 2; ++t) {
        const int i = s + 1 + t;
        const T ai = (T)__ldg(a + i), ci = (T)__ldg(c + i);
        T rhs = tile[i * NC + lane];
        if (t == 0) rhs -= ai * xs;
        if (t == CH - 3) rhs -= ci * xe;  // row e-1: x_e is known, no super-diagonal left
        Y = (t == 0 ? rhs : rhs - ai * Y) * rp[t];
        tile[i * NC + lane] = Y;
      }
      T* out = work + col0 + lane;
      const bool keep = !(serial0 && lane == 0);
      if (keep) {
        out[(size_t)s * ncol] = xs;
        out[(size_t)e * ncol] = xe;
        out[(size_t)(e - 1) * ncol] = Y;
      }
      T x = Y;
#pragma unroll
      for (int t = CH - 4; t >= 0; --t) {
        const int i = s + 1 + t;
        x = tile[i * NC + lane] - ((T)__ldg(c + i) * rp[t]) * x;
        if (keep) out[(size_t)i * ncol] = x;
      }
    }
    if (serial0 && threadIdx.x == 0) {
      // gaussel's elimination order and rounding for the singular mode
      T* pv = s0;
      T* dd = s0 + nz;
      const bool pin = sizeof(T) == 4 && zsing;
      T dprev = 0, pprev = 0;
      for (int l = 0; l < nz; ++l) {
        const T z = piv_inv<T>(l, nz, (T)__ldg(b + l), (T)0, (T)__ldg(a + l), dprev, pin);
        const T d = R::mul((T)__ldg(c + l), z);
        const T pn = l == 0 ? R::mul(pv[l], z) : R::mul(R::sub(pv[l], R::mul((T)__ldg(a + l), pprev)), z);
        dd[l] = d;
        pv[l] = pn;
        dprev = d;
        pprev = pn;
      }
      T pnext = 0;
      for (int l = nz - 1; l >= 0; --l) {
        if (l < nz - 1) pv[l] = R::sub(pv[l], R::mul(dd[l], pnext));
        pnext = pv[l];
        work[(size_t)l * ncol] = pv[l];
      }
    }
  }
};
template <typename T, int CH>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2) k_zsolve_part(int ncol, int nz, const double* __restrict__ lam,
    const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
    const DevScalars* __restrict__ sc, T* __restrict__ work, int zsing) {
  ZSolvePart<T, CH>::run(blk_here(), ncol, nz, lam, a, b, c, sc, work, zsing);
}

// periodic z: gaussel_periodic (src/solver.f90:107-149)
template <typename T>
struct ZSolvePeriodic {
  static __device__ __forceinline__ void run(const Blk& bk, int ncol, int nz, const double* __restrict__ lam,
      const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
      const DevScalars* __restrict__ sc, T* __restrict__ work, T* __restrict__ work2) {
    if (HALTED(sc)) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* dchk = reinterpret_cast<T*>(smraw);
    const int col = bk.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int n = nz;
    const double lmd = __ldg(lam + col);
    const T lm = (T)lmd;
    T* p = work + col;
    T* p2 = work2 + col;
    const size_t st = (size_t)ncol;
    // p1 = solution of the (n-1) system with the RHS, in place
    thomas_column<T>(n - 1, a, b, c, lm, p, st, dchk + threadIdx.x, blockDim.x, false);
    // p2 = solution with the spike RHS
    for (int k = 0; k < n - 1; ++k) p2[(size_t)k * st] = 0;
    p2[0] = (T)-a[0];
    p2[(size_t)(n - 2) * st] = (T)-c[n - 2];
    thomas_column<T>(n - 1, a, b, c, lm, p2, st, dchk + threadIdx.x, blockDim.x, false);
    const T bbn = (T)b[n - 1] + lm;
    const T den = bbn + (T)c[n - 1] * p2[0] + (T)a[n - 1] * p2[(size_t)(n - 2) * st] + (T)CANSFZ_EPS;
    T pn = (p[(size_t)(n - 1) * st] - (T)c[n - 1] * p[0] - (T)a[n - 1] * p[(size_t)(n - 2) * st]) / den;
    if (sizeof(T) == 4 && lmd == 0.) pn = 0;  // FP32: pin the singular mode
    p[(size_t)(n - 1) * st] = pn;
    for (int k = 0; k < n - 1; ++k) p[(size_t)k * st] = p[(size_t)k * st] + p2[(size_t)k * st] * pn;
  }
};
template <typename T>
__global__ void __launch_bounds__(128) k_zsolve_periodic(int ncol, int nz, const double* __restrict__ lam,
    const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
    const DevScalars* __restrict__ sc, T* __restrict__ work, T* __restrict__ work2) {
  ZSolvePeriodic<T>::run(blk_here(), ncol, nz, lam, a, b, c, sc, work, work2);
}

// periodic z with the precomputed factors (those of the first n-1 levels)
template <typename T>
struct ZSolvePeriodicF {
  static __device__ __forceinline__ void run(const Blk& bk, int ncol, int nz, const double* __restrict__ lam,
      const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
      const T* __restrict__ piv, const T* __restrict__ df, const DevScalars* __restrict__ sc,
      T* __restrict__ work, T* __restrict__ work2) {
    if (HALTED(sc)) return;
    const int col = bk.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int n = nz;
    const double lmd = __ldg(lam + col);
    const T lm = (T)lmd;
    T* p = work + col;
    T* p2 = work2 + col;
    const size_t st = (size_t)ncol;
    thomas_factored<T>(n - 1, a, piv + col, df + col, p, st);
    for (int k = 0; k < n - 1; ++k) p2[(size_t)k * st] = 0;
    p2[0] = (T)-a[0];
    p2[(size_t)(n - 2) * st] = (T)-c[n - 2];
    thomas_factored<T>(n - 1, a, piv + col, df + col, p2, st);
    const T bbn = (T)b[n - 1] + lm;
    const T den = bbn + (T)c[n - 1] * p2[0] + (T)a[n - 1] * p2[(size_t)(n - 2) * st] + (T)CANSFZ_EPS;
    T pn = (p[(size_t)(n - 1) * st] - (T)c[n - 1] * p[0] - (T)a[n - 1] * p[(size_t)(n - 2) * st]) / den;
    if (sizeof(T) == 4 && lmd == 0.) pn = 0;  // FP32: pin the singular mode
    p[(size_t)(n - 1) * st] = pn;
    for (int k = 0; k < n - 1; ++k) p[(size_t)k * st] = p[(size_t)k * st] + p2[(size_t)k * st] * pn;
  }
};
template <typename T>
__global__ void __launch_bounds__(128) k_zsolve_periodic_f(int ncol, int nz, const double* __restrict__ lam,
    const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
    const T* __restrict__ piv, const T* __restrict__ df, const DevScalars* __restrict__ sc, T* __restrict__ work,
    T* __restrict__ work2) {
  ZSolvePeriodicF<T>::run(blk_here(), ncol, nz, lam, a, b, c, piv, df, sc, work, work2);
}

// ---------------------------------------------------------------------------
// FP64 residual of the discrete operator the spectral solve inverts: the
// 7-point Laplacian with the BC ghosts of cbcpre (chk_poisson,
// src/debug.f90:100-106).  res = rhs - L(phi) on the interior; phi's ghost
// layer must be filled (boundp) before.
// ---------------------------------------------------------------------------
struct Residual {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const DevScalars* __restrict__ sc,
      const double* __restrict__ rhs, const double* __restrict__ phi, double* __restrict__ res) {
    if (HALTED(sc)) return;
    const int i = bk.x * blockDim.x + threadIdx.x + 1;
    if (i > g.nx) return;
    const int j = bk.y + 1, k = bk.z + 1;
    const int c = g.h(i, j, k);
    const double pc = __ldg(phi + c);
    const double lap = (__ldg(phi + c + 1) - 2. * pc + __ldg(phi + c - 1)) * (g.dxi * g.dxi) +
                       (__ldg(phi + c + g.sx) - 2. * pc + __ldg(phi + c - g.sx)) * (g.dyi * g.dyi) +
                       ((__ldg(phi + c + g.sxy) - pc) * g.dzci[k] - (pc - __ldg(phi + c - g.sxy)) * g.dzci[k - 1]) *
                           g.dzfi[k];
    res[c] = __ldg(rhs + c) - lap;
  }
};
__global__ void k_residual(Geo g, const DevScalars* __restrict__ sc, const double* __restrict__ rhs,
                           const double* __restrict__ phi, double* __restrict__ res) {
  Residual::run(blk_here(), g, sc, rhs, phi, res);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// lines per CTA: keep the 4*m*LP elements of shared memory within ~96 KB
constexpr int lines_per_cta(int m, int maxL, int tsize) {
  int L = maxL;
  while (L > 1 && 4LL * m * (L | 1) * tsize > 96 * 1024) L >>= 1;
  return L;
}
constexpr int x_maxL(int m) { return 2 * m >= 128 ? 4 : 16; }
// y lines per CTA: 16, and more for very short lines (ny = 2 in the 2-D
// convention), which would otherwise leave most threads of a CTA idle and
// launch nx/16 * nz CTAs of a few points each
constexpr int y_maxL(int m) { return 2 * m >= 32 ? 16 : (2 * m >= 8 ? 64 : 256); }
template <typename T, int MC>
constexpr int xL() { return MC ? lines_per_cta(MC, x_maxL(MC), sizeof(T)) : 0; }
template <typename T, int MC>
constexpr int yL() { return MC ? lines_per_cta(MC, y_maxL(MC), sizeof(T)) : 0; }

// the compile-time complex lengths (real lines of 32 to 512 points with
// factors 2 and 3); other lengths take the runtime-length kernels
#define CANSFZ_FOR_LENGTHS(X) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256)

template <typename T, int MC>
static void set_attr_len() {
  const int lim = 100 * 1024;
  cudaFuncSetAttribute(k_fft_x_fwd<T, true, MC, xL<T, MC>()>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_x_fwd<T, false, MC, xL<T, MC>()>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_x_bwd<T, false, MC, xL<T, MC>()>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_x_bwd<T, true, MC, xL<T, MC>()>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_y<T, 1, MC, yL<T, MC>()>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_y<T, -1, MC, yL<T, MC>()>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

// opt the transform kernels into > 48 KB of dynamic shared memory (once)
template <typename T, int CH>
static void set_attr_zpart() {
  cudaFuncSetAttribute(k_zsolve_part<T, CH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)zpart_smem<T>(CH * ZP_P));
  // all of the unified L1/shared storage as shared memory: 2 FP64 or 4 FP32
  // tiles per SM
  cudaFuncSetAttribute(k_zsolve_part<T, CH>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

void poisson_set_attributes() {
#define X(C) set_attr_zpart<double, C>(); set_attr_zpart<float, C>();
  CANSFZ_FOR_ZCHUNKS(X)
#undef X
  set_attr_len<double, 0>();
  set_attr_len<float, 0>();
#define X(M) set_attr_len<double, M>(); set_attr_len<float, M>();
  CANSFZ_FOR_LENGTHS(X)
#undef X
}

template <typename T> static T* wbuf(const PoissonPlan& pl);
template <> double* wbuf<double>(const PoissonPlan& pl) { return pl.work; }
template <> float* wbuf<float>(const PoissonPlan& pl) { return pl.workf; }
template <typename T> static T* wbuf2(const PoissonPlan& pl);
template <> double* wbuf2<double>(const PoissonPlan& pl) { return pl.work2; }
template <> float* wbuf2<float>(const PoissonPlan& pl) { return pl.work2f; }

template <typename T, int MC>
static void x_forward_len(const Launch& Lc, const Geo& g, const PoissonPlan& pl, const DevScalars* sc,
                          const double* src, const double* u, const double* v, const double* w, const Phys* ph,
                          bool fused) {
  const int m = pl.px.m < 1 ? 1 : pl.px.m;
  const int L = MC ? xL<T, MC>() : lines_per_cta(m, x_maxL(m), sizeof(T));
  const size_t smem = 4 * (size_t)m * (L | 1) * sizeof(T);
  const int nlines = g.ny * g.nz;
  const dim3 grid((nlines + L - 1) / L);
  Phys pz{};
  // the two-pass x forward; with fillps fused in (11 loads per sample pair),
  // lines of 128 and 256 points keep the one-warp-per-line kernel, whose
  // lanes hold 4 or 8 samples instead of 32 (0.158 against 0.184 ms at 256^3)
  if constexpr (y2_length(MC)) {
    if (pl.px.kind == 0 && pl.lmode == 0 && !(fused && (MC == 64 || MC == 128))) {
      using X = FftX2Fwd<T, true, MC>;
      const dim3 g2((nlines + X::L - 1) / X::L);
      if (fused)
        kgo<FftX2Fwd<T, true, MC>, X::NT, 3>(Lc, k_fft_x2_fwd<T, true, MC>, g2, X::NT, 0, g, pl.px, sc, nullptr, u, v,
                                            w, *ph, wbuf<T>(pl));
      else
        kgo<FftX2Fwd<T, false, MC>, X::NT, 3>(Lc, k_fft_x2_fwd<T, false, MC>, g2, X::NT, 0, g, pl.px, sc, src,
                                             nullptr, nullptr, nullptr, pz, wbuf<T>(pl));
      return;
    }
  }
  if constexpr (MC == 64 || MC == 128) {
    if (pl.px.kind == 0) {
      constexpr int R = MC / 32;
      const dim3 gw((nlines + 8 * kWarpLines - 1) / (8 * kWarpLines));
      if (fused)
        kgo<FftXFwdW<T, true, R>, 256, 1>(Lc, k_fft_x_fwd_w<T, true, R>, gw, 256, 0, g, pl.px, sc, nullptr, u, v, w,
                                          *ph, wbuf<T>(pl));
      else
        kgo<FftXFwdW<T, false, R>, 256, 1>(Lc, k_fft_x_fwd_w<T, false, R>, gw, 256, 0, g, pl.px, sc, src, nullptr,
                                           nullptr, nullptr, pz, wbuf<T>(pl));
      return;
    }
  }
  if (fused)
    kgo<FftXFwd<T, true, MC, xL<T, MC>()>, 256, 1>(Lc, k_fft_x_fwd<T, true, MC, xL<T, MC>()>, grid, 256, smem, g,
                                                   pl.px, sc, nullptr, u, v, w, *ph, wbuf<T>(pl), L);
  else
    kgo<FftXFwd<T, false, MC, xL<T, MC>()>, 256, 1>(Lc, k_fft_x_fwd<T, false, MC, xL<T, MC>()>, grid, 256, smem, g,
                                                    pl.px, sc, src, nullptr, nullptr, nullptr, pz, wbuf<T>(pl), L);
}

template <typename T>
static void x_forward(const Launch& Lc, const Geo& g, const PoissonPlan& pl, const DevScalars* sc,
                      const double* src, const double* u, const double* v, const double* w, const Phys* ph,
                      bool fused) {
  switch (pl.px.m) {
#define X(M) case M: x_forward_len<T, M>(Lc, g, pl, sc, src, u, v, w, ph, fused); return;
    CANSFZ_FOR_LENGTHS(X)
#undef X
    default: x_forward_len<T, 0>(Lc, g, pl, sc, src, u, v, w, ph, fused);
  }
}

template <typename T, int MC>
static void y_pass_len(const Launch& Lc, const Geo& g, const PoissonPlan& pl, const DevScalars* sc, int dir) {
  const int m = pl.py.m < 1 ? 1 : pl.py.m;
  if constexpr (y2_length(MC)) {
    if (pl.py.kind == 0 && pl.lmode == 0) {
      using Y = FftY2<T, 1, MC>;
      const dim3 g2((g.nx + Y::L - 1) / Y::L, g.nz);
      if (dir > 0)
        kgo<FftY2<T, 1, MC>, Y::NT, 3>(Lc, k_fft_y2<T, 1, MC>, g2, Y::NT, 0, g, pl.py, sc, wbuf<T>(pl));
      else
        kgo<FftY2<T, -1, MC>, Y::NT, 3>(Lc, k_fft_y2<T, -1, MC>, g2, Y::NT, 0, g, pl.py, sc, wbuf<T>(pl));
      return;
    }
  }
  const int L = MC ? yL<T, MC>() : lines_per_cta(m, y_maxL(m), sizeof(T));
  const size_t smem = 4 * (size_t)m * (L | 1) * sizeof(T);
  const dim3 grid((g.nx + L - 1) / L, g.nz);
  if (dir > 0)
    kgo<FftY<T, 1, MC, yL<T, MC>()>, 256, 1>(Lc, k_fft_y<T, 1, MC, yL<T, MC>()>, grid, 256, smem, g, pl.py, sc,
                                             wbuf<T>(pl), L);
  else
    kgo<FftY<T, -1, MC, yL<T, MC>()>, 256, 1>(Lc, k_fft_y<T, -1, MC, yL<T, MC>()>, grid, 256, smem, g, pl.py, sc,
                                              wbuf<T>(pl), L);
}

template <typename T>
static void y_pass(const Launch& Lc, const Geo& g, const PoissonPlan& pl, const DevScalars* sc, int dir) {
  switch (pl.py.m) {
#define X(M) case M: y_pass_len<T, M>(Lc, g, pl, sc, dir); return;
    CANSFZ_FOR_LENGTHS(X)
#undef X
    default: y_pass_len<T, 0>(Lc, g, pl, sc, dir);
  }
}

template <typename T> static const T* zpiv(const PoissonPlan& pl);
template <> const double* zpiv<double>(const PoissonPlan& pl) { return pl.zpiv; }
template <> const float* zpiv<float>(const PoissonPlan& pl) { return pl.zpivf; }
template <typename T> static const T* zdf(const PoissonPlan& pl);
template <> const double* zdf<double>(const PoissonPlan& pl) { return pl.zdf; }
template <> const float* zdf<float>(const PoissonPlan& pl) { return pl.zdff; }

void launch_z_factors(const Launch& L, const Geo& g, const PoissonPlan& pl, bool f32, void* piv, void* df) {
  const int ncol = g.nx * g.ny, tb = 128;
  if (f32)
    k_z_factors<float><<<(ncol + tb - 1) / tb, tb, 0, L.st>>>(ncol, g.nz, pl.lam, pl.a, pl.b, pl.c, pl.zsing,
                                                             static_cast<float*>(piv), static_cast<float*>(df));
  else
    k_z_factors<double><<<(ncol + tb - 1) / tb, tb, 0, L.st>>>(ncol, g.nz, pl.lam, pl.a, pl.b, pl.c, pl.zsing,
                                                              static_cast<double*>(piv), static_cast<double*>(df));
}

template <typename T, int CH>
static void z_part_len(const Launch& Lc, const Geo& g, const PoissonPlan& pl, const DevScalars* sc) {
  const int ncol = g.nx * g.ny;
  kgo<ZSolvePart<T, CH>, 256, sizeof(T) == 4 ? 4 : 2>(Lc, k_zsolve_part<T, CH>, ncol / ZP_NC, 32 * ZP_P, zpart_smem<T>(g.nz), ncol,
                                 g.nz, pl.lam, pl.a, pl.b, pl.c, sc, wbuf<T>(pl), pl.zsing);
}

bool poisson_y2_applies(const PoissonPlan& pl) {
  return (pl.py.kind == 0 && y2_length(pl.py.m)) || (pl.px.kind == 0 && y2_length(pl.px.m));
}

// the partitioned solve serves non-periodic z with nz = 8 * CH and whole
// tiles of columns; few-column grids keep the factored solve
bool z_part_ok(const Geo& g, const PoissonPlan& pl) {
  const int ncol = g.nx * g.ny;
  if (pl.zper || ncol % ZP_NC != 0 || g.nz % ZP_P != 0) return false;
  switch (g.nz / ZP_P) {
#define X(C) case C:
    CANSFZ_FOR_ZCHUNKS(X)
#undef X
    return true;
    default: return false;
  }
}

template <typename T>
static void z_pass(const Launch& Lc, const Geo& g, const PoissonPlan& pl, const DevScalars* sc) {
  const int ncol = g.nx * g.ny;
  const int tb = 64;
  if (pl.zmode != 1 && !(zpiv<T>(pl) && zdf<T>(pl)) && z_part_ok(g, pl)) {
    switch (g.nz / ZP_P) {
#define X(C) case C: z_part_len<T, C>(Lc, g, pl, sc); return;
      CANSFZ_FOR_ZCHUNKS(X)
#undef X
      default: break;
    }
  }
  if (zpiv<T>(pl) && zdf<T>(pl)) {
    if (pl.zper)
      kgo<ZSolvePeriodicF<T>, 128, 1>(Lc, k_zsolve_periodic_f<T>, (ncol + tb - 1) / tb, tb, 0, ncol, g.nz, pl.lam,
                                      pl.a, pl.b, pl.c, zpiv<T>(pl), zdf<T>(pl), sc, wbuf<T>(pl), wbuf2<T>(pl));
    else
      kgo<ZSolveF<T>, 128, 1>(Lc, k_zsolve_f<T>, (ncol + tb - 1) / tb, tb, 0, ncol, g.nz, pl.a, zpiv<T>(pl),
                              zdf<T>(pl), sc, wbuf<T>(pl));
    return;
  }
  const int nch = (g.nz + ZCH - 1) / ZCH;
  const size_t smem = (size_t)nch * tb * sizeof(T);
  if (pl.zper)
    kgo<ZSolvePeriodic<T>, 128, 1>(Lc, k_zsolve_periodic<T>, (ncol + tb - 1) / tb, tb, smem, ncol, g.nz, pl.lam,
                                   pl.a, pl.b, pl.c, sc, wbuf<T>(pl), wbuf2<T>(pl));
  else
    kgo<ZSolve<T>, 128, 1>(Lc, k_zsolve<T>, (ncol + tb - 1) / tb, tb, smem, ncol, g.nz, pl.lam, pl.a, pl.b, pl.c,
                           sc, wbuf<T>(pl), pl.zsing);
}

template <typename T, bool ADD, int MC>
static void x_backward_len(const Launch& Lc, const Geo& g, const PoissonPlan& pl, const DevScalars* sc,
                           double* dst) {
  const int m = pl.px.m < 1 ? 1 : pl.px.m;
  const int L = MC ? xL<T, MC>() : lines_per_cta(m, x_maxL(m), sizeof(T));
  const size_t smem = 4 * (size_t)m * (L | 1) * sizeof(T);
  const int nlines = g.ny * g.nz;
  if constexpr (y2_length(MC)) {
    if (pl.px.kind == 0 && pl.lmode == 0) {
      using X = FftX2Bwd<T, ADD, MC>;
      kgo<FftX2Bwd<T, ADD, MC>, X::NT, 4>(Lc, k_fft_x2_bwd<T, ADD, MC>, (nlines + X::L - 1) / X::L, X::NT, 0, g,
                                         pl.px, sc, wbuf<T>(pl), pl.normfft, dst, ADD ? 0 : Lc.wrap);
      return;
    }
  }
  if constexpr (MC == 64 || MC == 128) {
    if (pl.px.kind == 0) {
      constexpr int R = MC / 32;
      kgo<FftXBwdW<T, ADD, R>, 256, 1>(Lc, k_fft_x_bwd_w<T, ADD, R>, (nlines + 8 * kWarpLines - 1) / (8 * kWarpLines),
                                       256, 0, g, pl.px, sc, wbuf<T>(pl), pl.normfft, dst, ADD ? 0 : Lc.wrap);
      return;
    }
  }
  kgo<FftXBwd<T, ADD, MC, xL<T, MC>()>, 256, 1>(Lc, k_fft_x_bwd<T, ADD, MC, xL<T, MC>()>, (nlines + L - 1) / L, 256,
                                                smem, g, pl.px, sc, wbuf<T>(pl), pl.normfft, dst, L,
                                                ADD ? 0 : Lc.wrap);
}

template <typename T, bool ADD>
static void x_backward(const Launch& Lc, const Geo& g, const PoissonPlan& pl, const DevScalars* sc, double* dst) {
  switch (pl.px.m) {
#define X(M) case M: x_backward_len<T, ADD, M>(Lc, g, pl, sc, dst); return;
    CANSFZ_FOR_LENGTHS(X)
#undef X
    default: x_backward_len<T, ADD, 0>(Lc, g, pl, sc, dst);
  }
}

// solver_gpu on the interior of the halo-layout field p (in place)
void launch_poisson(const Launch& L, const Geo& g, const PoissonPlan& pl, const DevScalars* sc, double* p,
                    const StageMark* mk) {
  x_forward<double>(L, g, pl, sc, p, nullptr, nullptr, nullptr, nullptr, false);
  if (mk) mk->mark("poisson_x_fwd");
  y_pass<double>(L, g, pl, sc, +1);
  if (mk) mk->mark("poisson_y_fwd");
  z_pass<double>(L, g, pl, sc);
  if (mk) mk->mark("poisson_z_solve");
  y_pass<double>(L, g, pl, sc, -1);
  if (mk) mk->mark("poisson_y_bwd");
  x_backward<double, false>(L, g, pl, sc, p);
  if (mk) mk->mark("poisson_x_bwd");
}

// fillps + solver_gpu: the RHS is formed inside the x transform from u, v, w;
// phi (the interior of a halo-layout field) receives the solution.
void launch_poisson_fused_rhs(const Launch& L, const Geo& g, const PoissonPlan& pl, const Phys& ph,
                              const DevScalars* sc, const double* u, const double* v, const double* w,
                              const double* rhsb_planes, double* phi, const StageMark* mk) {
  (void)rhsb_planes;
  x_forward<double>(L, g, pl, sc, nullptr, u, v, w, &ph, true);
  if (mk) mk->mark("poisson_x_fwd_fillps");
  y_pass<double>(L, g, pl, sc, +1);
  if (mk) mk->mark("poisson_y_fwd");
  z_pass<double>(L, g, pl, sc);
  if (mk) mk->mark("poisson_z_solve");
  y_pass<double>(L, g, pl, sc, -1);
  if (mk) mk->mark("poisson_y_bwd");
  x_backward<double, false>(L, g, pl, sc, phi);
  if (mk) mk->mark("poisson_x_bwd");
}

// FP32 spectral solve of the mixed form: dst = S(src), or dst += S(src) (add)
void launch_poisson_f32(const Launch& L, const Geo& g, const PoissonPlan& pl, const DevScalars* sc,
                        const double* src, double* dst, bool add, const StageMark* mk) {
  DevScalars* scw = const_cast<DevScalars*>(sc);  // the tensor-core passes report a timed-out wait there
  if (pl.gx[0]) launch_xform_gemm(L, g, 0, false, pl.gx[0], g.nx, src, pl.workf, 1., scw);
  else x_forward<float>(L, g, pl, sc, src, nullptr, nullptr, nullptr, nullptr, false);
  if (pl.gy[0]) launch_xform_gemm(L, g, 1, false, pl.gy[0], g.ny, pl.workf, pl.workf, 1., scw);
  else y_pass<float>(L, g, pl, sc, +1);
  z_pass<float>(L, g, pl, sc);
  if (pl.gy[1]) launch_xform_gemm(L, g, 1, false, pl.gy[1], g.ny, pl.workf, pl.workf, 1., scw);
  else y_pass<float>(L, g, pl, sc, -1);
  if (pl.gx[1]) launch_xform_gemm(L, g, 2, add, pl.gx[1], g.nx, pl.workf, dst, pl.normfft, scw);
  else if (add) x_backward<float, true>(L, g, pl, sc, dst);
  else x_backward<float, false>(L, g, pl, sc, dst);
  if (mk) mk->mark(add ? "poisson_f32_correction" : "poisson_f32");
}

void launch_residual(const Launch& L, const Geo& g, const DevScalars* sc, const double* rhs, const double* phi,
                     double* res) {
  const int bx = g.nx >= 128 ? 128 : (g.nx >= 64 ? 64 : 32);
  kgo<Residual, 128, 1>(L, k_residual, dim3((g.nx + bx - 1) / bx, g.ny, g.nz), bx, 0, g, sc, rhs, phi, res);
}

}  // namespace cansfz
