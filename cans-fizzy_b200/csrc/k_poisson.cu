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
    auto get = [&](int it) -> double {
      const int line = it / n, i = it - line * n;
      const int gl = l0 + line;
      double x = 0.;
      if (gl < nlines) {
        const int j = gl % g.ny + 1, k = gl / g.ny + 1;
        const int c = g.h(i + 1, j, k);
        if (FUSED) {
          x = ph.rho0 * ((__ldg(w + c) - __ldg(w + c - g.sxy)) * dti * g.dzfi[k] +
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
template <typename T, bool ADD, int MC, int LC>
struct FftXBwd {
  static __device__ __forceinline__ void run(const Blk& bk, const Geo& g, const LinePlan& pl,
      const DevScalars* __restrict__ sc, const T* __restrict__ work, double normfft, double* __restrict__ dst,
      int Lrt) {
    if (HALTED(sc)) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    T* sm = reinterpret_cast<T*>(smraw);
    const int n = MC ? 2 * MC : pl.n, m = MC ? MC : pl.m;
    const int L = LC ? LC : Lrt;
    const Bufs<T> B = smem_bufs<T>(sm, m < 1 ? 1 : m, L);
    const int nlines = g.ny * g.nz;
    const int l0 = bk.x * L;
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
      const int gl = l0 + line;
      if (gl < nlines) {
        const int j = gl % g.ny + 1, k = gl / g.ny + 1;
        const int c = g.h(i + 1, j, k);
        if (ADD) dst[c] = dst[c] + (double)val * normfft;
        else dst[c] = (double)val * normfft;
      }
    });
  }
};
template <typename T, bool ADD, int MC, int LC>
__global__ void __launch_bounds__(256) k_fft_x_bwd(Geo g, LinePlan pl, const DevScalars* __restrict__ sc,
    const T* __restrict__ work, double normfft, double* __restrict__ dst, int Lrt) {
  FftXBwd<T, ADD, MC, LC>::run(blk_here(), g, pl, sc, work, normfft, dst, Lrt);
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
void poisson_set_attributes() {
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

template <typename T>
static void z_pass(const Launch& Lc, const Geo& g, const PoissonPlan& pl, const DevScalars* sc) {
  const int ncol = g.nx * g.ny;
  const int tb = 64;
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
  kgo<FftXBwd<T, ADD, MC, xL<T, MC>()>, 256, 1>(Lc, k_fft_x_bwd<T, ADD, MC, xL<T, MC>()>, (nlines + L - 1) / L, 256,
                                                smem, g, pl.px, sc, wbuf<T>(pl), pl.normfft, dst, L);
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
  x_forward<float>(L, g, pl, sc, src, nullptr, nullptr, nullptr, nullptr, false);
  y_pass<float>(L, g, pl, sc, +1);
  z_pass<float>(L, g, pl, sc);
  y_pass<float>(L, g, pl, sc, -1);
  if (add) x_backward<float, true>(L, g, pl, sc, dst);
  else x_backward<float, false>(L, g, pl, sc, dst);
  if (mk) mk->mark(add ? "poisson_f32_correction" : "poisson_f32");
}

void launch_residual(const Launch& L, const Geo& g, const DevScalars* sc, const double* rhs, const double* phi,
                     double* res) {
  const int bx = g.nx >= 128 ? 128 : (g.nx >= 64 ? 64 : 32);
  kgo<Residual, 128, 1>(L, k_residual, dim3((g.nx + bx - 1) / bx, g.ny, g.nz), bx, 0, g, sc, rhs, phi, res);
}

}  // namespace cansfz
