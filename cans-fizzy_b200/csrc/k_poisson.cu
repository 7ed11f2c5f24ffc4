// Constant-coefficient Poisson solve of solver_gpu (src/solver_gpu.f90:31-163)
// on one GPU, 1x1 pencil, FP64.  No transposes: the x lines are contiguous
// rows, the y lines are read as column tiles of TL consecutive x positions,
// and the z tridiagonal systems are solved one column per thread.
//
//   x: real transform of each row    (R2HC packed / DCT-II / DST-II)
//   y: real transform of each column (same kinds, per BC)
//   z: Thomas per (x,y) mode with b + lambda_x + lambda_y (gaussel_gpu,
//      src/solver_gpu.f90:165-230), Sherman-Morrison for periodic z
//      (gaussel_periodic_gpu, :232-370)
//   y, x: inverse transforms; x inverse scales by normfft and writes the
//      interior of the halo-layout output.
//
// Line transforms: a complex FFT of length m = n/2 (the real sequence packed
// as z_j = x_2j + i x_2j+1), Stockham auto-sort, radix 4/2/3 (generic radix
// via the twiddle table), in shared memory laid out position-major /
// line-minor so that consecutive threads touch consecutive lines.  The
// periodic kind stores the spectrum as (r0, r_{n/2}, r1, i1, r2, i2, ...);
// the eigenvalues are permuted to that order on the host.  The cosine and
// sine kinds follow Makhoul's reordering (as src/fft.f90:320-658 does).
#include "cansfz_internal.cuh"

namespace cansfz {

#define HALTED(sc) ((sc) != nullptr && (sc)->halted)

struct Bufs {
  double* re[2];
  double* im[2];
  int LP;  // line pitch in shared memory (odd: conflict-free strided access)
};

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 mul_i(double2 a) { return make_double2(-a.y, a.x); }  // i*a

__device__ __forceinline__ double2 ld2(const Bufs& B, int b, int pos, int line) {
  const int q = pos * B.LP + line;
  return make_double2(B.re[b][q], B.im[b][q]);
}
__device__ __forceinline__ void st2(const Bufs& B, int b, int pos, int line, double2 v) {
  const int q = pos * B.LP + line;
  B.re[b][q] = v.x;
  B.im[b][q] = v.y;
}
// raw real position s of a line stored as complex pairs (s even: re, odd: im)
__device__ __forceinline__ double ldr(const Bufs& B, int b, int s, int line) {
  const int q = (s >> 1) * B.LP + line;
  return (s & 1) ? B.im[b][q] : B.re[b][q];
}
__device__ __forceinline__ void str(const Bufs& B, int b, int s, int line, double v) {
  const int q = (s >> 1) * B.LP + line;
  if (s & 1) B.im[b][q] = v; else B.re[b][q] = v;
}

// complex FFT (sign -1 forward, +1 backward) of length pl.m on L lines held
// in buffer `in`; returns the buffer index holding the result.
__device__ int fft_lines(const LinePlan& pl, const Bufs& B, int in, int L, int sign) {
  const int m = pl.m;
  int len = m, s = 1, cur = in;
  for (int st = 0; st < pl.nst; ++st) {
    const int r = pl.radix[st];
    const int mm = len / r;
    const int tstep = m / len;  // exp(-2 pi i p u / len) = tw[p*u*tstep]
    const int nb = m / r;       // butterflies per line (= mm * s)
    const int nxt = cur ^ 1;
    for (int it = threadIdx.x; it < L * nb; it += blockDim.x) {
      const int line = it % L, b = it / L;
      const int p = b / s, q = b - p * s;
      auto put = [&](int u, double2 y) {
        if (u > 0 && p > 0) {
          double2 wp = __ldg(&pl.tw[(p * u * tstep) % m]);
          if (sign > 0) wp = cconj(wp);
          y = cmul(y, wp);
        }
        st2(B, nxt, q + s * (r * p + u), line, y);
      };
      if (r == 2) {
        const double2 a0 = ld2(B, cur, q + s * p, line), a1 = ld2(B, cur, q + s * (p + mm), line);
        put(0, cadd(a0, a1));
        put(1, csub(a0, a1));
      } else if (r == 4) {
        const double2 a0 = ld2(B, cur, q + s * p, line), a1 = ld2(B, cur, q + s * (p + mm), line);
        const double2 a2 = ld2(B, cur, q + s * (p + 2 * mm), line), a3 = ld2(B, cur, q + s * (p + 3 * mm), line);
        const double2 t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = csub(a1, a3);
        // W4 = exp(sign * i pi / 2) = sign * i
        const double2 it3 = sign < 0 ? make_double2(t3.y, -t3.x) : make_double2(-t3.y, t3.x);  // W4 * t3
        put(0, cadd(t0, t2));
        put(1, cadd(t1, it3));
        put(2, csub(t0, t2));
        put(3, csub(t1, it3));
      } else if (r == 3) {
        const double2 a0 = ld2(B, cur, q + s * p, line), a1 = ld2(B, cur, q + s * (p + mm), line);
        const double2 a2 = ld2(B, cur, q + s * (p + 2 * mm), line);
        const double2 t1 = cadd(a1, a2), t2 = csub(a1, a2);
        const double c3 = 0.86602540378443864676 * (double)(-sign);  // -sign*sqrt(3)/2
        const double2 base = make_double2(a0.x - 0.5 * t1.x, a0.y - 0.5 * t1.y);
        const double2 rot = make_double2(c3 * t2.y, -c3 * t2.x);  // -i * c3 * t2
        put(0, cadd(a0, t1));
        put(1, cadd(base, rot));
        put(2, csub(base, rot));
      } else {
        // generic radix (5, 7): direct r-point DFT with the twiddle table
        for (int u = 0; u < r; ++u) {
          double2 acc = make_double2(0., 0.);
          for (int v = 0; v < r; ++v) {
            double2 wv = __ldg(&pl.tw[((v * u) % r) * (m / r)]);
            if (sign > 0) wv = cconj(wv);
            acc = cadd(acc, cmul(ld2(B, cur, q + s * (p + v * mm), line), wv));
          }
          put(u, acc);
        }
      }
    }
    __syncthreads();
    cur = nxt;
    len = mm;
    s *= r;
  }
  return cur;
}

// post-processing of a forward real transform: X_k, k = 0..m, from Z
__device__ __forceinline__ double2 real_fwd_X(const LinePlan& pl, const Bufs& B, int zb, int k, int line) {
  const int m = pl.m;
  const double2 zk = ld2(B, zb, k % m, line);
  const double2 zc = cconj(ld2(B, zb, (m - k) % m, line));
  const double2 w = __ldg(&pl.tw2[k]);
  const double2 sum = make_double2(0.5 * (zk.x + zc.x), 0.5 * (zk.y + zc.y));
  const double2 dif = csub(zk, zc);
  const double2 wd = cmul(w, dif);
  // -i/2 * wd = (0.5*wd.y, -0.5*wd.x)
  return make_double2(sum.x + 0.5 * wd.y, sum.y - 0.5 * wd.x);
}

// Z_k = (X_k + conj X_{m-k}) + i (X_k - conj X_{m-k}) conj(W^k), k = 0..m-1
__device__ __forceinline__ double2 real_bwd_Z(const LinePlan& pl, double2 xk, double2 xmk, int k) {
  const double2 xc = cconj(xmk);
  const double2 w = cconj(__ldg(&pl.tw2[k]));
  return cadd(cadd(xk, xc), mul_i(cmul(csub(xk, xc), w)));
}

// packed spectrum of the periodic kind: complex index k -> X_k with
// X_0 = (r0, 0), X_m = (r_m, 0) both held in complex slot 0
__device__ __forceinline__ double2 packed_X(const Bufs& B, int b, int k, int m, int line) {
  if (k == 0) return make_double2(B.re[b][line], 0.);
  if (k == m) return make_double2(B.im[b][line], 0.);
  return ld2(B, b, k, line);
}

// ---------------------------------------------------------------------------
// the four line transforms on L lines already in shared memory
// ---------------------------------------------------------------------------
// forward: input real line in buffer 0 as pairs (x_2j, x_2j+1) (after the
// kind's input reordering); output real line written through `out(line, s, v)`
template <bool LF, typename OUT>
__device__ void line_forward(const LinePlan& pl, const Bufs& B, int L, OUT out) {
  const int m = pl.m, n = pl.n;
  const int zb = fft_lines(pl, B, 0, L, -1);
  if (pl.kind == 0) {
    for (int it = threadIdx.x; it < L * m; it += blockDim.x) {
      const int line = LF ? it % L : it / m, k = LF ? it / L : it - line * m;
      const double2 X = real_fwd_X(pl, B, zb, k, line);
      if (k == 0) {
        const double2 Xm = real_fwd_X(pl, B, zb, m, line);
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
      const double2 V = real_fwd_X(pl, B, zb, k, line);
      const double2 wk = __ldg(&pl.twc[k]);
      const double yk = 2. * (wk.x * V.x - wk.y * V.y);
      if (k < n) out(line, dst ? n - 1 - k : k, yk);
      if (k > 0 && k < m) {
        const double2 wn = __ldg(&pl.twc[n - k]);
        const double ynk = 2. * (wn.x * V.x + wn.y * V.y);  // Re(w_{n-k} conj(V_k))
        out(line, dst ? k - 1 : n - k, ynk);
      }
    }
  }
}

// backward: input real line (packed spectrum or natural DCT/DST coefficients)
// in buffer 1 as pairs; output real line through `out(line, i, v)`
template <bool LF, typename OUT>
__device__ void line_backward(const LinePlan& pl, const Bufs& B, int L, OUT out) {
  const int m = pl.m, n = pl.n;
  if (pl.kind == 0) {
    for (int it = threadIdx.x; it < L * m; it += blockDim.x) {
      const int line = it % L, k = it / L;
      st2(B, 0, k, line, real_bwd_Z(pl, packed_X(B, 1, k, m, line), packed_X(B, 1, m - k, m, line), k));
    }
  } else {
    const bool dst = pl.kind == 2;
    // X_k of the DCT-III (for the sine kind: the reversed input)
    auto X = [&](int k, int line) -> double {
      if (k >= n) return 0.;
      return ldr(B, 1, dst ? n - 1 - k : k, line);
    };
    auto V = [&](int k, int line) -> double2 {  // e^{i pi k/(2n)} (X_k - i X_{n-k})
      const double2 w = cconj(__ldg(&pl.twc[k]));
      const double2 a = make_double2(X(k, line), -X(n - k, line));
      return cmul(w, a);
    };
    for (int it = threadIdx.x; it < L * m; it += blockDim.x) {
      const int line = it % L, k = it / L;
      st2(B, 0, k, line, real_bwd_Z(pl, V(k, line), V(m - k, line), k));
    }
  }
  __syncthreads();
  const int zb = fft_lines(pl, B, 0, L, +1);
  if (pl.kind == 0) {
    for (int it = threadIdx.x; it < L * n; it += blockDim.x) {
      const int line = LF ? it % L : it / n, i = LF ? it / L : it - line * n;
      out(line, i, ldr(B, zb, i, line));
    }
  } else {
    const bool dst = pl.kind == 2;
    for (int it = threadIdx.x; it < L * n; it += blockDim.x) {
      const int line = LF ? it % L : it / n, i = LF ? it / L : it - line * n;
      const int pos = (i & 1) ? n - 1 - (i >> 1) : (i >> 1);
      double v = ldr(B, zb, pos, line);
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

__device__ __forceinline__ Bufs smem_bufs(double* sm, int m, int L) {
  Bufs B;
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
// Forward input: the interior of a halo-layout field, or (FUSED) the
// fillps right-hand side rho0*div(u)/dt computed on the fly
// (src/fillps.f90:39-50) plus the updt_rhs_b planes.
// ---------------------------------------------------------------------------
template <bool FUSED>
__global__ void __launch_bounds__(256) k_fft_x_fwd(Geo g, LinePlan pl, const DevScalars* __restrict__ sc,
    const double* __restrict__ src, const double* __restrict__ u, const double* __restrict__ v,
    const double* __restrict__ w, Phys ph, double* __restrict__ work, int L) {
  if (HALTED(sc)) return;
  extern __shared__ double sm[];
  const int n = pl.n, m = pl.m;
  const Bufs B = smem_bufs(sm, m < 1 ? 1 : m, L);
  const int nlines = g.ny * g.nz;
  const int l0 = blockIdx.x * L;
  const double dti = FUSED ? sc->dti : 0.;
  const double dtidxi = dti * g.dxi, dtidyi = dti * g.dyi;
  for (int it = threadIdx.x; it < L * n; it += blockDim.x) {
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
    double xv = x;
    if (pl.kind == 2 && (i & 1)) xv = -xv;  // sine kind: negate odd samples
    str(B, 0, fwd_pos(pl.kind, n, i), line, xv);
  }
  __syncthreads();
  line_forward<false>(pl, B, L, [&](int line, int s, double val) {
    const int gl = l0 + line;
    if (gl < nlines) work[(size_t)gl * n + s] = val;
  });
}

__global__ void __launch_bounds__(256) k_fft_x_bwd(Geo g, LinePlan pl, const DevScalars* __restrict__ sc,
    const double* __restrict__ work, double normfft, double* __restrict__ dst, int L) {
  if (HALTED(sc)) return;
  extern __shared__ double sm[];
  const int n = pl.n, m = pl.m;
  const Bufs B = smem_bufs(sm, m < 1 ? 1 : m, L);
  const int nlines = g.ny * g.nz;
  const int l0 = blockIdx.x * L;
  for (int it = threadIdx.x; it < L * n; it += blockDim.x) {
    const int line = it / n, s = it - line * n;
    const int gl = l0 + line;
    str(B, 1, s, line, gl < nlines ? __ldg(work + (size_t)gl * n + s) : 0.);
  }
  __syncthreads();
  line_backward<false>(pl, B, L, [&](int line, int i, double val) {
    const int gl = l0 + line;
    if (gl < nlines) {
      const int j = gl % g.ny + 1, k = gl / g.ny + 1;
      dst[g.h(i + 1, j, k)] = val * normfft;
    }
  });
}

// ---------------------------------------------------------------------------
// y transforms, in place on the spectral buffer.  Lines = TL consecutive x
// positions of one z plane; the tile is read and written row by row.
// ---------------------------------------------------------------------------
template <int DIR>
__global__ void __launch_bounds__(256) k_fft_y(Geo g, LinePlan pl, const DevScalars* __restrict__ sc,
                                               double* __restrict__ work, int L) {
  if (HALTED(sc)) return;
  extern __shared__ double sm[];
  const int n = pl.n, m = pl.m, nx = g.nx;
  const Bufs B = smem_bufs(sm, m < 1 ? 1 : m, L);
  const int i0 = blockIdx.x * L, k = blockIdx.y;
  double* plane = work + (size_t)k * nx * n;
  const int buf = DIR > 0 ? 0 : 1;
  for (int it = threadIdx.x; it < L * n; it += blockDim.x) {
    const int line = it % L, j = it / L;
    const int i = i0 + line;
    double x = i < nx ? plane[(size_t)j * nx + i] : 0.;
    if (DIR > 0) {
      if (pl.kind == 2 && (j & 1)) x = -x;
      str(B, 0, fwd_pos(pl.kind, n, j), line, x);
    } else {
      str(B, 1, j, line, x);
    }
  }
  __syncthreads();
  (void)buf;
  auto out = [&](int line, int j, double val) {
    const int i = i0 + line;
    if (i < nx) plane[(size_t)j * nx + i] = val;
  };
  if (DIR > 0) line_forward<true>(pl, B, L, out);
  else line_backward<true>(pl, B, L, out);
}

// ---------------------------------------------------------------------------
// z: batched Thomas (dgtsv_homebrewed with the eps pivot shift, src/solver.f90:
// 151-177 / src/solver_gpu.f90:179-203).  One column per thread; the forward
// sweep writes p' in place and keeps d only at chunk ends (shared memory);
// the backward sweep recomputes d per chunk from those checkpoints with the
// same operations, so it equals the stored one bit for bit.  The pivots use
// round-to-nearest intrinsics (no FMA contraction), as the reference's CPU
// build evaluates them.
// ---------------------------------------------------------------------------
#define ZCH 16

__device__ __forceinline__ double piv_inv(double bl, double lam, double al, double dprev) {
  // 1./(b(l)+lambda - a(l)*d(l-1) + eps)
  return __ddiv_rn(1.0, __dadd_rn(__dsub_rn(__dadd_rn(bl, lam), __dmul_rn(al, dprev)), CANSFZ_EPS));
}

__device__ void thomas_column(int n, const double* __restrict__ a, const double* __restrict__ b,
                              const double* __restrict__ c, double lam, double* __restrict__ col,
                              size_t st, double* __restrict__ dchk, int tpitch) {
  // forward elimination
  double dprev = 0., pprev = 0.;
  const int nch = (n + ZCH - 1) / ZCH;
  for (int ch = 0; ch < nch; ++ch) {
    const int k0 = ch * ZCH;
    double pv[ZCH];
#pragma unroll
    for (int q = 0; q < ZCH; ++q) pv[q] = (k0 + q < n) ? col[(size_t)(k0 + q) * st] : 0.;
#pragma unroll
    for (int q = 0; q < ZCH; ++q) {
      const int l = k0 + q;
      if (l < n) {
        double z;
        if (l == 0) z = __ddiv_rn(1.0, __dadd_rn(__dadd_rn(b[0], lam), CANSFZ_EPS));
        else z = piv_inv(b[l], lam, a[l], dprev);
        const double d = __dmul_rn(c[l], z);
        const double pn = (l == 0) ? __dmul_rn(pv[q], z) : __dmul_rn(__dsub_rn(pv[q], __dmul_rn(a[l], pprev)), z);
        dprev = d;
        pprev = pn;
        pv[q] = pn;
      }
    }
#pragma unroll
    for (int q = 0; q < ZCH; ++q)
      if (k0 + q < n) col[(size_t)(k0 + q) * st] = pv[q];
    dchk[ch * tpitch] = dprev;  // d at the last element of chunk ch
  }
  // backward substitution, chunk by chunk from the top
  double pnext = 0.;
  for (int ch = nch - 1; ch >= 0; --ch) {
    const int k0 = ch * ZCH;
    double dd[ZCH], pv[ZCH];
    double dp = ch > 0 ? dchk[(ch - 1) * tpitch] : 0.;
#pragma unroll
    for (int q = 0; q < ZCH; ++q) {
      const int l = k0 + q;
      double d = 0.;
      if (l < n) {
        double z;
        if (l == 0) z = __ddiv_rn(1.0, __dadd_rn(__dadd_rn(b[0], lam), CANSFZ_EPS));
        else z = piv_inv(b[l], lam, a[l], dp);
        d = __dmul_rn(c[l], z);
      }
      dd[q] = d;
      dp = d;
    }
#pragma unroll
    for (int q = 0; q < ZCH; ++q) pv[q] = (k0 + q < n) ? col[(size_t)(k0 + q) * st] : 0.;
#pragma unroll
    for (int q = ZCH - 1; q >= 0; --q) {
      const int l = k0 + q;
      if (l < n) {
        if (l < n - 1) pv[q] = __dsub_rn(pv[q], __dmul_rn(dd[q], pnext));
        pnext = pv[q];
      }
    }
#pragma unroll
    for (int q = 0; q < ZCH; ++q)
      if (k0 + q < n) col[(size_t)(k0 + q) * st] = pv[q];
  }
}

__global__ void __launch_bounds__(128) k_zsolve(int ncol, int nz, const double* __restrict__ lam,
    const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
    const DevScalars* __restrict__ sc, double* __restrict__ work) {
  if (HALTED(sc)) return;
  extern __shared__ double dchk[];  // [nch][blockDim]
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  thomas_column(nz, a, b, c, __ldg(lam + col), work + col, (size_t)ncol, dchk + threadIdx.x, blockDim.x);
}

// periodic z: gaussel_periodic (src/solver.f90:107-149)
__global__ void __launch_bounds__(128) k_zsolve_periodic(int ncol, int nz, const double* __restrict__ lam,
    const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ c,
    const DevScalars* __restrict__ sc, double* __restrict__ work, double* __restrict__ work2) {
  if (HALTED(sc)) return;
  extern __shared__ double dchk[];
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  const int n = nz;
  const double lm = __ldg(lam + col);
  double* p = work + col;
  double* p2 = work2 + col;
  const size_t st = (size_t)ncol;
  // p1 = solution of the (n-1) system with the RHS, in place
  thomas_column(n - 1, a, b, c, lm, p, st, dchk + threadIdx.x, blockDim.x);
  // p2 = solution with the spike RHS
  for (int k = 0; k < n - 1; ++k) p2[(size_t)k * st] = 0.;
  p2[0] = -a[0];
  p2[(size_t)(n - 2) * st] = -c[n - 2];
  thomas_column(n - 1, a, b, c, lm, p2, st, dchk + threadIdx.x, blockDim.x);
  const double bbn = b[n - 1] + lm;
  const double pn = (p[(size_t)(n - 1) * st] - c[n - 1] * p[0] - a[n - 1] * p[(size_t)(n - 2) * st]) /
                    (bbn + c[n - 1] * p2[0] + a[n - 1] * p2[(size_t)(n - 2) * st] + CANSFZ_EPS);
  p[(size_t)(n - 1) * st] = pn;
  for (int k = 0; k < n - 1; ++k) p[(size_t)k * st] = p[(size_t)k * st] + p2[(size_t)k * st] * pn;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
// opt the transform kernels into > 48 KB of dynamic shared memory (once)
void poisson_set_attributes() {
  const int lim = 100 * 1024;
  cudaFuncSetAttribute(k_fft_x_fwd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_x_fwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_x_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_y<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  cudaFuncSetAttribute(k_fft_y<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
}

static int lines_per_cta(int m, int maxL) {
  // keep 4*m*LP doubles within ~96 KB
  int L = maxL;
  while (L > 1 && 4 * (size_t)m * (L | 1) * 8 > 96 * 1024) L >>= 1;
  return L;
}

static void x_forward(const Launch& Lc, const Geo& g, const PoissonPlan& pl, const DevScalars* sc,
                      const double* src, const double* u, const double* v, const double* w, const Phys* ph,
                      bool fused) {
  const int m = pl.px.m < 1 ? 1 : pl.px.m;
  const int L = lines_per_cta(m, pl.px.n >= 128 ? 8 : 32);
  const size_t smem = 4 * (size_t)m * (L | 1) * sizeof(double);
  const int nlines = g.ny * g.nz;
  const dim3 grid((nlines + L - 1) / L);
  Phys pz{};
  if (fused)
    k_fft_x_fwd<true><<<grid, 256, smem, Lc.st>>>(g, pl.px, sc, nullptr, u, v, w, *ph, pl.work, L);
  else
    k_fft_x_fwd<false><<<grid, 256, smem, Lc.st>>>(g, pl.px, sc, src, nullptr, nullptr, nullptr, pz, pl.work, L);
}

static void y_pass(const Launch& Lc, const Geo& g, const PoissonPlan& pl, const DevScalars* sc, int dir) {
  const int m = pl.py.m < 1 ? 1 : pl.py.m;
  const int L = lines_per_cta(m, 16);
  const size_t smem = 4 * (size_t)m * (L | 1) * sizeof(double);
  const dim3 grid((g.nx + L - 1) / L, g.nz);
  if (dir > 0) k_fft_y<1><<<grid, 256, smem, Lc.st>>>(g, pl.py, sc, pl.work, L);
  else k_fft_y<-1><<<grid, 256, smem, Lc.st>>>(g, pl.py, sc, pl.work, L);
}

static void z_pass(const Launch& Lc, const Geo& g, const PoissonPlan& pl, const DevScalars* sc) {
  const int ncol = g.nx * g.ny;
  const int tb = 128;
  const int nch = (g.nz + ZCH - 1) / ZCH;
  const size_t smem = (size_t)nch * tb * sizeof(double);
  if (pl.zper)
    k_zsolve_periodic<<<(ncol + tb - 1) / tb, tb, smem, Lc.st>>>(ncol, g.nz, pl.lam, pl.a, pl.b, pl.c, sc, pl.work,
                                                                  pl.work2);
  else
    k_zsolve<<<(ncol + tb - 1) / tb, tb, smem, Lc.st>>>(ncol, g.nz, pl.lam, pl.a, pl.b, pl.c, sc, pl.work);
}

static void x_backward(const Launch& Lc, const Geo& g, const PoissonPlan& pl, const DevScalars* sc, double* dst) {
  const int m = pl.px.m < 1 ? 1 : pl.px.m;
  const int L = lines_per_cta(m, pl.px.n >= 128 ? 8 : 32);
  const size_t smem = 4 * (size_t)m * (L | 1) * sizeof(double);
  const int nlines = g.ny * g.nz;
  k_fft_x_bwd<<<(nlines + L - 1) / L, 256, smem, Lc.st>>>(g, pl.px, sc, pl.work, pl.normfft, dst, L);
}

// solver_gpu on the interior of the halo-layout field p (in place)
void launch_poisson(const Launch& L, const Geo& g, const PoissonPlan& pl, const DevScalars* sc, double* p,
                    const StageMark* mk) {
  x_forward(L, g, pl, sc, p, nullptr, nullptr, nullptr, nullptr, false);
  if (mk) mk->mark("poisson_x_fwd");
  y_pass(L, g, pl, sc, +1);
  if (mk) mk->mark("poisson_y_fwd");
  z_pass(L, g, pl, sc);
  if (mk) mk->mark("poisson_z_solve");
  y_pass(L, g, pl, sc, -1);
  if (mk) mk->mark("poisson_y_bwd");
  x_backward(L, g, pl, sc, p);
  if (mk) mk->mark("poisson_x_bwd");
}

// fillps + solver_gpu: the RHS is formed inside the x transform from u, v, w;
// phi (the interior of a halo-layout field) receives the solution.
void launch_poisson_fused_rhs(const Launch& L, const Geo& g, const PoissonPlan& pl, const Phys& ph,
                              const DevScalars* sc, const double* u, const double* v, const double* w,
                              const double* rhsb_planes, double* phi, const StageMark* mk) {
  (void)rhsb_planes;
  x_forward(L, g, pl, sc, nullptr, u, v, w, &ph, true);
  if (mk) mk->mark("poisson_x_fwd_fillps");
  y_pass(L, g, pl, sc, +1);
  if (mk) mk->mark("poisson_y_fwd");
  z_pass(L, g, pl, sc);
  if (mk) mk->mark("poisson_z_solve");
  y_pass(L, g, pl, sc, -1);
  if (mk) mk->mark("poisson_y_bwd");
  x_backward(L, g, pl, sc, phi);
  if (mk) mk->mark("poisson_x_bwd");
}

}  // namespace cansfz
