// libcansfz context: set-up of program cans (src/main.f90:147-412) for one
// GPU and a 1x1 pencil, the per-step sequence (src/main.f90:414-562) as two
// CUDA graphs (the double-buffer parities), and the C ABI of
// include/cansfz.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "batch.cuh"
#include "cansfz_internal.cuh"

using namespace cansfz;


#define CK(x)                                                                  \
  do {                                                                         \
    cudaError_t e_ = (x);                                                      \
    if (e_ != cudaSuccess) {                                                   \
      std::fprintf(stderr, "cansfz: %s failed: %s\n", #x, cudaGetErrorString(e_)); \
      return CANSFZ_ERR_CUDA;                                                  \
    }                                                                          \
  } while (0)

namespace {

const double PI_D = 3.14159265358979323846;

// initgrid, src/initgrid.f90:14-78 (z0 is a default-kind real quotient)
void host_initgrid(int gtype, int n, double gr, double lz, double* dzc, double* dzf, double* zc, double* zf) {
  zf[0] = 0.;
  for (int k = 1; k <= n; ++k) {
    const float z0f = ((float)k - 0.f) / (1.f * (float)n);
    const double z0 = (double)z0f, alpha = gr;
    double z;
    if (alpha == 0.) z = z0;
    else if (gtype == 2) z = 1.0 * (1. + std::tanh((z0 - 1.0) * alpha) / std::tanh(alpha / 1.));
    else if (gtype == 3) z = 1. - 1.0 * (1. + std::tanh((1. - z0 - 1.0) * alpha) / std::tanh(alpha / 1.));
    else if (gtype == 4) {
      if (z0 <= 0.5) z = 0.5 * (1. - 1. + std::tanh(2. * alpha * (z0 - 0.)) / std::tanh(alpha));
      else z = 0.5 * (1. + 1. + std::tanh(2. * alpha * (z0 - 1.)) / std::tanh(alpha));
    } else z = 0.5 * (1. + std::tanh((z0 - 0.5) * alpha) / std::tanh(alpha / 2.));
    zf[k] = z * lz;
  }
  for (int k = 1; k <= n; ++k) dzf[k] = zf[k] - zf[k - 1];
  dzf[0] = dzf[1];
  dzf[n + 1] = dzf[n];
  for (int k = 0; k <= n; ++k) dzc[k] = .5 * (dzf[k] + dzf[k + 1]);
  dzc[n + 1] = dzc[n];
  zc[0] = -dzc[0] / 2.;
  zf[0] = 0.;
  for (int k = 1; k <= n + 1; ++k) {
    zc[k] = zc[k - 1] + dzc[k - 1];
    zf[k] = zf[k - 1] + dzf[k];
  }
}

bool is_pp(const char c[2]) { return c[0] == 'P' && c[1] == 'P'; }
std::string bc2(const char c[2]) { return std::string{c[0], c[1]}; }

}  // namespace

// ---------------------------------------------------------------------------
// the context
// ---------------------------------------------------------------------------
struct cansfz_ctx {
  cansfz_params P{};
  cudaStream_t st = nullptr;
  bool own_stream = false;
  Launch L{};
  Geo g{};
  Phys ph{};
  int n[3]{};
  double dl[3]{}, dli[3]{};
  std::vector<double> dzc, dzf, zc, zf, dzci, dzfi, gvr_c, gvr_f;
  double* d_grid = nullptr;  // dzc,dzf,dzci,dzfi,gvr_c,gvr_f on the device
  int is_bound[3][2]{};
  int halo_periodic[3]{};
  // directions whose periodic ghost images the step's producing kernels write
  // themselves (store_wraps), so that the ghost fills after them skip those
  // copies: bit d when every field is periodic along d and n_d >= 2
  int wrap = 0;
  int images = 1;  // launch plan: 1 the producers write those images (cansfz_plan.ghost_images)
  char cbccur[3][2]{};
  double bccur[3][2]{};
  double seps = 0., beta = 1.;
  // fields (halo layout unless noted)
  double *u[2]{}, *v[2]{}, *w[2]{}, *psi[2]{}, *p[2]{};
  double *phip = nullptr, *phi = nullptr, *kappa = nullptr, *nx = nullptr, *ny = nullptr, *nz = nullptr;
  double *fx = nullptr, *fy = nullptr, *fz = nullptr;
  double *hpsi = nullptr, *hu = nullptr, *hv = nullptr, *hw = nullptr;       // AB2 histories (interior)
  double *tu = nullptr, *tv = nullptr, *tw_ = nullptr, *tpsi = nullptr;     // per-procedure scratch (interior)
  // scalar (_SCALAR): s by parity like u,v,w,psi; the dsdtrko history (interior)
  double *s[2]{}, *hs = nullptr;
  // balanced capillary split: surf?_n = surf[cur][?], surf?_o = surf[cur^1][?] (interior)
  double* surf[2][3]{};
  int cur = 0;  // index of the current u,v,w,psi,s and of p (= pn); po = p[cur^1]
  // Poisson solver (initsolver)
  PoissonPlan pl{};
  double* d_solver = nullptr;  // lam, a, b, c, twiddles, rhsb
  std::vector<double> lam_h, a_h, b_h, c_h;
  double* rhsbx = nullptr; double* rhsby = nullptr; double* rhsbz = nullptr;
  bool rhsb_zero = true;
  double* d_work = nullptr;
  // mixed form: FP64 right-hand side and refinement residual (halo layout)
  double* rhs64 = nullptr;
  double* res64 = nullptr;
  bool mixed = false;
  int sweeps = 2;
  // mixed form: FP32 intermediates of the phase-field and momentum stages
  float *phif = nullptr, *kappaf = nullptr, *nxf = nullptr, *nyf = nullptr, *nzf = nullptr;
  float *fxf = nullptr, *fyf = nullptr, *fzf = nullptr;                     // halo layout
  float *hpsif = nullptr, *huf = nullptr, *hvf = nullptr, *hwf = nullptr;   // AB2 histories (interior)
  // reductions, scalars
  double* partial = nullptr;
  DevScalars* sc = nullptr;       // the step scalars (device)
  DevScalars* sc_call = nullptr;  // scalars of a per-procedure call (device)
  DevScalars* sc_host = nullptr;  // pinned mirror
  bool first_rk_call = true, first_rk2fl_call = true, first_rkscal_call = true;
  // the tensor-core transform matrices while a plan selects the FFTs
  const uint16_t* gsave[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
  // graphs
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  bool prepared = false;
  int last_status = CANSFZ_OK;
  std::vector<void*> allocs;
  char inivel[8] = "zer";
};

namespace {

template <typename T>
int dalloc(cansfz_ctx* c, T** p, size_t n) {
  void* q = nullptr;
  if (cudaMalloc(&q, n * sizeof(T) + 256) != cudaSuccess) return CANSFZ_ERR_NOMEM;
  if (cudaMemset(q, 0, n * sizeof(T) + 256) != cudaSuccess) return CANSFZ_ERR_CUDA;
  c->allocs.push_back(q);
  *p = (T*)q;
  return CANSFZ_OK;
}

// set_bc's factor/sgn for one face (src/bound.f90:138-152)
BcFace make_face(char ctype, int ib, bool centered, double rvalue, double dr) {
  BcFace f{};
  f.centered = centered ? 1 : 0;
  double factor = rvalue, sgn = 0.;
  if (ctype == 'D' && centered) { factor = 2. * factor; sgn = -1.; }
  if (ctype == 'N') {
    if (ib == 0) factor = -dr * factor;
    else factor = dr * factor;
    sgn = 1.;
  }
  f.factor = factor;
  f.sgn = sgn;
  f.type = ctype == 'P' ? BC_P : (ctype == 'D' ? BC_D : (ctype == 'N' ? BC_N : BC_NONE));
  return f;
}

// boundp for one scalar field, src/bound.f90:81-124
BcField bc_scalar(const cansfz_ctx* c, const char cbc[3][2], const double bc[3][2], double* p) {
  BcField F{};
  F.p = p;
  for (int d = 0; d < 3; ++d) F.halo_periodic[d] = c->halo_periodic[d];
  for (int d = 0; d < 3; ++d)
    for (int ib = 0; ib < 2; ++ib) {
      if (!c->is_bound[d][ib]) continue;
      double dr = d == 0 ? c->dl[0] : (d == 1 ? c->dl[1] : (ib == 0 ? c->dzc[0] : c->dzc[c->n[2]]));
      F.face[d][ib] = make_face(cbc[d][ib], ib, true, bc[d][ib], dr);
    }
  return F;
}

BcField bc_scalar(const cansfz_ctx* c, const char cbc[3][2], const double bc[3][2], float* p) {
  BcField F = bc_scalar(c, cbc, bc, (double*)nullptr);
  F.p = p;
  F.f32 = 1;
  return F;
}

// bounduvw, src/bound.f90:15-79: the three velocity components (or the three
// phase fluxes, which take the velocity's boundary rules)
template <typename E>
void bc_vel(const cansfz_ctx* c, bool is_correc, E* u, E* v, E* w, BcField out[3]) {
  const cansfz_params& P = c->P;
  E* fld[3] = {u, v, w};
  for (int ivel = 0; ivel < 3; ++ivel) {
    BcField& F = out[ivel];
    F = BcField{};
    F.p = fld[ivel];
    F.f32 = sizeof(E) == sizeof(float);
    for (int d = 0; d < 3; ++d) F.halo_periodic[d] = c->halo_periodic[d];
    for (int d = 0; d < 3; ++d) {
      const bool normal = (ivel == d);
      const bool imp = (!is_correc) || is_pp(P.cbcvel[d][d]);
      if (normal && !imp) continue;
      for (int ib = 0; ib < 2; ++ib) {
        if (!c->is_bound[d][ib]) continue;
        double dr;
        if (d == 0) dr = c->dl[0];
        else if (d == 1) dr = c->dl[1];
        else {
          const int kk = ib == 0 ? 0 : c->n[2];
          dr = normal ? c->dzf[kk] : c->dzc[kk];
        }
        F.face[d][ib] = make_face(P.cbcvel[ivel][d][ib], ib, !normal, P.bcvel[ivel][d][ib], dr);
      }
    }
  }
}

// which: 0 cbcpre, 1 cbcpsi, 2 cbccur, 3..5 cbcnor(:,:,1..3)
void scalar_bc_spec(const cansfz_ctx* c, int which, const char (**cbc)[2], const double (**bc)[2]) {
  const cansfz_params& P = c->P;
  *cbc = P.cbcpre; *bc = P.bcpre;
  if (which == 1) { *cbc = P.cbcpsi; *bc = P.bcpsi; }
  else if (which == 2) { *cbc = c->cbccur; *bc = c->bccur; }
  else if (which >= 3 && which <= 5) { *cbc = P.cbcnor[which - 3]; *bc = P.bcnor[which - 3]; }
  else if (which == 6) { *cbc = P.cbcsca; *bc = P.bcsca; }
}

// wrapped: the periodic images the producing kernel already wrote (BcField::wrapped)
void run_bc(cansfz_ctx* c, std::initializer_list<BcField> fields, const DevScalars* sc, int wrapped = 0) {
  BcGroup grp{};
  for (const BcField& f : fields) {
    if (grp.nf == BC_MAXF) { launch_bc_group(c->L, c->g, grp, sc); grp.nf = 0; }
    grp.f[grp.nf] = f;
    grp.f[grp.nf++].wrapped = wrapped;
  }
  launch_bc_group(c->L, c->g, grp, sc);
}

void run_bcp(cansfz_ctx* c, int which, double* p, const DevScalars* sc, int wrapped = 0) {
  const char(*cbc)[2];
  const double(*bc)[2];
  scalar_bc_spec(c, which, &cbc, &bc);
  run_bc(c, {bc_scalar(c, cbc, bc, p)}, sc, wrapped);
}

void run_bcuvw(cansfz_ctx* c, bool is_correc, double* u, double* v, double* w, const DevScalars* sc,
               int wrapped = 0) {
  BcField F[3];
  bc_vel(c, is_correc, u, v, w, F);
  run_bc(c, {F[0], F[1], F[2]}, sc, wrapped);
}

// ---------------------------------------------------------------------------
// initsolver + fftini (src/initsolver.f90:15-228, src/fft.f90:20-140) for the
// packed spectral layout of the transforms in k_poisson.cu
// ---------------------------------------------------------------------------
int line_kind(const char c[2]) {
  const std::string s = bc2(c);
  if (s == "PP") return 0;
  if (s == "NN") return 1;
  if (s == "DD") return 2;
  return -1;
}

// eigenvalues (src/initsolver.f90:81-139) in the order of the device layout
void eigen_device_order(int n, int kind, std::vector<double>& lam) {
  lam.assign(n, 0.);
  if (kind == 0) {
    // packed (r0, r_{n/2}, r1, i1, ...).  The reference's CPU order is the
    // half-complex one: index m <= n/2 is r_m, index n-k is i_k, with
    // lambda(l) = -2(1-cos(2(l-1)pi/n)); the same expression is evaluated
    // at the same l for each slot.
    auto lamhc = [&](int m) { return -2. * (1. - std::cos((double)(2 * m) * PI_D / (1. * n))); };
    const int h = n / 2;
    lam[0] = lamhc(0);
    if (n > 1) lam[1] = lamhc(h);
    for (int k = 1; k < h; ++k) {
      lam[2 * k] = lamhc(k);
      lam[2 * k + 1] = lamhc(n - k);
    }
  } else if (kind == 1) {
    for (int l = 1; l <= n; ++l) lam[l - 1] = -2. * (1. - std::cos((double)(l - 1) * PI_D / (1. * n)));
  } else {
    for (int l = 1; l <= n; ++l) lam[l - 1] = -2. * (1. - std::cos((double)l * PI_D / (1. * n)));
  }
}

bool factorize(int m, int radix[FFT_MAXSTAGES], int* nst) {
  int k = 0;
  while (m % 4 == 0 && m > 4) { radix[k++] = 4; m /= 4; }
  for (int r : {4, 2, 3, 5, 7}) while (m % r == 0) { radix[k++] = r; m /= r; }
  *nst = k;
  return m == 1 && k <= FFT_MAXSTAGES;
}

// z solves with fewer columns than this read precomputed elimination factors
bool zsolve_factored(const cansfz_ctx* c) { return (long long)c->g.nx * c->g.ny < 32768; }

// FP32 spectral buffers and z factors of the mixed-form solve (once)
// the split-BF16 matrices of the tensor-core transforms (once), for the
// line lengths and kinds they serve
int alloc_xform_gemm(cansfz_ctx* c) {
  const cansfz_params& P = c->P;
  if (P.fp32_transforms != 0 || c->pl.gx[0] || c->pl.gy[0]) return CANSFZ_OK;
  static bool attrs = false;
  if (!attrs) {
    if (xform_gemm_set_attributes()) return CANSFZ_ERR_CUDA;
    attrs = true;
  }
  const int kinds[2] = {line_kind(P.cbcpre[0]), line_kind(P.cbcpre[1])};
  const int ns[2] = {c->n[0], c->n[1]};
  for (int d = 0; d < 2; ++d) {
    if (!xform_gemm_length(ns[d])) continue;
    for (int dir = 0; dir < 2; ++dir) {
      const std::vector<uint16_t> m = xform_bmat(kinds[d], dir == 0 ? 1 : -1, ns[d]);
      uint16_t* dm = nullptr;
      int rc;
      if ((rc = dalloc(c, &dm, m.size()))) return rc;
      CK(cudaMemcpyAsync(dm, m.data(), m.size() * sizeof(uint16_t), cudaMemcpyHostToDevice, c->st));
      CK(cudaStreamSynchronize(c->st));
      (d == 0 ? c->pl.gx : c->pl.gy)[dir] = dm;
    }
  }
  return CANSFZ_OK;
}

int alloc_f32_solver(cansfz_ctx* c) {
  const size_t nint = (size_t)c->g.tsize();
  int rc;
  if ((rc = alloc_xform_gemm(c))) return rc;
  if (!c->pl.workf && (rc = dalloc(c, &c->pl.workf, nint))) return rc;
  if (c->pl.zper && !c->pl.work2f && (rc = dalloc(c, &c->pl.work2f, nint))) return rc;
  if (!c->pl.zpivf && zsolve_factored(c)) {
    if ((rc = dalloc(c, &c->pl.zpivf, nint)) || (rc = dalloc(c, &c->pl.zdff, nint))) return rc;
    launch_z_factors(c->L, c->g, c->pl, true, c->pl.zpivf, c->pl.zdff);
    CK(cudaGetLastError());
  }
  return CANSFZ_OK;
}

int setup_solver(cansfz_ctx* c) {
  const cansfz_params& P = c->P;
  const int nx = c->n[0], ny = c->n[1], nz = c->n[2];
  const int kx = line_kind(P.cbcpre[0]), ky = line_kind(P.cbcpre[1]);
  if (kx < 0 || ky < 0) return CANSFZ_ERR_UNSUPPORTED;  // ND/DN in x,y (also rejected by the reference GPU path)
  if ((nx & 1) || (ny & 1)) return CANSFZ_ERR_UNSUPPORTED;
  // eigenvalues
  std::vector<double> lx, ly;
  eigen_device_order(nx, kx, lx);
  eigen_device_order(ny, ky, ly);
  for (auto& x : lx) x = x * (c->dli[0] * c->dli[0]);
  for (auto& x : ly) x = x * (c->dli[1] * c->dli[1]);
  c->lam_h.resize((size_t)nx * ny);
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) c->lam_h[i + (size_t)nx * j] = lx[i] + ly[j];
  // tridmatrix, src/initsolver.f90:141-183 (c_or_f = 'c')
  c->a_h.resize(nz); c->b_h.resize(nz); c->c_h.resize(nz);
  for (int k = 1; k <= nz; ++k) {
    c->a_h[k - 1] = c->dzfi[k] * c->dzci[k - 1];
    c->c_h[k - 1] = c->dzfi[k] * c->dzci[k];
  }
  for (int k = 0; k < nz; ++k) c->b_h[k] = -(c->a_h[k] + c->c_h[k]);
  double factor[2];
  for (int ib = 0; ib < 2; ++ib) {
    const char t = P.cbcpre[2][ib];
    factor[ib] = t == 'P' ? 0. : (t == 'D' ? -1. : 1.);
  }
  c->b_h[0] = c->b_h[0] + factor[0] * c->a_h[0];
  c->b_h[nz - 1] = c->b_h[nz - 1] + factor[1] * c->c_h[nz - 1];
  // bc_rhs (src/initsolver.f90:185-228)
  std::vector<double> dzc_(nz + 2), dzf_(nz + 2);
  for (int k = 0; k <= nz + 1; ++k) { dzc_[k] = 1. / c->dzci[k]; dzf_[k] = 1. / c->dzfi[k]; }
  auto bcr = [&](const char cbc[2], const double bcv[2], const double dlc[2], const double dlf[2], size_t plane,
                 std::vector<double>& rhs) {
    double f[2];
    for (int ib = 0; ib < 2; ++ib) {
      if (cbc[ib] == 'P') f[ib] = 0.;
      else if (cbc[ib] == 'D') f[ib] = -2. * bcv[ib];
      else f[ib] = (ib == 0 ? 1. : -1.) * dlc[ib] * bcv[ib];
    }
    rhs.assign(plane * 2, 0.);
    for (int ib = 0; ib < 2; ++ib)
      for (size_t q = 0; q < plane; ++q) rhs[q + plane * ib] = f[ib] / dlc[ib] / dlf[ib];
  };
  std::vector<double> rx, ry, rz;
  {
    const double dlx[2] = {c->dl[0], c->dl[0]}, dly[2] = {c->dl[1], c->dl[1]};
    const double dlcz[2] = {dzc_[0], dzc_[nz]}, dlfz[2] = {dzf_[1], dzf_[nz]};
    bcr(P.cbcpre[0], P.bcpre[0], dlx, dlx, (size_t)ny * nz, rx);
    bcr(P.cbcpre[1], P.bcpre[1], dly, dly, (size_t)nx * nz, ry);
    bcr(P.cbcpre[2], P.bcpre[2], dlcz, dlfz, (size_t)nx * ny, rz);
  }
  c->rhsb_zero = true;
  for (auto* r : {&rx, &ry, &rz})
    for (double x : *r) if (x != 0.) c->rhsb_zero = false;
  // normfft (src/fft.f90:96,133,139): PP -> n, NN/DD -> 2n
  double normfft = 1.;
  normfft = normfft * (kx == 0 ? 1. : 2.) * (nx + 0.);
  normfft = normfft * (ky == 0 ? 1. : 2.) * (ny + 0.);
  // line plans
  LinePlan* lps[2] = {&c->pl.px, &c->pl.py};
  const int ns[2] = {nx, ny}, kinds[2] = {kx, ky};
  std::vector<double> host;  // everything device-side for the solver, packed
  size_t off_lam = 0, off_a, off_b, off_c, off_tw[2], off_tw2[2], off_twc[2], off_rx, off_ry, off_rz;
  host.insert(host.end(), c->lam_h.begin(), c->lam_h.end());
  off_a = host.size(); host.insert(host.end(), c->a_h.begin(), c->a_h.end());
  off_b = host.size(); host.insert(host.end(), c->b_h.begin(), c->b_h.end());
  off_c = host.size(); host.insert(host.end(), c->c_h.begin(), c->c_h.end());
  for (int d = 0; d < 2; ++d) {
    LinePlan& lp = *lps[d];
    lp.n = ns[d];
    lp.kind = kinds[d];
    lp.m = ns[d] / 2;
    if (!factorize(lp.m, lp.radix, &lp.nst)) return CANSFZ_ERR_UNSUPPORTED;
    const long double pi = 3.14159265358979323846264338327950288L;
    auto pad2 = [&]() { if (host.size() & 1) host.push_back(0.); };  // double2 alignment
    pad2();
    off_tw[d] = host.size();
    for (int q = 0; q < lp.m; ++q) {
      const long double a = -2.0L * pi * q / (long double)lp.m;
      host.push_back((double)cosl(a)); host.push_back((double)sinl(a));
    }
    off_tw2[d] = host.size();
    for (int k = 0; k <= lp.m; ++k) {
      const long double a = -2.0L * pi * k / (long double)lp.n;
      host.push_back((double)cosl(a)); host.push_back((double)sinl(a));
    }
    off_twc[d] = host.size();
    for (int k = 0; k <= lp.n; ++k) {
      const long double a = -pi * k / (2.0L * lp.n);
      host.push_back((double)cosl(a)); host.push_back((double)sinl(a));
    }
  }
  off_rx = host.size(); host.insert(host.end(), rx.begin(), rx.end());
  off_ry = host.size(); host.insert(host.end(), ry.begin(), ry.end());
  off_rz = host.size(); host.insert(host.end(), rz.begin(), rz.end());
  int rc = dalloc(c, &c->d_solver, host.size() + 2);
  if (rc) return rc;
  CK(cudaMemcpy(c->d_solver, host.data(), host.size() * sizeof(double), cudaMemcpyHostToDevice));
  double* D = c->d_solver;
  c->pl.lam = D + off_lam;
  c->pl.a = D + off_a;
  c->pl.b = D + off_b;
  c->pl.c = D + off_c;
  for (int d = 0; d < 2; ++d) {
    lps[d]->tw = (const double2*)(D + off_tw[d]);
    lps[d]->tw2 = (const double2*)(D + off_tw2[d]);
    lps[d]->twc = (const double2*)(D + off_twc[d]);
  }
  c->rhsbx = D + off_rx; c->rhsby = D + off_ry; c->rhsbz = D + off_rz;
  // FP32 copies of the twiddle tables (mixed form)
  {
    std::vector<float> hf(host.size());
    for (size_t q = 0; q < host.size(); ++q) hf[q] = (float)host[q];
    float* F = nullptr;
    rc = dalloc(c, &F, hf.size() + 4);
    if (rc) return rc;
    CK(cudaMemcpy(F, hf.data(), hf.size() * sizeof(float), cudaMemcpyHostToDevice));
    for (int d = 0; d < 2; ++d) {
      lps[d]->twf = (const float2*)(F + off_tw[d]);
      lps[d]->tw2f = (const float2*)(F + off_tw2[d]);
      lps[d]->twcf = (const float2*)(F + off_twc[d]);
    }
  }
  c->pl.zsing = (P.cbcpre[2][0] != 'D' && P.cbcpre[2][1] != 'D') ? 1 : 0;
  c->pl.normfft = 1. / normfft;
  c->pl.zper = is_pp(P.cbcpre[2]) ? 1 : 0;
  const size_t nint = (size_t)nx * ny * nz;
  rc = dalloc(c, &c->pl.work, nint);
  if (rc) return rc;
  if (c->pl.zper) {
    rc = dalloc(c, &c->pl.work2, nint);
    if (rc) return rc;
  }
  // the z systems' elimination factors, once per plan, where the solve has
  // few columns: there the pivot recurrence's latency bounds the solve,
  // while with many columns reading the factors costs more than evaluating
  // them
  if (zsolve_factored(c)) {
    if ((rc = dalloc(c, &c->pl.zpiv, nint)) || (rc = dalloc(c, &c->pl.zdf, nint))) return rc;
    launch_z_factors(c->L, c->g, c->pl, false, c->pl.zpiv, c->pl.zdf);
    CK(cudaGetLastError());
  }
  if (P.form == CANSFZ_FORM_MIXED && P.refine_sweeps >= 0) {
    if (!c->rhsb_zero) return CANSFZ_ERR_UNSUPPORTED;  // refinement assumes homogeneous pressure BCs
    if ((rc = alloc_f32_solver(c))) return rc;
  }
  CK(cudaStreamSynchronize(c->st));
  return CANSFZ_OK;
}

int upload_scalars(cansfz_ctx* c, DevScalars* dst, const DevScalars& h) {
  CK(cudaMemcpyAsync(dst, &h, sizeof(DevScalars), cudaMemcpyHostToDevice, c->st));
  return CANSFZ_OK;
}

// scalars for one per-procedure call: a copy of the step scalars with overrides
int call_scalars(cansfz_ctx* c, DevScalars& h) {
  h.halted = 0;
  h.status = 0;
  return upload_scalars(c, c->sc_call, h);
}

int sync_status(cansfz_ctx* c) {
  CK(cudaMemcpyAsync(c->sc_host, c->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CANSFZ_OK;
}

// ---------------------------------------------------------------------------
// prescribed velocity for is_solve_ns = F ('voy'/'vox'/'zer' of initflow,
// src/initflow.f90:242-275), evaluated at the step's time
// ---------------------------------------------------------------------------
__global__ void k_prescribed_vel(Geo g, const DevScalars* __restrict__ sc, int which, double lx, double ly,
                                 double lz, const double* __restrict__ zc, const double* __restrict__ zf,
                                 double* __restrict__ u, double* __restrict__ v, double* __restrict__ w,
                                 double* __restrict__ p) {
  if (sc->halted) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
  if (i > g.nx) return;
  const int j = blockIdx.y + 1, k = blockIdx.z + 1;
  const double pi = 3.14159265358979323846;
  const double time = sc->time;
  const double zcc = zc[k] / lz, zff = zf[k] / lz;
  const double yc = ((double)j - .5) * g.dy / ly, yf = ((double)j - .0) * g.dy / ly;
  const double xc = ((double)i - .5) * g.dx / lx, xf = ((double)i - .0) * g.dx / lx;
  const int c = g.h(i, j, k);
  const double ct = cos(pi * time / 4.);
  if (which == 1) {  // voy
    const double sx = sin(pi * xf), sz = sin(pi * zff);
    u[c] = sx * sx * sin(2 * pi * zcc) * ct;
    v[c] = 0.;
    w[c] = -(sz * sz) * sin(2 * pi * xc) * ct;
  } else if (which == 2) {  // vox
    const double sy = sin(pi * yf), sz = sin(pi * zff);
    u[c] = 0.;
    v[c] = sy * sy * sin(2 * pi * zcc) * ct;
    w[c] = -(sz * sz) * sin(2 * pi * yc) * ct;
  } else {
    u[c] = 0.; v[c] = 0.; w[c] = 0.;
  }
  p[c] = 0.;
}

// phi, Youngs normals and curvature and their ghost fills in FP32 (mixed
// form); wrap: the periodic images the Youngs tile writes itself
void normals_f32(cansfz_ctx* c, const double* psi, const DevScalars* sc, const StageMark* mk = nullptr,
                 int wrap = 0) {
  const cansfz_params& P = c->P;
  Launch Lw = c->L;
  Lw.wrap = wrap;
  launch_cmpt_phi_f32(c->L, c->g, sc, c->ph.acdi != 0, psi, c->phif, c->ph.sdf == 0);
  if (mk) mk->mark("cmpt_phi");
  launch_youngs_t<float>(Lw, c->g, sc, c->phif, c->nxf, c->nyf, c->nzf, c->kappaf);
  if (mk) mk->mark("youngs");
  run_bc(c, {bc_scalar(c, c->cbccur, c->bccur, c->kappaf), bc_scalar(c, P.cbcnor[0], P.bcnor[0], c->nxf),
             bc_scalar(c, P.cbcnor[1], P.bcnor[1], c->nyf), bc_scalar(c, P.cbcnor[2], P.bcnor[2], c->nzf)},
         sc, wrap);
  if (mk) mk->mark("bc_normals");
}

// ---------------------------------------------------------------------------
// one time step (src/main.f90:422-529) on the current parity `c->cur`
// ---------------------------------------------------------------------------
void enqueue_step(cansfz_ctx* c, const StageMark* mk = nullptr) {
#define MARK(nm) do { if (mk) mk->mark(nm); } while (0)
  const cansfz_params& P = c->P;
  const Launch& L = c->L;
  const Geo& g = c->g;
  const int a = c->cur, b = a ^ 1;
  DevScalars* sc = c->sc;
  // the producing kernels below also write the periodic ghost images
  // (c->wrap), and the ghost fills after them skip those copies
  const int wr = c->images ? c->wrap : 0;
  Launch Lw = L;
  Lw.wrap = wr;
  launch_step_begin(L, sc, P.icheck);
  MARK("step_begin");
  // phase field: rk_2fl + boundary fills + phi + normals/curvature
  if (P.is_track_interface && c->mixed) {
    const bool sdf = c->ph.sdf != 0;
    if (c->ph.acdi)
      launch_acdi_t<float>(Lw, g, sc, sdf, true, c->u[a], c->v[a], c->w[a], c->nxf, c->nyf, c->nzf, c->phif,
                           c->psi[a], c->psi[b], c->hpsif, c->fxf, c->fyf, c->fzf);
    else
      launch_thinc_step_t<float>(L, g, sc, sdf, c->u[a], c->v[a], c->w[a], c->nxf, c->nyf, c->nzf, c->phif,
                                 c->psi[a], c->psi[b], c->hpsif, c->fxf, c->fyf, c->fzf);
    MARK("phase_transport");
    BcField F[3];
    bc_vel(c, false, c->fxf, c->fyf, c->fzf, F);
    run_bc(c, {F[0], F[1], F[2], bc_scalar(c, P.cbcpsi, P.bcpsi, c->psi[b])}, sc, c->ph.acdi ? wr : 0);
    MARK("bc_phase");
    normals_f32(c, c->psi[b], sc, mk, wr);
  } else if (P.is_track_interface) {
    if (c->ph.acdi)
      launch_acdi_step(Lw, g, sc, c->ph.sdf != 0, c->u[a], c->v[a], c->w[a], c->nx, c->ny, c->nz, c->phi,
                       c->psi[a], c->psi[b], c->hpsi, c->fx, c->fy, c->fz);
    else
      launch_thinc_step(L, g, sc, c->ph.sdf != 0, c->u[a], c->v[a], c->w[a], c->nx, c->ny, c->nz, c->phi,
                        c->psi[a], c->psi[b], c->hpsi, c->fx, c->fy, c->fz);
    MARK("phase_transport");
    BcField F[3];
    bc_vel(c, false, c->fx, c->fy, c->fz, F);
    run_bc(c, {F[0], F[1], F[2], bc_scalar(c, P.cbcpsi, P.bcpsi, c->psi[b])}, sc, c->ph.acdi ? wr : 0);
    MARK("bc_phase");
    if (c->ph.sdf) launch_cmpt_phi(L, g, sc, c->ph.acdi != 0, c->psi[b], c->phi);
    MARK("cmpt_phi");
    launch_youngs(Lw, g, sc, c->ph.sdf ? c->phi : c->psi[b], c->nx, c->ny, c->nz, c->kappa);
    MARK("youngs");
    run_bc(c, {bc_scalar(c, c->cbccur, c->bccur, c->kappa), bc_scalar(c, P.cbcnor[0], P.bcnor[0], c->nx),
               bc_scalar(c, P.cbcnor[1], P.bcnor[1], c->ny), bc_scalar(c, P.cbcnor[2], P.bcnor[2], c->nz)},
           sc, wr);
    MARK("bc_normals");
  } else {
    launch_copy(L, (size_t)g.hsize(), c->psi[a], c->psi[b]);
    if (c->mixed) {
      for (float* f : {c->fxf, c->fyf, c->fzf}) launch_fill(L, (size_t)g.hsize(), 0.f, f);
    } else {
      launch_fill(L, (size_t)g.hsize(), 0., c->fx);
      launch_fill(L, (size_t)g.hsize(), 0., c->fy);
      launch_fill(L, (size_t)g.hsize(), 0., c->fz);
    }
  }
  if (P.scalar) {
    // rk_scal + boundp(cbcsca), src/main.f90:460-463: the old scalar, the
    // old velocity, the new and old phase and the phase fluxes
    if (c->mixed)
      launch_scal_step<float>(L, g, c->ph, sc, c->fxf, c->fyf, c->fzf, c->psi[b], c->psi[a], c->u[a], c->v[a],
                              c->w[a], c->s[a], c->hs, c->s[b]);
    else
      launch_scal_step<double>(L, g, c->ph, sc, c->fx, c->fy, c->fz, c->psi[b], c->psi[a], c->u[a], c->v[a],
                               c->w[a], c->s[a], c->hs, c->s[b]);
    MARK("scalar");
    run_bcp(c, 6, c->s[b], sc);
    MARK("bc_scalar");
  }
  if (!P.is_solve_ns) {
    const std::string iv(c->inivel);
    const int which = iv == "voy" ? 1 : (iv == "vox" ? 2 : 0);
    dim3 bb(g.nx >= 128 ? 128 : 64), gg((g.nx + bb.x - 1) / bb.x, g.ny, g.nz);
    k_prescribed_vel<<<gg, bb, 0, L.st>>>(g, sc, which, P.l[0], P.l[1], P.l[2], c->d_grid + 6 * (g.nz + 2),
                                          c->d_grid + 7 * (g.nz + 2), c->u[b], c->v[b], c->w[b], c->p[a]);
    run_bcuvw(c, false, c->u[b], c->v[b], c->w[b], sc);
    launch_copy(L, (size_t)g.hsize(), c->p[a], c->p[b]);
  } else {
    // bulk_mean_12_stag for periodic gravity directions (src/main.f90:470-477)
    for (int d = 0; d < 3; ++d)
      if (std::fabs(P.gacc[d]) > 0. && is_pp(P.cbcpre[d]))
        launch_bulk_mean(L, g, c->ph, sc, c->partial, d + 1, c->d_grid + (d == 2 ? 5 : 4) * (g.nz + 2), c->psi[b]);
    // rk: the whole momentum update in one pass (the buoyancy reads the new scalar)
    const double* sb = c->ph.boussinesq ? c->s[b] : nullptr;
    // balanced split: read surf[a] (n) and surf[b] (o), the new force into
    // surf[b], which the parity flip makes the next step's n
    SurfSplit split{};
    if (c->ph.balanced)
      for (int d = 0; d < 3; ++d) { split.n[d] = c->surf[a][d]; split.o[d] = c->surf[b][d]; split.out_n[d] = c->surf[b][d]; }
    const SurfSplit* sp = c->ph.balanced ? &split : nullptr;
    if (c->mixed)
      launch_momentum_t<float>(Lw, g, c->ph, sc, c->u[a], c->v[a], c->w[a], c->psi[b], c->psi[a], c->fxf, c->fyf,
                               c->fzf, c->p[a], c->p[b], c->kappaf, sb, sp, c->huf, c->hvf, c->hwf, c->u[b], c->v[b],
                               c->w[b]);
    else
      launch_momentum_fused(Lw, g, c->ph, sc, c->u[a], c->v[a], c->w[a], c->psi[b], c->psi[a], c->fx, c->fy,
                            c->fz, c->p[a], c->p[b], c->kappa, sb, sp, c->hu, c->hv, c->hw, c->u[b], c->v[b],
                            c->w[b]);
    MARK("momentum");
    run_bcuvw(c, false, c->u[b], c->v[b], c->w[b], sc, wr);
    MARK("bc_uvw");
    // fillps + updt_rhs_b + solver
    if (c->mixed && c->sweeps >= 0) {
      // FP32 spectral solve + FP64-residual refinement sweeps
      launch_fillps(L, g, c->ph, sc, c->u[b], c->v[b], c->w[b], c->rhs64);
      MARK("fillps");
      launch_poisson_f32(L, g, c->pl, sc, c->rhs64, c->phip, false, mk);
      for (int sw = 0; sw < c->sweeps; ++sw) {
        run_bcp(c, 0, c->phip, sc);
        launch_residual(L, g, sc, c->rhs64, c->phip, c->res64);
        MARK("residual");
        launch_poisson_f32(L, g, c->pl, sc, c->res64, c->phip, true, mk);
      }
    } else if (c->rhsb_zero) {
      launch_poisson_fused_rhs(Lw, g, c->pl, c->ph, sc, c->u[b], c->v[b], c->w[b], nullptr, c->phip, mk);
    } else {
      launch_fillps(L, g, c->ph, sc, c->u[b], c->v[b], c->w[b], c->phip);
      launch_updt_rhs_b(L, g, c->is_bound, c->rhsbx, c->rhsby, c->rhsbz, c->phip);
      launch_poisson(Lw, g, c->pl, sc, c->phip, mk);
    }
    // the FP64 solve's inverse x pass wrote the periodic images
    run_bcp(c, 0, c->phip, sc, (c->mixed && c->sweeps >= 0) ? 0 : wr);
    MARK("bc_pcorr");
    // correc, and updatep (p_new = phi + p into the po slot, then po <- p by
    // the parity flip), in one pass over phi
    launch_correc_updatep(Lw, g, c->ph, sc, c->phip, c->u[b], c->v[b], c->w[b], c->p[a], c->p[b]);
    MARK("correc_updatep");
    {
      // bounduvw after correc and boundp of the new pressure: independent
      // fields, one launch per fill stage for the four
      BcField F[3];
      bc_vel(c, true, c->u[b], c->v[b], c->w[b], F);
      const char(*cbc)[2];
      const double(*bcv)[2];
      scalar_bc_spec(c, 0, &cbc, &bcv);
      run_bc(c, {F[0], F[1], F[2], bc_scalar(c, cbc, bcv, c->p[b])}, sc, wr);
    }
    MARK("bc_uvw_p");
  }
  launch_step_end(L, c->ph, sc);
  // acdi_set_gamma, and on icheck steps chkdt + chkdiv, in one pass
  launch_step_reductions(L, g, c->ph, sc, c->partial, c->u[b], c->v[b], c->w[b]);
  MARK("gamma_chkdt_chkdiv");
#undef MARK
}

// One step of case c recorded instead of issued.  Launches that do not go
// through the recorder are caught by a throwaway stream capture: the record
// is complete (the step can be replayed batched) when that capture is empty.
int record_step(cansfz_ctx* c, Recorder* rec, bool* complete) {
  *complete = false;
  cudaGraph_t g = nullptr;
  CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
  c->L.rec = rec;
  c->L.batched = 1;
  enqueue_step(c);
  c->L.rec = nullptr;
  c->L.batched = 0;
  CK(cudaStreamEndCapture(c->st, &g));
  size_t nodes = 0;
  const cudaError_t e = cudaGraphGetNodes(g, nullptr, &nodes);
  cudaGraphDestroy(g);
  CK(e);
  *complete = nodes == 0 && !rec->e.empty();
  return CANSFZ_OK;
}

bool same_record(const Recorder& a, const Recorder& b) {
  if (a.e.size() != b.e.size()) return false;
  for (size_t q = 0; q < a.e.size(); ++q)
    if (!a.e[q].same_launch(b.e[q])) return false;
  return true;
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int cansfz_version(void) { return 100; }

const char* cansfz_status_string(int s) {
  switch (s) {
    case CANSFZ_OK: return "ok";
    case CANSFZ_ERR_ARG: return "invalid argument";
    case CANSFZ_ERR_CUDA: return "CUDA runtime error";
    case CANSFZ_ERR_TIMEOUT: return "bounded device wait ran out";
    case CANSFZ_ERR_NAN: return "ERROR: maximum divergence is too large (NaN)";
    case CANSFZ_ERR_DIVERGENCE: return "ERROR: maximum divergence is too large.";
    case CANSFZ_ERR_DT: return "ERROR: time step is too small / fixed time step exceeds the stability limit";
    case CANSFZ_ERR_UNSUPPORTED: return "boundary condition or option not supported on the GPU path";
    case CANSFZ_ERR_NOMEM: return "device allocation failed";
    case CANSFZ_ERR_NOT_FOUND: return "no CUDA device";
    default: return "unknown status";
  }
}

int cansfz_create(const cansfz_params* prm, void* stream, cansfz_ctx** out) {
  if (!prm || !out) return CANSFZ_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return CANSFZ_ERR_NOT_FOUND;
  const cansfz_params& P = *prm;
  for (int d = 0; d < 3; ++d)
    if (P.ng[d] < 2) return CANSFZ_ERR_ARG;
  if (P.ng[2] < 3) return CANSFZ_ERR_ARG;
  if ((double)(P.ng[0] + 2) * (P.ng[1] + 2) * (P.ng[2] + 2) > 2.0e9) return CANSFZ_ERR_ARG;
  cansfz_ctx* c = new cansfz_ctx();
  c->P = P;
  int rc = CANSFZ_OK;
  auto fail = [&](int r) { cansfz_destroy(c); return r; };
  if (stream) c->st = (cudaStream_t)stream;
  else {
    if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) return fail(CANSFZ_ERR_CUDA);
    c->own_stream = true;
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&c->L.nsm, cudaDevAttrMultiProcessorCount, dev);
  c->L.st = c->st;
  poisson_set_attributes();
  tiles_set_attributes();
  momentum_set_attributes();
  for (int d = 0; d < 3; ++d) c->n[d] = P.ng[d];
  const int nx = c->n[0], ny = c->n[1], nz = c->n[2];
  for (int d = 0; d < 3; ++d) {
    c->dl[d] = P.l[d] / (1. * P.ng[d]);
    c->dli[d] = 1. / c->dl[d];
  }
  // initgrid and the z metrics (src/main.f90:230-272)
  c->dzc.assign(nz + 2, 0.); c->dzf = c->dzc; c->zc = c->dzc; c->zf = c->dzc; c->dzci = c->dzc; c->dzfi = c->dzc;
  host_initgrid(P.gtype, nz, P.gr, P.l[2], c->dzc.data(), c->dzf.data(), c->zc.data(), c->zf.data());
  for (int k = 0; k <= nz + 1; ++k) { c->dzci[k] = 1. / c->dzc[k]; c->dzfi[k] = 1. / c->dzf[k]; }
  c->gvr_c.resize(nz + 2); c->gvr_f.resize(nz + 2);
  for (int k = 0; k <= nz + 1; ++k) {
    c->gvr_c[k] = c->dl[0] * c->dl[1] * c->dzc[k] / (P.l[0] * P.l[1] * P.l[2]);
    c->gvr_f[k] = c->dl[0] * c->dl[1] * c->dzf[k] / (P.l[0] * P.l[1] * P.l[2]);
  }
  {
    std::vector<double> gh;
    for (auto* v : {&c->dzc, &c->dzf, &c->dzci, &c->dzfi, &c->gvr_c, &c->gvr_f, &c->zc, &c->zf})
      gh.insert(gh.end(), v->begin(), v->end());
    if ((rc = dalloc(c, &c->d_grid, gh.size()))) return fail(rc);
    if (cudaMemcpy(c->d_grid, gh.data(), gh.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(CANSFZ_ERR_CUDA);
  }
  const int S = nz + 2;
  Geo& g = c->g;
  g.nx = nx; g.ny = ny; g.nz = nz;
  g.sx = nx + 2; g.sxy = (nx + 2) * (ny + 2);
  g.dxi = c->dli[0]; g.dyi = c->dli[1];
  g.dx = c->dl[0]; g.dy = c->dl[1];
  g.dzc = c->d_grid; g.dzf = c->d_grid + S; g.dzci = c->d_grid + 2 * S; g.dzfi = c->d_grid + 3 * S;
  // topology of the 1x1 pencil (src/initmpi.f90:148-183)
  for (int d = 0; d < 3; ++d) {
    const bool per = is_pp(P.cbcpre[d]);
    c->halo_periodic[d] = (d > 0 && per) ? 1 : 0;
    c->is_bound[d][0] = c->is_bound[d][1] = (d == 0) ? 1 : (per ? 0 : 1);
  }
  for (int d = 0; d < 3; ++d)
    for (int ib = 0; ib < 2; ++ib) { c->cbccur[d][ib] = P.cbcpsi[d][ib]; c->bccur[d][ib] = P.bcpre[d][ib]; }
  {
    bool xp = is_pp(P.cbcpre[0]) && is_pp(P.cbcpsi[0]) && (!P.scalar || is_pp(P.cbcsca[0]));
    for (int q = 0; q < 3; ++q) xp = xp && is_pp(P.cbcvel[q][0]) && is_pp(P.cbcnor[q][0]);
    c->wrap = (xp && nx >= 2 ? 1 : 0) | (c->halo_periodic[1] && ny >= 2 ? 2 : 0) |
              (c->halo_periodic[2] && nz >= 2 ? 4 : 0);
  }
  // physics constants (src/param.f90:170-178)
  Phys& ph = c->ph;
  for (int q = 0; q < 2; ++q) { ph.rho12[q] = P.rho12[q]; ph.mu12[q] = P.mu12[q]; }
  ph.rho0 = std::min(P.rho12[0], P.rho12[1]);
  ph.irho0 = 1. / ph.rho0;
  ph.sigma = P.sigma;
  ph.brackbill = P.brackbill ? 1 : 0;
  ph.surf_factor = ph.brackbill ? P.sigma * 2. / (P.rho12[0] + P.rho12[1]) : P.sigma;
  for (int d = 0; d < 3; ++d) { ph.bforce[d] = P.bforce[d]; ph.gacc[d] = P.gacc[d]; }
  ph.gam_factor = P.acdi_gam_factor;
  ph.gam_min = P.acdi_gam_min;
  ph.cfl = P.cfl; ph.dtmax = P.dtmax; ph.dt_f = P.dt_f;
  ph.small = CANSFZ_EPS * 1.0e7;
  ph.icheck = P.icheck;
  ph.acdi = P.interface_capturing == CANSFZ_ACDI ? 1 : 0;
  ph.sdf = P.sdf_normals ? 1 : 0;
  ph.solve_ns = P.is_solve_ns ? 1 : 0;
  ph.track = P.is_track_interface ? 1 : 0;
  ph.dlmin = std::min(c->dl[0], c->dl[1]);
  for (int k = 0; k <= nz + 1; ++k) ph.dlmin = std::min(ph.dlmin, 1. / c->dzfi[k]);
  ph.mu_over_rho_max = std::max(P.mu12[0] / P.rho12[0], P.mu12[1] / P.rho12[1]);
  ph.rho_min = std::min(P.rho12[0], P.rho12[1]);
  ph.gmax = std::max(std::fabs(P.gacc[0]), std::max(std::fabs(P.gacc[1]), std::fabs(P.gacc[2])));
  // scalar transport; the buoyancy term exists only with the scalar (src/mom.f90:1017)
  ph.scalar = P.scalar ? 1 : 0;
  ph.boussinesq = (P.scalar && P.boussinesq) ? 1 : 0;
  for (int q = 0; q < 2; ++q) { ph.ka12[q] = P.ka12[q]; ph.rhocp12[q] = P.rho12[q] * P.cp12[q]; }
  ph.ssource = P.ssource;
  ph.ka_rhocp_max = std::max(P.ka12[0] / (P.rho12[0] * P.cp12[0]), P.ka12[1] / (P.rho12[1] * P.cp12[1]));
  ph.rhobeta = P.rho12[1] * P.beta12[1];
  ph.drhobeta = P.rho12[0] * P.beta12[0] - P.rho12[1] * P.beta12[1];
  ph.balanced = P.balanced ? 1 : 0;
  // acdi_set_epsilon (src/acdi.f90:16-30) and the THINC beta (src/param.f90:178)
  double dlmax = std::max(c->dl[0], c->dl[1]);
  for (int k = 0; k <= nz + 1; ++k) dlmax = std::max(dlmax, 1. / c->dzfi[k]);
  c->seps = dlmax * P.psi_thickness_factor;
  c->beta = 1. / (2. * P.psi_thickness_factor);
  // device fields
  const size_t H = (size_t)g.hsize(), I = (size_t)g.tsize();
  for (int q = 0; q < 2; ++q)
    for (double** f : {&c->u[q], &c->v[q], &c->w[q], &c->psi[q], &c->p[q]})
      if ((rc = dalloc(c, f, H))) return fail(rc);
  for (double** f : {&c->phip, &c->phi, &c->kappa, &c->nx, &c->ny, &c->nz, &c->fx, &c->fy, &c->fz})
    if ((rc = dalloc(c, f, H))) return fail(rc);
  for (double** f : {&c->hpsi, &c->hu, &c->hv, &c->hw, &c->tu, &c->tv, &c->tw_, &c->tpsi})
    if ((rc = dalloc(c, f, I))) return fail(rc);
  if (P.balanced)  // zero, as src/main.f90:205-213 sets them
    for (int q = 0; q < 2; ++q)
      for (int d = 0; d < 3; ++d)
        if ((rc = dalloc(c, &c->surf[q][d], I))) return fail(rc);
  if (P.scalar) {
    for (int q = 0; q < 2; ++q)
      if ((rc = dalloc(c, &c->s[q], H))) return fail(rc);
    if ((rc = dalloc(c, &c->hs, I))) return fail(rc);
  }
  if ((rc = setup_solver(c))) return fail(rc);
  c->mixed = P.form == CANSFZ_FORM_MIXED;
  c->sweeps = P.refine_sweeps < 0 ? -1 : (P.refine_sweeps > 8 ? 8 : P.refine_sweeps);
  if (c->mixed) {
    if ((rc = dalloc(c, &c->rhs64, H))) return fail(rc);
    if ((rc = dalloc(c, &c->res64, H))) return fail(rc);
    for (float** f : {&c->phif, &c->kappaf, &c->nxf, &c->nyf, &c->nzf, &c->fxf, &c->fyf, &c->fzf})
      if ((rc = dalloc(c, f, H))) return fail(rc);
    for (float** f : {&c->hpsif, &c->huf, &c->hvf, &c->hwf})
      if ((rc = dalloc(c, f, I))) return fail(rc);
  }
  // reductions: partial sums of one launch over the interior blocks
  const int bx = nx >= 128 ? 128 : (nx >= 64 ? 64 : 32);
  const size_t nblk = (size_t)((nx + bx - 1) / bx) * ny * nz;
  // ... and four per block of the fused end-of-step reduction (4 blocks per SM)
  const size_t nred = 4 * (size_t)(c->L.nsm > 0 ? c->L.nsm : 148) * 8;
  if ((rc = dalloc(c, &c->partial, std::max(2 * nblk, nred) + 64))) return fail(rc);
  if ((rc = dalloc(c, &c->sc, 1))) return fail(rc);
  if ((rc = dalloc(c, &c->sc_call, 1))) return fail(rc);
  if (cudaMallocHost(&c->sc_host, sizeof(DevScalars)) != cudaSuccess) return fail(CANSFZ_ERR_NOMEM);
  std::memset(c->sc_host, 0, sizeof(DevScalars));
  DevScalars h{};
  h.seps = c->seps;
  h.beta = c->beta;
  h.first_rk = 1;
  h.first_rk2fl = 1;
  h.first_scal = 1;
  if ((rc = upload_scalars(c, c->sc, h))) return fail(rc);
  if (cudaStreamSynchronize(c->st) != cudaSuccess) return fail(CANSFZ_ERR_CUDA);
  *out = c;
  return CANSFZ_OK;
}

int cansfz_destroy(cansfz_ctx* c) {
  if (!c) return CANSFZ_OK;
  if (c->st) cudaStreamSynchronize(c->st);
  for (auto& ge : c->gexec)
    if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
  for (void* q : c->allocs) cudaFree(q);
  if (c->sc_host) cudaFreeHost(c->sc_host);
  if (c->own_stream && c->st) cudaStreamDestroy(c->st);
  delete c;
  return CANSFZ_OK;
}

void* cansfz_stream(cansfz_ctx* c) { return c ? (void*)c->st : nullptr; }

int cansfz_set_fields(cansfz_ctx* c, const double* u, const double* v, const double* w, const double* p,
                      const double* psi, int on_device) {
  if (!c) return CANSFZ_ERR_ARG;
  const size_t bytes = (size_t)c->g.hsize() * sizeof(double);
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  const int a = c->cur;
  const double* src[5] = {u, v, w, p, psi};
  double* dst[5] = {c->u[a], c->v[a], c->w[a], c->p[a], c->psi[a]};
  for (int q = 0; q < 5; ++q)
    if (src[q]) CK(cudaMemcpyAsync(dst[q], src[q], bytes, kind, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->prepared = false;
  return CANSFZ_OK;
}

int cansfz_get_fields(cansfz_ctx* c, double* u, double* v, double* w, double* p, double* psi, int on_device) {
  if (!c) return CANSFZ_ERR_ARG;
  const size_t bytes = (size_t)c->g.hsize() * sizeof(double);
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
  const int a = c->cur;
  double* dst[5] = {u, v, w, p, psi};
  const double* src[5] = {c->u[a], c->v[a], c->w[a], c->p[a], c->psi[a]};
  for (int q = 0; q < 5; ++q)
    if (dst[q]) CK(cudaMemcpyAsync(dst[q], src[q], bytes, kind, c->st));
  CK(cudaStreamSynchronize(c->st));
  return CANSFZ_OK;
}

int cansfz_set_scalar(cansfz_ctx* c, const double* s, int on_device) {
  if (!c || !s) return CANSFZ_ERR_ARG;
  if (!c->P.scalar) return CANSFZ_ERR_UNSUPPORTED;
  const size_t bytes = (size_t)c->g.hsize() * sizeof(double);
  CK(cudaMemcpyAsync(c->s[c->cur], s, bytes, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  c->prepared = false;
  return CANSFZ_OK;
}

int cansfz_get_aux(cansfz_ctx* c, const char* name, double* out, int on_device) {
  if (!c || !name || !out) return CANSFZ_ERR_ARG;
  const std::string s(name);
  const int a = c->cur;
  const double* src = nullptr;
  size_t n = (size_t)c->g.hsize();
  if (s == "phi") src = c->phi;
  else if (s == "kappa") src = c->kappa;
  else if (s == "normx") src = c->nx;
  else if (s == "normy") src = c->ny;
  else if (s == "normz") src = c->nz;
  else if (s == "psiflx_x") src = c->fx;
  else if (s == "psiflx_y") src = c->fy;
  else if (s == "psiflx_z") src = c->fz;
  else if (s == "psio") src = c->psi[a ^ 1];
  else if (s == "pn") src = c->p[a];
  else if (s == "po") src = c->p[a ^ 1];
  else if (s == "pcorr") src = c->phip;
  else if (s == "dpsidtrko") { src = c->hpsi; n = c->g.tsize(); }
  else if (s == "dudtrko") { src = c->hu; n = c->g.tsize(); }
  else if (s == "dvdtrko") { src = c->hv; n = c->g.tsize(); }
  else if (s == "dwdtrko") { src = c->hw; n = c->g.tsize(); }
  else if (s == "s" && c->P.scalar) src = c->s[a];
  else if (c->P.balanced && s.size() == 7 && s.compare(0, 4, "surf") == 0 && s[5] == '_' &&
           (s[4] == 'x' || s[4] == 'y' || s[4] == 'z') && (s[6] == 'n' || s[6] == 'o')) {
    src = c->surf[s[6] == 'n' ? a : a ^ 1][s[4] - 'x'];
    n = c->g.tsize();
  }
  else if (s == "dsdtrko" && c->P.scalar) { src = c->hs; n = c->g.tsize(); }
  else return CANSFZ_ERR_ARG;
  if (c->mixed) {  // FP32 intermediates, widened into scratch for the caller
    const float* f = nullptr;
    double* tmp = c->res64;
    if (s == "phi") f = c->phif;
    else if (s == "kappa") f = c->kappaf;
    else if (s == "normx") f = c->nxf;
    else if (s == "normy") f = c->nyf;
    else if (s == "normz") f = c->nzf;
    else if (s == "psiflx_x") f = c->fxf;
    else if (s == "psiflx_y") f = c->fyf;
    else if (s == "psiflx_z") f = c->fzf;
    else if (s == "dpsidtrko") f = c->hpsif;
    else if (s == "dudtrko") f = c->huf;
    else if (s == "dvdtrko") f = c->hvf;
    else if (s == "dwdtrko") f = c->hwf;
    if (f) {
      launch_widen(c->L, n, f, tmp);
      src = tmp;
    }
  }
  CK(cudaMemcpyAsync(out, src, n * sizeof(double), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                     c->st));
  CK(cudaStreamSynchronize(c->st));
  return CANSFZ_OK;
}

int cansfz_prepare(cansfz_ctx* c) {
  if (!c) return CANSFZ_ERR_ARG;
  const cansfz_params& P = c->P;
  const int a = c->cur;
  DevScalars* sc = c->sc;
  const Launch& L = c->L;
  // src/main.f90:337-412
  run_bcuvw(c, false, c->u[a], c->v[a], c->w[a], sc);
  run_bcp(c, 0, c->p[a], sc);
  launch_copy(L, (size_t)c->g.hsize(), c->p[a], c->p[a ^ 1]);  // po = pn = p
  if (P.scalar) run_bcp(c, 6, c->s[a], sc);
  run_bcp(c, 1, c->psi[a], sc);
  if (c->mixed) {
    normals_f32(c, c->psi[a], sc);
  } else {
    if (c->ph.sdf) launch_cmpt_phi(L, c->g, sc, c->ph.acdi != 0, c->psi[a], c->phi);
    launch_youngs(L, c->g, sc, c->ph.sdf ? c->phi : c->psi[a], c->nx, c->ny, c->nz, c->kappa);
    run_bc(c, {bc_scalar(c, c->cbccur, c->bccur, c->kappa), bc_scalar(c, P.cbcnor[0], P.bcnor[0], c->nx),
               bc_scalar(c, P.cbcnor[1], P.bcnor[1], c->ny), bc_scalar(c, P.cbcnor[2], P.bcnor[2], c->nz)},
           sc);
  }
  if (c->ph.acdi) launch_gamma(L, c->g, c->ph, sc, c->partial, c->u[a], c->v[a], c->w[a], true);
  launch_chkdt(L, c->g, c->ph, sc, c->partial, c->u[a], c->v[a], c->w[a], false);
  // dto = dt (src/main.f90:409)
  if (int rc = sync_status(c)) return rc;
  c->sc_host->dto = c->sc_host->dt;
  if (int rc = upload_scalars(c, sc, *c->sc_host)) return rc;
  CK(cudaStreamSynchronize(c->st));
  c->prepared = true;
  return CANSFZ_OK;
}

// ---------------------------------------------------------------------------
// Batched ensemble: independent cases (any sizes, any parameters) advance
// together.  One CUDA graph per step parity holds every case's whole step as
// a parallel branch (fork/join capture over the cases' own streams), so one
// graph launch advances all cases by a step and the GPU overlaps the small
// cases' kernels instead of running them one case at a time.
// ---------------------------------------------------------------------------
struct cansfz_ensemble {
  std::vector<cansfz_ctx*> cases;
  cudaStream_t st = nullptr;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  int cur = 0;
  int ngroups = 0, grouped = 0;  // case groups of the last graph built, cases in groups of two or more
  void* argtab[2] = {nullptr, nullptr};  // the groups' argument tables of each parity's graph
  int batch = 1;  // cases per batched launch chain (1: every case its own branch)
};

int cansfz_ensemble_create(cansfz_ctx* const* cases, int ncases, void* stream, cansfz_ensemble** out) {
  if (!cases || ncases <= 0 || !out) return CANSFZ_ERR_ARG;
  *out = nullptr;
  for (int q = 0; q < ncases; ++q) {
    if (!cases[q]) return CANSFZ_ERR_ARG;
    if (!cases[q]->prepared) {
      if (int rc = cansfz_prepare(cases[q])) return rc;
    }
    if (cases[q]->cur != cases[0]->cur) return CANSFZ_ERR_ARG;  // all cases at the same buffer parity
  }
  auto* e = new cansfz_ensemble();
  e->cases.assign(cases, cases + ncases);
  e->cur = cases[0]->cur;
  bool ok = true;
  if (stream) e->st = (cudaStream_t)stream;
  else ok = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess;
  e->join.resize(ncases, nullptr);
  for (int q = 0; ok && q < ncases; ++q)
    ok = cudaEventCreateWithFlags(&e->join[q], cudaEventDisableTiming) == cudaSuccess;

  if (!ok) {
    cansfz_ensemble_destroy(e);
    return CANSFZ_ERR_CUDA;
  }
  *out = e;
  return CANSFZ_OK;
}

int cansfz_ensemble_destroy(cansfz_ensemble* e) {
  if (!e) return CANSFZ_ERR_ARG;
  for (int q = 0; q < 2; ++q) {
    if (e->gexec[q]) cudaGraphExecDestroy(e->gexec[q]);
    if (e->argtab[q]) cudaFree(e->argtab[q]);
  }
  for (cudaEvent_t ev : e->join)
    if (ev) cudaEventDestroy(ev);

  if (e->fork) cudaEventDestroy(e->fork);
  // the stream is the caller's when one was given; a created one is released
  bool own = true;
  for (cansfz_ctx* c : e->cases)
    if (c && c->st == e->st) own = false;
  if (own && e->st) cudaStreamDestroy(e->st);
  delete e;
  return CANSFZ_OK;
}

// status_out (optional, ncases entries): each case's status after the steps
int cansfz_ensemble_step(cansfz_ensemble* e, int nsteps, int* status_out) {
  if (!e || nsteps < 0) return CANSFZ_ERR_ARG;
  const int n = (int)e->cases.size();
  std::vector<long long> istep0(n);
  for (int q = 0; q < n; ++q) {
    cansfz_ctx* c = e->cases[q];
    if (c->last_status != CANSFZ_OK) return c->last_status;  // an aborted case stops the ensemble
    if (c->cur != e->cur) return CANSFZ_ERR_ARG;  // a case was stepped on its own in between
    if (int rc = sync_status(c)) return rc;
    istep0[q] = c->sc_host->istep;
  }
  for (int s = 0; s < nsteps; ++s) {
    const int par = e->cur;
    if (!e->gexec[par]) {
      // record every case's step; cases whose records agree launch for
      // launch (same kernels, grids and shared memory: same sizes and
      // options) form a group that is replayed as batched launches
      std::vector<Recorder> rec(n);
      std::vector<std::vector<int>> groups;
      // branches in order of decreasing size, so that the longest steps
      // start first
      std::vector<int> order(n);
      for (int q = 0; q < n; ++q) order[q] = q;
      std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        return e->cases[x]->g.tsize() > e->cases[y]->g.tsize();
      });
      for (int q : order) {
        bool complete = false;
        if (e->batch > 1) {
          if (int rc = record_step(e->cases[q], &rec[q], &complete)) return rc;
        }
        bool placed = false;
        for (auto& gr : groups)
          if (complete && gr.size() > 0 && !rec[gr[0]].e.empty() && same_record(rec[gr[0]], rec[q])) {
            gr.push_back(q);
            placed = true;
            break;
          }
        if (!placed) {
          groups.push_back({q});
          if (!complete) rec[q].e.clear();  // never joined by another case
        }
      }
      // a group runs as chains of at most e->batch cases, so that the
      // latency-bound stages of one chain overlap the others' work
      {
        const size_t chain = (size_t)std::max(1, e->batch);
        std::vector<std::vector<int>> split;
        for (auto& gr : groups)
          for (size_t q0 = 0; q0 < gr.size(); q0 += chain)
            split.emplace_back(gr.begin() + q0, gr.begin() + std::min(gr.size(), q0 + chain));
        groups.swap(split);
      }
      e->ngroups = (int)groups.size();
      e->grouped = 0;
      // argument tables: per group and launch, the cases' argument lists in
      // case order, in one device buffer; each table starts on a 128-byte
      // boundary (argument lists that hold tensor maps need 64)
      std::vector<std::vector<size_t>> off(groups.size());
      size_t total = 0;
      for (size_t gi = 0; gi < groups.size(); ++gi) {
        const auto& gr = groups[gi];
        if (gr.size() < 2) continue;
        e->grouped += (int)gr.size();
        for (const RecEntry& en : rec[gr[0]].e) {
          if (en.prepare(en)) return CANSFZ_ERR_CUDA;
          off[gi].push_back(total);
          total += (gr.size() * en.args.size() + 127) / 128 * 128;
        }
      }
      if (e->argtab[par]) {
        cudaFree(e->argtab[par]);
        e->argtab[par] = nullptr;
      }
      if (total > 0) {
        std::vector<unsigned char> host(total, 0);
        for (size_t gi = 0; gi < groups.size(); ++gi) {
          const auto& gr = groups[gi];
          if (gr.size() < 2) continue;
          for (size_t p = 0; p < rec[gr[0]].e.size(); ++p) {
            const size_t sz = rec[gr[0]].e[p].args.size();
            for (size_t q = 0; q < gr.size(); ++q)
              std::memcpy(host.data() + off[gi][p] + q * sz, rec[gr[q]].e[p].args.data(), sz);
          }
        }
        CK(cudaMalloc(&e->argtab[par], total));
        CK(cudaMemcpy(e->argtab[par], host.data(), total, cudaMemcpyHostToDevice));
      }
      cudaGraph_t graph;
      CK(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
      CK(cudaEventRecord(e->fork, e->st));
      for (size_t gi = 0; gi < groups.size(); ++gi) {
        const auto& gr = groups[gi];
        cansfz_ctx* c0 = e->cases[gr[0]];
        cudaStream_t bs = c0->st;
        CK(cudaStreamWaitEvent(bs, e->fork, 0));
        if (gr.size() == 1) {
          c0->L.batched = 1;
          enqueue_step(c0);
          c0->L.batched = 0;
        } else {
          const unsigned char* tab = static_cast<const unsigned char*>(e->argtab[par]);
          for (size_t p = 0; p < rec[gr[0]].e.size(); ++p) {
            const RecEntry& en = rec[gr[0]].e[p];
            if (en.launch(en, (int)gr.size(), tab + off[gi][p], bs)) {
              cudaGraph_t bad = nullptr;
              cudaStreamEndCapture(e->st, &bad);
              if (bad) cudaGraphDestroy(bad);
              return CANSFZ_ERR_CUDA;
            }
          }
        }
        CK(cudaEventRecord(e->join[gr[0]], bs));
        CK(cudaStreamWaitEvent(e->st, e->join[gr[0]], 0));
      }
      CK(cudaStreamEndCapture(e->st, &graph));
      CK(cudaGraphInstantiate(&e->gexec[par], graph, 0));
      cudaGraphDestroy(graph);
    }
    CK(cudaGraphLaunch(e->gexec[par], e->st));
    e->cur ^= 1;
    for (cansfz_ctx* c : e->cases) c->cur ^= 1;
  }
  CK(cudaStreamSynchronize(e->st));
  int worst = CANSFZ_OK;
  for (int q = 0; q < n; ++q) {
    cansfz_ctx* c = e->cases[q];
    if (int rc = sync_status(c)) return rc;
    // a case that aborted skipped its later steps: its parity follows the executed count
    const long long done = c->sc_host->istep - istep0[q];
    if ((long long)nsteps != done) c->cur ^= (int)((nsteps - done) & 1);
    c->last_status = c->sc_host->status;
    if (status_out) status_out[q] = c->last_status;
    if (c->last_status != CANSFZ_OK && worst == CANSFZ_OK) worst = c->last_status;
  }
  return worst;
}

int cansfz_ensemble_set_batching(cansfz_ensemble* e, int cases_per_launch) {
  if (!e || cases_per_launch < 1) return CANSFZ_ERR_ARG;
  if (cases_per_launch != e->batch) {
    e->batch = cases_per_launch;
    for (int q = 0; q < 2; ++q)
      if (e->gexec[q]) {
        cudaGraphExecDestroy(e->gexec[q]);
        e->gexec[q] = nullptr;
      }
  }
  return CANSFZ_OK;
}

int cansfz_ensemble_info(cansfz_ensemble* e, int* ngroups, int* grouped_cases) {
  if (!e) return CANSFZ_ERR_ARG;
  if (ngroups) *ngroups = e->ngroups;
  if (grouped_cases) *grouped_cases = e->grouped;
  return CANSFZ_OK;
}

int cansfz_step(cansfz_ctx* c, int nsteps) {
  if (!c || nsteps < 0) return CANSFZ_ERR_ARG;
  if (!c->prepared) {
    int rc = cansfz_prepare(c);
    if (rc) return rc;
  }
  if (c->last_status != CANSFZ_OK) return c->last_status;
  if (int rc = sync_status(c)) return rc;
  const long long istep0 = c->sc_host->istep;
  for (int s = 0; s < nsteps; ++s) {
    const int par = c->cur;
    if (!c->gexec[par]) {
      cudaGraph_t graph;
      CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
      enqueue_step(c);
      CK(cudaStreamEndCapture(c->st, &graph));
      CK(cudaGraphInstantiate(&c->gexec[par], graph, 0));
      cudaGraphDestroy(graph);
    }
    CK(cudaGraphLaunch(c->gexec[par], c->st));
    c->cur ^= 1;
  }
  if (int rc = sync_status(c)) return rc;
  // steps after an abort did nothing: put the parity back to the executed count
  const long long done = c->sc_host->istep - istep0;
  if ((long long)nsteps != done) c->cur ^= (int)((nsteps - done) & 1);
  c->last_status = c->sc_host->status;
  return c->last_status;
}

namespace {
int fill_diag(cansfz_ctx* c, cansfz_diag* d, bool with_mass) {
  if (!c || !d) return CANSFZ_ERR_ARG;
  if (with_mass)
    launch_mass(c->L, c->g, c->ph, c->sc, c->partial, c->psi[c->cur], c->P.l[0] * c->P.l[1] * c->P.l[2]);
  if (int rc = sync_status(c)) return rc;
  const DevScalars& h = *c->sc_host;
  std::memset(d, 0, sizeof(*d));
  d->time = h.time; d->istep = h.istep; d->dt = h.dt; d->dto = h.dto; d->dt_cfl = h.dt_cfl;
  d->gam = h.gam; d->seps = h.seps; d->divtot = h.divtot; d->divmax = h.divmax;
  d->mass12[0] = with_mass ? h.mass12[0] : std::nan("");
  d->mass12[1] = with_mass ? h.mass12[1] : std::nan("");
  d->status = h.status;
  return CANSFZ_OK;
}
}  // namespace

int cansfz_get_diag(cansfz_ctx* c, cansfz_diag* d) { return fill_diag(c, d, true); }
int cansfz_get_status(cansfz_ctx* c, cansfz_diag* d) { return fill_diag(c, d, false); }

int cansfz_initgrid(int gtype, int nz, double gr, double lz, double* dzc, double* dzf, double* zc, double* zf) {
  if (nz < 1 || !dzc || !dzf || !zc || !zf) return CANSFZ_ERR_ARG;
  host_initgrid(gtype, nz, gr, lz, dzc, dzf, zc, zf);
  return CANSFZ_OK;
}

int cansfz_get_grid(cansfz_ctx* c, double* dzc, double* dzf, double* zc, double* zf, double* dzci, double* dzfi) {
  if (!c) return CANSFZ_ERR_ARG;
  const size_t m = c->dzc.size() * sizeof(double);
  if (dzc) std::memcpy(dzc, c->dzc.data(), m);
  if (dzf) std::memcpy(dzf, c->dzf.data(), m);
  if (zc) std::memcpy(zc, c->zc.data(), m);
  if (zf) std::memcpy(zf, c->zf.data(), m);
  if (dzci) std::memcpy(dzci, c->dzci.data(), m);
  if (dzfi) std::memcpy(dzfi, c->dzfi.data(), m);
  return CANSFZ_OK;
}

// ---------------------------------------------------------------------------
// per-procedure drop-in entries
// ---------------------------------------------------------------------------
int cansfz_acdi_transport_pf(cansfz_ctx* c, double gam, double seps, const double* u, const double* v,
                             const double* w, const double* normx, const double* normy, const double* normz,
                             const double* phi, const double* psi, double* dpsidt, double* fx, double* fy,
                             double* fz) {
  if (!c) return CANSFZ_ERR_ARG;
  DevScalars h{};
  h.gam = gam; h.seps = seps;
  if (int rc = call_scalars(c, h)) return rc;
  launch_acdi_transport(c->L, c->g, c->sc_call, c->ph.sdf != 0, u, v, w, normx, normy, normz, phi, psi, dpsidt, fx,
                        fy, fz);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_vof_thinc_transport_psi(cansfz_ctx* c, double beta, const double* u, const double* v, const double* w,
                                   const double* normx, const double* normy, const double* normz, const double* phi,
                                   const double* psi, double* dpsidt, double* fx, double* fy, double* fz) {
  if (!c) return CANSFZ_ERR_ARG;
  DevScalars h{};
  h.beta = beta;
  if (int rc = call_scalars(c, h)) return rc;
  launch_thinc_transport(c->L, c->g, c->sc_call, c->ph.sdf != 0, u, v, w, normx, normy, normz, phi, psi, dpsidt,
                         fx, fy, fz);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_rk_2fl(cansfz_ctx* c, const double rkpar[2], double dt, double gam, double seps, double beta,
                  const double* u, const double* v, const double* w, const double* normx, const double* normy,
                  const double* normz, const double* phi, double* psi, double* fx, double* fy, double* fz) {
  if (!c || !rkpar) return CANSFZ_ERR_ARG;
  DevScalars h{};
  h.gam = gam; h.seps = seps; h.beta = beta;
  h.f1 = rkpar[0] * dt; h.f2 = rkpar[1] * dt; h.f12 = h.f1 + h.f2;
  h.first_rk2fl = c->first_rk2fl_call ? 1 : 0;
  if (int rc = call_scalars(c, h)) return rc;
  if (c->ph.acdi)
    launch_acdi_transport(c->L, c->g, c->sc_call, c->ph.sdf != 0, u, v, w, normx, normy, normz, phi, psi, c->tpsi,
                          fx, fy, fz);
  else
    launch_thinc_transport(c->L, c->g, c->sc_call, c->ph.sdf != 0, u, v, w, normx, normy, normz, phi, psi, c->tpsi,
                           fx, fy, fz);
  // psi += f1*d + f2*d_old (in place), d_old <- d; then clip_field (whole array)
  launch_psi_update(c->L, c->g, c->sc_call, psi, psi, c->tpsi, c->hpsi);
  launch_copy(c->L, (size_t)c->g.tsize(), c->tpsi, c->hpsi);
  launch_clip(c->L, c->g, 0., 1., psi);
  c->first_rk2fl_call = false;
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_acdi_cmpt_phi(cansfz_ctx* c, double seps, const double* psi, double* phi) {
  if (!c) return CANSFZ_ERR_ARG;
  DevScalars h{};
  h.seps = seps;
  if (int rc = call_scalars(c, h)) return rc;
  launch_cmpt_phi(c->L, c->g, c->sc_call, true, psi, phi);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_vof_thinc_cmpt_phi(cansfz_ctx* c, double beta, const double* psi, double* phi) {
  if (!c) return CANSFZ_ERR_ARG;
  DevScalars h{};
  h.beta = beta;
  if (int rc = call_scalars(c, h)) return rc;
  launch_cmpt_phi(c->L, c->g, c->sc_call, false, psi, phi);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_acdi_set_gamma(cansfz_ctx* c, double gam_factor, const double* u, const double* v, const double* w,
                          double* gam) {
  if (!c || !gam) return CANSFZ_ERR_ARG;
  DevScalars h{};
  if (int rc = call_scalars(c, h)) return rc;
  Phys ph = c->ph;
  ph.gam_factor = gam_factor;
  launch_gamma(c->L, c->g, ph, c->sc_call, c->partial, u, v, w, false);
  DevScalars r{};
  CK(cudaMemcpyAsync(&r, c->sc_call, sizeof(r), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  *gam = r.gam;
  return CANSFZ_OK;
}

int cansfz_cmpt_norm_curv_youngs(cansfz_ctx* c, const double* psi, double* normx, double* normy, double* normz,
                                 double* kappa) {
  if (!c) return CANSFZ_ERR_ARG;
  launch_youngs(c->L, c->g, nullptr, psi, normx, normy, normz, kappa);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_clip_field(cansfz_ctx* c, double rmin, double rmax, double* p) {
  if (!c) return CANSFZ_ERR_ARG;
  launch_clip(c->L, c->g, rmin, rmax, p);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_mom_xyz_ad(cansfz_ctx* c, const double* fx, const double* fy, const double* fz, const double* u,
                      const double* v, const double* w, const double* psi, double* dudt, double* dvdt,
                      double* dwdt) {
  if (!c) return CANSFZ_ERR_ARG;
  launch_mom_ad(c->L, c->g, c->ph, fx, fy, fz, u, v, w, psi, dudt, dvdt, dwdt);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

// the balanced-split histories of a per-procedure call: the reference's
// in-place update (surf_o = surf_n, surf_n = new) on the current slots
static SurfSplit call_split(const cansfz_ctx* c) {
  SurfSplit sp{};
  if (!c->ph.balanced) return sp;
  const int a = c->cur;
  for (int d = 0; d < 3; ++d) {
    sp.n[d] = sp.out_n[d] = c->surf[a][d];
    sp.o[d] = sp.out_o[d] = c->surf[a ^ 1][d];
  }
  return sp;
}

int cansfz_mom_xyz_oth(cansfz_ctx* c, double dt_r, const double rho_av[3], const double* p, const double* psi,
                       const double* kappa, const double* s, const double* pn, const double* po, double* dudt,
                       double* dvdt, double* dwdt) {
  if (!c || !rho_av) return CANSFZ_ERR_ARG;
  DevScalars h{};
  h.dt_r = dt_r;
  for (int d = 0; d < 3; ++d) h.rho_av[d] = rho_av[d];
  if (int rc = call_scalars(c, h)) return rc;
  if (c->ph.boussinesq && !s) return CANSFZ_ERR_ARG;
  const SurfSplit sp = call_split(c);
  launch_mom_oth(c->L, c->g, c->ph, c->sc_call, p, psi, kappa, c->ph.boussinesq ? s : nullptr,
                 c->ph.balanced ? &sp : nullptr, pn, po, dudt, dvdt,
                 dwdt);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_rk(cansfz_ctx* c, const double rkpar[2], double dt, double dt_r, const double rho_av[3], const double* psi,
              const double* kappa, const double* p, const double* pn, const double* po, const double* s,
              const double* psio, const double* fx, const double* fy, const double* fz, double* u, double* v,
              double* w) {
  if (!c || !rkpar || !rho_av) return CANSFZ_ERR_ARG;
  if (c->ph.boussinesq && !s) return CANSFZ_ERR_ARG;
  DevScalars h{};
  h.f1 = rkpar[0] * dt; h.f2 = rkpar[1] * dt; h.f12 = h.f1 + h.f2;
  h.dt_r = dt_r;
  for (int d = 0; d < 3; ++d) h.rho_av[d] = rho_av[d];
  h.first_rk = c->first_rk_call ? 1 : 0;
  if (int rc = call_scalars(c, h)) return rc;
  const Launch& L = c->L;
  // src/rk.f90:72-130: mom_xyz_ad -> update 1 (history in place) -> mom_xyz_oth -> update 2
  launch_mom_ad(L, c->g, c->ph, fx, fy, fz, u, v, w, psi, c->tu, c->tv, c->tw_);
  launch_rk_update1(L, c->g, c->ph, c->sc_call, psio, psi, c->tu, c->tv, c->tw_, c->hu, c->hv, c->hw, u, v, w);
  launch_copy(L, (size_t)c->g.tsize(), c->tu, c->hu);
  launch_copy(L, (size_t)c->g.tsize(), c->tv, c->hv);
  launch_copy(L, (size_t)c->g.tsize(), c->tw_, c->hw);
  const SurfSplit sp = call_split(c);
  launch_mom_oth(L, c->g, c->ph, c->sc_call, p, psi, kappa, c->ph.boussinesq ? s : nullptr,
                 c->ph.balanced ? &sp : nullptr, pn, po, c->tu, c->tv,
                 c->tw_);
  launch_rk_update2(L, c->g, c->ph, c->sc_call, psi, c->tu, c->tv, c->tw_, u, v, w);
  c->first_rk_call = false;
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_scal_ad(cansfz_ctx* c, const double* fx, const double* fy, const double* fz, const double* psi,
                   const double* u, const double* v, const double* w, const double* s, double* dsdt) {
  if (!c) return CANSFZ_ERR_ARG;
  if (!c->P.scalar) return CANSFZ_ERR_UNSUPPORTED;
  launch_scal_ad<double>(c->L, c->g, c->ph, fx, fy, fz, psi, u, v, w, s, dsdt);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_rk_scal(cansfz_ctx* c, const double rkpar[2], double dt, const double* psi, const double* u,
                   const double* v, const double* w, const double* psio, const double* fx, const double* fy,
                   const double* fz, double* s) {
  if (!c || !rkpar) return CANSFZ_ERR_ARG;
  if (!c->P.scalar) return CANSFZ_ERR_UNSUPPORTED;
  DevScalars h{};
  h.f1 = rkpar[0] * dt; h.f2 = rkpar[1] * dt; h.f12 = h.f1 + h.f2;
  h.first_scal = c->first_rkscal_call ? 1 : 0;
  if (int rc = call_scalars(c, h)) return rc;
  // src/rk.f90:169-190: scal_ad into scratch, then the update in place (history in ctx)
  launch_scal_ad<double>(c->L, c->g, c->ph, fx, fy, fz, psi, u, v, w, s, c->tpsi);
  launch_scal_update(c->L, c->g, c->ph, c->sc_call, psi, psio, c->tpsi, c->hs, s);
  c->first_rkscal_call = false;
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_fillps(cansfz_ctx* c, double dti, const double* u, const double* v, const double* w, double* p) {
  if (!c) return CANSFZ_ERR_ARG;
  DevScalars h{};
  h.dti = dti;
  if (int rc = call_scalars(c, h)) return rc;
  launch_fillps(c->L, c->g, c->ph, c->sc_call, u, v, w, p);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_updt_rhs_b(cansfz_ctx* c, double* p) {
  if (!c) return CANSFZ_ERR_ARG;
  if (!c->rhsb_zero) launch_updt_rhs_b(c->L, c->g, c->is_bound, c->rhsbx, c->rhsby, c->rhsbz, p);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_solver(cansfz_ctx* c, double* p) {
  if (!c) return CANSFZ_ERR_ARG;
  DevScalars h{};
  if (int rc = call_scalars(c, h)) return rc;
  launch_poisson(c->L, c->g, c->pl, c->sc_call, p);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_correc(cansfz_ctx* c, double dt, const double* p, double* u, double* v, double* w) {
  if (!c) return CANSFZ_ERR_ARG;
  DevScalars h{};
  h.dt = dt;
  if (int rc = call_scalars(c, h)) return rc;
  launch_correc(c->L, c->g, c->ph, c->sc_call, p, u, v, w);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_updatep(cansfz_ctx* c, const double* pp, double* p) {
  if (!c) return CANSFZ_ERR_ARG;
  launch_updatep_full(c->L, c->g, pp, p);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_boundp(cansfz_ctx* c, int which, double* p) {
  if (!c || which < 0 || which > 6) return CANSFZ_ERR_ARG;
  if (which == 6 && !c->P.scalar) return CANSFZ_ERR_UNSUPPORTED;
  run_bcp(c, which, p, nullptr);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_bounduvw(cansfz_ctx* c, int is_correc, double* u, double* v, double* w) {
  if (!c) return CANSFZ_ERR_ARG;
  run_bcuvw(c, is_correc != 0, u, v, w, nullptr);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

int cansfz_chkdt(cansfz_ctx* c, const double* u, const double* v, const double* w, double gam, double seps,
                 double* dtmax) {
  if (!c || !dtmax) return CANSFZ_ERR_ARG;
  DevScalars h{};
  h.gam = gam; h.seps = seps;
  if (int rc = call_scalars(c, h)) return rc;
  launch_chkdt(c->L, c->g, c->ph, c->sc_call, c->partial, u, v, w, false);
  DevScalars r{};
  CK(cudaMemcpyAsync(&r, c->sc_call, sizeof(r), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  *dtmax = r.dt_cfl;
  return CANSFZ_OK;
}

int cansfz_chkdiv(cansfz_ctx* c, const double* u, const double* v, const double* w, double* divtot, double* divmax) {
  if (!c || !divtot || !divmax) return CANSFZ_ERR_ARG;
  DevScalars h{};
  if (int rc = call_scalars(c, h)) return rc;
  launch_chkdiv(c->L, c->g, c->sc_call, c->partial, u, v, w, false);
  DevScalars r{};
  CK(cudaMemcpyAsync(&r, c->sc_call, sizeof(r), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  *divtot = r.divtot;
  *divmax = r.divmax;
  return CANSFZ_OK;
}

int cansfz_bulk_mean_12_stag(cansfz_ctx* c, int idir, const double* psi, double* mean) {
  if (!c || !mean || idir < 1 || idir > 3) return CANSFZ_ERR_ARG;
  DevScalars h{};
  if (int rc = call_scalars(c, h)) return rc;
  const double* gvr = c->d_grid + (idir == 3 ? 5 : 4) * (c->g.nz + 2);
  launch_bulk_mean(c->L, c->g, c->ph, c->sc_call, c->partial, idir, gvr, psi);
  DevScalars r{};
  CK(cudaMemcpyAsync(&r, c->sc_call, sizeof(r), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  *mean = r.rho_av[idir - 1];
  return CANSFZ_OK;
}

int cansfz_cmpt_mean_mass(cansfz_ctx* c, const double* psi, double mass12[2]) {
  if (!c || !mass12) return CANSFZ_ERR_ARG;
  launch_mass(c->L, c->g, c->ph, c->sc_call, c->partial, psi, c->P.l[0] * c->P.l[1] * c->P.l[2]);
  DevScalars r{};
  CK(cudaMemcpyAsync(&r, c->sc_call, sizeof(r), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  mass12[0] = r.mass12[0];
  mass12[1] = r.mass12[1];
  return CANSFZ_OK;
}

// Library-only controls used by the Python host (not reference procedures).
int cansfz_set_time(cansfz_ctx* c, double time, long long istep) {
  if (!c) return CANSFZ_ERR_ARG;
  if (int rc = sync_status(c)) return rc;
  c->sc_host->time = time;
  c->sc_host->istep = istep;
  if (int rc = upload_scalars(c, c->sc, *c->sc_host)) return rc;
  CK(cudaStreamSynchronize(c->st));
  return CANSFZ_OK;
}

int cansfz_set_inivel(cansfz_ctx* c, const char* inivel) {
  if (!c || !inivel) return CANSFZ_ERR_ARG;
  std::snprintf(c->inivel, sizeof(c->inivel), "%s", inivel);
  for (auto& ge : c->gexec)
    if (ge) { cudaGraphExecDestroy(ge); ge = nullptr; }
  return CANSFZ_OK;
}

// ---------------------------------------------------------------------------
// initial conditions on the device, into the current slot (cansfz_prepare
// follows, as the reference's start-up follows its init calls)
// ---------------------------------------------------------------------------
// init2fl, src/two_fluid.f90:247-437 (spheres: nspheres rows x, y, z, r as
// read_sphere_file reads spheres.in; none: the reference's default sphere)
int cansfz_init2fl(cansfz_ctx* c, const char* inipsi, const double* spheres, int nspheres) {
  if (!c || !inipsi || nspheres < 0 || (nspheres > 0 && !spheres)) return CANSFZ_ERR_ARG;
  const cansfz_params& P = c->P;
  const std::string s(inipsi);
  Init2fl a{};
  for (int d = 0; d < 3; ++d) a.idir[d] = 1;
  if (s == "uni") {
  } else if (s == "zer") {
    a.zer = 1;
  } else if (s == "bub3" || s == "drp3" || s == "dis3") {
    a.sphere = 1; a.swap = s != "bub3";
  } else if (s == "bub2" || s == "drp2" || s == "dis2") {
    a.sphere = 1; a.swap = s != "bub2"; a.idir[1] = 0;
  } else if (s == "bub1" || s == "drp1" || s == "dis1") {
    a.sphere = 1; a.swap = s != "bub1"; a.idir[0] = a.idir[1] = 0;
  } else if (s == "flm") {
    a.flm = 1;
  } else {
    return CANSFZ_ERR_ARG;
  }
  std::vector<double> sph;
  if (a.sphere) {
    sph.assign(spheres, spheres + 4 * (size_t)nspheres);
    if (nspheres == 0) {
      double lmin = 1e300;
      for (int d = 0; d < 3; ++d)
        if (a.idir[d]) lmin = std::min(lmin, P.l[d]);
      sph = {P.l[0] / 2, P.l[1] / 2, P.l[2] / 2, 0.25 * lmin};
    }
  }
  a.nsph = (int)(sph.size() / 4);
  for (int d = 0; d < 3; ++d) {
    a.l[d] = P.l[d];
    a.iperiod[d] = is_pp(P.cbcpsi[d]) ? 1 : 0;
    a.lmax = std::max(a.lmax, P.l[d] * a.idir[d]);
  }
  a.seps = c->seps;
  a.reach = 40. * c->seps;
  double* d_sph = nullptr;
  if (a.nsph > 0 && cudaMalloc(&d_sph, sph.size() * sizeof(double)) != cudaSuccess) return CANSFZ_ERR_NOMEM;
  cudaError_t e = cudaSuccess;
  if (d_sph) e = cudaMemcpyAsync(d_sph, sph.data(), sph.size() * sizeof(double), cudaMemcpyHostToDevice, c->st);
  if (e == cudaSuccess) {
    launch_init2fl(c->L, c->g, a, d_sph, c->d_grid + 6 * (c->g.nz + 2), c->psi[c->cur]);
    e = cudaGetLastError();
  }
  const cudaError_t es = cudaStreamSynchronize(c->st);  // the copy and kernel are done before the free
  if (d_sph) cudaFree(d_sph);
  if (e != cudaSuccess || es != cudaSuccess) return CANSFZ_ERR_CUDA;
  c->prepared = false;
  return CANSFZ_OK;
}

// a z profile (nz+2 values, k = 0..nz+1) into a halo field's interior
static int fill_profile(cansfz_ctx* c, const std::vector<double>& prof, double* f) {
  CK(cudaMemcpyAsync(c->tpsi, prof.data(), prof.size() * sizeof(double), cudaMemcpyHostToDevice, c->st));
  launch_fill_zprofile(c->L, c->g, c->tpsi, f);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

// initflow, src/initflow.f90:16-361: 'zer', 'uni', 'cou', 'poi' (with
// set_mean, :464-485) from their z profiles, 'voy' and 'vox' at the
// context's time; v, w, p zero elsewhere
int cansfz_initflow(cansfz_ctx* c, const char* inivel) {
  if (!c || !inivel) return CANSFZ_ERR_ARG;
  const cansfz_params& P = c->P;
  const Geo& g = c->g;
  const std::string s(inivel);
  const int a = c->cur, nz = g.nz;
  const size_t H = (size_t)g.hsize();
  for (double* f : {c->v[a], c->w[a], c->p[a]}) launch_fill(c->L, H, 0., f);
  if (s == "voy" || s == "vox") {
    launch_fill(c->L, H, 0., c->u[a]);
    dim3 bb(g.nx >= 128 ? 128 : 64), gg((g.nx + bb.x - 1) / bb.x, g.ny, g.nz);
    k_prescribed_vel<<<gg, bb, 0, c->st>>>(g, c->sc, s == "voy" ? 1 : 2, P.l[0], P.l[1], P.l[2],
                                          c->d_grid + 6 * (nz + 2), c->d_grid + 7 * (nz + 2), c->u[a], c->v[a],
                                          c->w[a], c->p[a]);
    CK(cudaGetLastError());
  } else if (s == "zer" || s == "uni" || s == "cou" || s == "poi") {
    std::vector<double> u1d(nz + 2, 0.);
    for (int k = 1; k <= nz; ++k) {
      const double z = c->zc[k] / P.l[2];
      if (s == "uni") u1d[k] = 1.;
      else if (s == "cou") u1d[k] = .5 * (1. - 2. * z) * (P.bcvel[0][2][0] - P.bcvel[0][2][1]);
      else if (s == "poi") u1d[k] = 6. * z * (1. - z) * 1.;
    }
    if (s == "poi") {  // set_mean over the interior, in the reference's loop order
      double meanold = 0.;
      for (int k = 1; k <= nz; ++k) {
        const double gk = c->dzf[k] / P.l[2] * (c->dl[0] / P.l[0]) * (c->dl[1] / P.l[1]);
        for (int j = 1; j <= g.ny; ++j)
          for (int i = 1; i <= g.nx; ++i) meanold = meanold + u1d[k] * gk;
      }
      if (meanold != 0.)
        for (int k = 1; k <= nz; ++k) u1d[k] = u1d[k] / meanold * 1.;
    }
    if (int rc = fill_profile(c, u1d, c->u[a])) return rc;
  } else {
    return CANSFZ_ERR_ARG;
  }
  CK(cudaStreamSynchronize(c->st));
  c->prepared = false;
  return CANSFZ_OK;
}

// initscal, src/initflow.f90:363-429 ('cou', 'dhc', 'uni', 'zer')
int cansfz_initscal(cansfz_ctx* c, const char* inisca) {
  if (!c || !inisca) return CANSFZ_ERR_ARG;
  const cansfz_params& P = c->P;
  if (!P.scalar) return CANSFZ_ERR_UNSUPPORTED;
  const std::string s(inisca);
  const int a = c->cur, nz = c->g.nz;
  if (s == "dhc") {
    launch_fill_xprofile(c->L, c->g, P.bcsca[0][0], P.bcsca[0][1], P.l[0], c->s[a]);
    CK(cudaGetLastError());
  } else if (s == "cou" || s == "uni" || s == "zer") {
    std::vector<double> s1d(nz + 2, 0.);
    const double sref = 0.5 * (P.bcsca[2][0] + P.bcsca[2][1]);
    for (int k = 1; k <= nz; ++k) {
      if (s == "uni") {
        s1d[k] = sref;
      } else if (s == "cou") {
        double v = .5 * (1. - 2. * (c->zc[k] / P.l[2])) * 1.;
        v = v + 0.5;
        s1d[k] = P.bcsca[2][0] * v + P.bcsca[2][1] * (1. - v);
      }
    }
    if (int rc = fill_profile(c, s1d, c->s[a])) return rc;
  } else {
    return CANSFZ_ERR_ARG;
  }
  CK(cudaStreamSynchronize(c->st));
  c->prepared = false;
  return CANSFZ_OK;
}


// ---------------------------------------------------------------------------
// library-only measurement helpers (no reference counterpart)
// ---------------------------------------------------------------------------
// Number of kernel nodes in the captured step graph of the current parity.
int cansfz_kernels_per_step(cansfz_ctx* c, int* count) {
  if (!c || !count) return CANSFZ_ERR_ARG;
  cudaGraph_t graph;
  CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
  enqueue_step(c);
  CK(cudaStreamEndCapture(c->st, &graph));
  size_t nn = 0;
  CK(cudaGraphGetNodes(graph, nullptr, &nn));
  std::vector<cudaGraphNode_t> nodes(nn);
  CK(cudaGraphGetNodes(graph, nodes.data(), &nn));
  int k = 0;
  for (auto nd : nodes) {
    cudaGraphNodeType t;
    cudaGraphNodeGetType(nd, &t);
    if (t == cudaGraphNodeTypeKernel) ++k;
  }
  cudaGraphDestroy(graph);
  *count = k;
  return CANSFZ_OK;
}

namespace {
struct ProfState {
  cansfz_ctx* c;
  std::vector<cudaEvent_t>* ev;
  std::vector<std::string>* names;
  size_t idx;
};
void prof_mark(void* arg, const char* name) {
  ProfState* s = (ProfState*)arg;
  if (s->idx >= s->ev->size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    s->ev->push_back(e);
  }
  cudaEventRecord((*s->ev)[s->idx], s->c->st);
  if (s->names->size() < s->idx + 1) s->names->push_back(name);
  ++s->idx;
}
}  // namespace

// Run nsteps time steps without the graph, with CUDA events between the
// stages; returns per stage the summed milliseconds (ms[i]) and the stage
// names as a comma-separated list in `names` (capacity `cap` bytes).
int cansfz_profile_stages(cansfz_ctx* c, int nsteps, double* ms, int maxstages, int* nstages, char* names,
                          int cap) {
  if (!c || !ms || !names || !nstages || nsteps < 1) return CANSFZ_ERR_ARG;
  if (!c->prepared) {
    int rc = cansfz_prepare(c);
    if (rc) return rc;
  }
  std::vector<cudaEvent_t> ev;
  std::vector<std::string> nm;
  cudaEvent_t e0;
  CK(cudaEventCreate(&e0));
  std::vector<double> acc;
  for (int s = 0; s < nsteps; ++s) {
    ProfState st{c, &ev, &nm, 0};
    StageMark mk{prof_mark, &st};
    CK(cudaEventRecord(e0, c->st));
    enqueue_step(c, &mk);
    CK(cudaStreamSynchronize(c->st));
    c->cur ^= 1;
    if (acc.size() < st.idx) acc.resize(st.idx, 0.);
    for (size_t q = 0; q < st.idx; ++q) {
      float t = 0.f;
      CK(cudaEventElapsedTime(&t, q == 0 ? e0 : ev[q - 1], ev[q]));
      acc[q] += t;
    }
  }
  std::string all;
  const int ns = std::min<int>((int)acc.size(), maxstages);
  for (int q = 0; q < ns; ++q) {
    ms[q] = acc[q];
    all += (q ? "," : "") + nm[q];
  }
  std::snprintf(names, cap, "%s", all.c_str());
  for (auto e : ev) cudaEventDestroy(e);
  cudaEventDestroy(e0);
  *nstages = ns;
  return sync_status(c);
}


// Mixed-form Poisson solve on its own: p = S32(rhs), then `sweeps` times
// p += S32(rhs - L(p)) with the FP64 residual of the 7-point operator.
// rhs and p are halo-layout device fields; p's ghosts are left filled.
int cansfz_solver_refined(cansfz_ctx* c, const double* rhs, double* p, int sweeps) {
  if (!c || !rhs || !p || sweeps < 0 || sweeps > 16) return CANSFZ_ERR_ARG;
  if (!c->rhsb_zero) return CANSFZ_ERR_UNSUPPORTED;
  const size_t H = (size_t)c->g.hsize();
  int rc;
  if ((rc = alloc_f32_solver(c))) return rc;
  if (!c->res64 && (rc = dalloc(c, &c->res64, H))) return rc;
  DevScalars h{};
  if ((rc = call_scalars(c, h))) return rc;
  launch_poisson_f32(c->L, c->g, c->pl, c->sc_call, rhs, p, false);
  for (int sw = 0; sw < sweeps; ++sw) {
    run_bcp(c, 0, p, nullptr);
    launch_residual(c->L, c->g, c->sc_call, rhs, p, c->res64);
    launch_poisson_f32(c->L, c->g, c->pl, c->sc_call, c->res64, p, true);
  }
  run_bcp(c, 0, p, nullptr);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}

// FP64 residual res = rhs - L(p) of the 7-point operator (p's ghosts filled here)
int cansfz_poisson_residual(cansfz_ctx* c, const double* rhs, double* p, double* res) {
  if (!c || !rhs || !p || !res) return CANSFZ_ERR_ARG;
  DevScalars h{};
  if (int rc = call_scalars(c, h)) return rc;
  run_bcp(c, 0, p, nullptr);
  launch_residual(c->L, c->g, c->sc_call, rhs, p, res);
  CK(cudaGetLastError());
  return CANSFZ_OK;
}
// ---------------------------------------------------------------------------
// launch plans and the autotuner (no reference counterpart)
// ---------------------------------------------------------------------------
static void drop_graphs(cansfz_ctx* c) {
  for (auto& ge : c->gexec)
    if (ge) {
      cudaGraphExecDestroy(ge);
      ge = nullptr;
    }
}

int cansfz_get_plan(cansfz_ctx* c, cansfz_plan* plan) {
  if (!c || !plan) return CANSFZ_ERR_ARG;
  std::memset(plan, 0, sizeof(*plan));
  plan->phase_slots = c->L.phase_slots;
  plan->momentum_slots = c->L.mom_slots;
  plan->zsolve = c->pl.zmode;
  plan->fp32_transforms = c->P.fp32_transforms;
  plan->tile_tma = c->L.tma;
  plan->ghost_images = c->images;
  plan->line_transforms = c->pl.lmode;
  return CANSFZ_OK;
}

int cansfz_set_plan(cansfz_ctx* c, const cansfz_plan* plan) {
  if (!c || !plan) return CANSFZ_ERR_ARG;
  if (plan->phase_slots < 1 || plan->phase_slots > 1024 || plan->momentum_slots < 1 ||
      plan->momentum_slots > 1024 || plan->zsolve < 0 || plan->zsolve > 1 || plan->fp32_transforms < 0 ||
      plan->fp32_transforms > 1 || plan->tile_tma < 0 || plan->tile_tma > 1 || plan->ghost_images < 0 ||
      plan->ghost_images > 1 || plan->line_transforms < 0 || plan->line_transforms > 1)
    return CANSFZ_ERR_ARG;
  CK(cudaStreamSynchronize(c->st));
  c->L.tma = plan->tile_tma;
  c->images = plan->ghost_images;
  c->L.phase_slots = plan->phase_slots;
  c->L.mom_slots = plan->momentum_slots;
  c->pl.zmode = plan->zsolve;
  c->pl.lmode = plan->line_transforms;
  if (plan->fp32_transforms != c->P.fp32_transforms) {
    if (plan->fp32_transforms == 1) {
      for (int d = 0; d < 2; ++d) {
        c->gsave[0][d] = c->pl.gx[d];
        c->gsave[1][d] = c->pl.gy[d];
        c->pl.gx[d] = c->pl.gy[d] = nullptr;
      }
      c->P.fp32_transforms = 1;
    } else {
      c->P.fp32_transforms = 0;
      if (c->gsave[0][0] || c->gsave[1][0]) {
        for (int d = 0; d < 2; ++d) {
          c->pl.gx[d] = c->gsave[0][d];
          c->pl.gy[d] = c->gsave[1][d];
        }
      } else if (c->pl.workf) {
        if (int rc = alloc_xform_gemm(c)) return rc;
      }
    }
  }
  drop_graphs(c);
  return CANSFZ_OK;
}

namespace {
std::string plan_key(const cansfz_ctx* c) {
  cudaDeviceProp prop{};
  int dev = 0;
  cudaGetDevice(&dev);
  cudaGetDeviceProperties(&prop, dev);
  std::string name(prop.name);
  for (auto& ch : name)
    if (ch == ' ') ch = '_';
  char buf[256];
  std::snprintf(buf, sizeof buf, "grid=%dx%dx%d form=%d sweeps=%d vof=%d scalar=%d balanced=%d gpu=%s", c->n[0],
                c->n[1], c->n[2], c->P.form, c->mixed ? c->sweeps : -1, c->P.interface_capturing, c->P.scalar,
                c->P.balanced, name.c_str());
  return buf;
}

// device time per step of `k` with `pl`, after two steps that capture the
// graphs; a huge value when the copy's run stops
double time_plan(cansfz_ctx* k, const cansfz_plan& pl, int nsteps) {
  if (cansfz_set_plan(k, &pl) != CANSFZ_OK) return 1e30;
  if (cansfz_step(k, 2) != CANSFZ_OK) return 1e30;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, k->st);
  const int rc = cansfz_step(k, nsteps);
  cudaEventRecord(e1, k->st);
  cudaEventSynchronize(e1);
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc == CANSFZ_OK ? (double)ms / nsteps : 1e30;
}
}  // namespace

int cansfz_autotune(cansfz_ctx* c, const char* cache_file, cansfz_plan* chosen, char* report, int cap) {
  if (!c) return CANSFZ_ERR_ARG;
  const std::string key = plan_key(c);
  cansfz_plan best{};
  cansfz_get_plan(c, &best);
  // a cached choice
  if (cache_file) {
    if (FILE* f = std::fopen(cache_file, "r")) {
      char line[512];
      bool found = false;
      while (std::fgets(line, sizeof line, f)) {
        const std::string ln(line);
        if (ln.compare(0, key.size(), key) != 0 || ln.size() <= key.size() || ln[key.size()] != ' ') continue;
        cansfz_plan q = best;
        double ms = 0.;
        const char* rest = ln.c_str() + key.size();
        if (std::sscanf(rest, " | phase=%d mom=%d z=%d xf=%d tma=%d img=%d yt=%d ms=%lf", &q.phase_slots,
                        &q.momentum_slots, &q.zsolve, &q.fp32_transforms, &q.tile_tma, &q.ghost_images,
                        &q.line_transforms, &ms) == 8 ||
            std::sscanf(rest, " | phase=%d mom=%d z=%d xf=%d tma=%d img=%d ms=%lf", &q.phase_slots,
                        &q.momentum_slots, &q.zsolve, &q.fp32_transforms, &q.tile_tma, &q.ghost_images, &ms) == 7 ||
            std::sscanf(rest, " | phase=%d mom=%d z=%d xf=%d tma=%d ms=%lf", &q.phase_slots, &q.momentum_slots,
                        &q.zsolve, &q.fp32_transforms, &q.tile_tma, &ms) == 6) {
          q.ms_per_step = ms;
          best = q;
          found = true;
        }
      }
      std::fclose(f);
      if (found) {
        if (int rc = cansfz_set_plan(c, &best)) return rc;
        if (chosen) *chosen = best;
        if (report && cap > 0)
          std::snprintf(report, cap, "cached: phase=%d mom=%d z=%d xf=%d tma=%d img=%d yt=%d ms=%.4f",
                        best.phase_slots, best.momentum_slots, best.zsolve, best.fp32_transforms, best.tile_tma,
                        best.ghost_images, best.line_transforms, best.ms_per_step);
        return CANSFZ_OK;
      }
    }
  }
  // a copy of the case to time on (from the case's current fields)
  if (!c->prepared) {
    if (int rc = cansfz_prepare(c)) return rc;
  }
  cansfz_ctx* k = nullptr;
  int rc = cansfz_create(&c->P, c->st, &k);
  if (rc) return rc;
  const int a = c->cur;
  rc = cansfz_set_fields(k, c->u[a], c->v[a], c->w[a], c->p[a], c->psi[a], 1);
  if (!rc && c->P.scalar) rc = cansfz_set_scalar(k, c->s[a], 1);
  if (!rc) rc = cansfz_prepare(k);
  if (rc) {
    cansfz_destroy(k);
    return rc;
  }
  const double cells = (double)c->n[0] * c->n[1] * c->n[2];
  const int nt = cells >= 8e6 ? 4 : (cells >= 1e6 ? 8 : 20);
  int evals = 0;
  double tbest = time_plan(k, best, nt);
  ++evals;
  auto try_knob = [&](int cansfz_plan::*knob, std::initializer_list<int> vals) {
    const int keep = best.*knob;
    for (int v : vals) {
      if (v == keep) continue;
      cansfz_plan q = best;
      q.*knob = v;
      const double t = time_plan(k, q, nt);
      ++evals;
      if (t < tbest) {
        tbest = t;
        best = q;
      }
    }
  };
  try_knob(&cansfz_plan::phase_slots, {12, 24, 48});
  try_knob(&cansfz_plan::momentum_slots, {24, 48, 96});
  try_knob(&cansfz_plan::tile_tma, {1, 0});
  if (c->wrap) try_knob(&cansfz_plan::ghost_images, {1, 0});
  if (z_part_ok(c->g, c->pl) && !c->pl.zpiv) try_knob(&cansfz_plan::zsolve, {0, 1});
  if (poisson_y2_applies(c->pl)) try_knob(&cansfz_plan::line_transforms, {0, 1});
  if (c->mixed && c->sweeps >= 0 && (xform_gemm_length(c->n[0]) || xform_gemm_length(c->n[1])))
    try_knob(&cansfz_plan::fp32_transforms, {0, 1});
  cansfz_destroy(k);
  best.ms_per_step = tbest;
  if ((rc = cansfz_set_plan(c, &best))) return rc;
  if (chosen) *chosen = best;
  if (cache_file) {
    if (FILE* f = std::fopen(cache_file, "a")) {
      std::fprintf(f, "%s | phase=%d mom=%d z=%d xf=%d tma=%d img=%d yt=%d ms=%.6f\n", key.c_str(),
                   best.phase_slots, best.momentum_slots, best.zsolve, best.fp32_transforms, best.tile_tma,
                   best.ghost_images, best.line_transforms, best.ms_per_step);
      std::fclose(f);
    }
  }
  if (report && cap > 0)
    std::snprintf(report, cap, "tuned (%d candidates): phase=%d mom=%d z=%d xf=%d tma=%d img=%d yt=%d ms=%.4f",
                  evals, best.phase_slots, best.momentum_slots, best.zsolve, best.fp32_transforms, best.tile_tma,
                  best.ghost_images, best.line_transforms, best.ms_per_step);
  return CANSFZ_OK;
}

}  // extern "C"
