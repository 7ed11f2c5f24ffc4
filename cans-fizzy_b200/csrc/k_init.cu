// Initial conditions on the device: init2fl (src/two_fluid.f90:247-437),
// the profile forms of initflow (src/initflow.f90:16-361) and initscal
// (src/initflow.f90:363-429).  The host evaluates what is one-dimensional
// (the z profiles, the set_mean normalisation); the kernels fill the 3-D
// fields, so a case (or an ensemble of cases) is initialised without
// host-side field arrays.
#include "cansfz_internal.cuh"

namespace cansfz {

// smooth_step_tanh, src/two_fluid.f90 (0.5*(1+tanh(r/(2 eps))))
__device__ __forceinline__ double smooth_step(double r, double eps) { return .5 * (1. + tanh(r / (2. * eps))); }

// init2fl over the whole halo array, one thread per point: 1 (or 0 for
// 'zer') everywhere, the film or the spheres on the interior, then the
// swap.  For every sphere the reference takes, over the 27 periodic images,
// the signed distance chosen by its `abs(sdist) <= sdistmin` rule; that loop
// is kept as it is.  A sphere whose nearest image lies beyond r + reach in
// one direction is skipped: every image is then farther than reach = 40 eps
// from its surface, where smooth_step is 1 and leaves the minimum unchanged.
__global__ void k_init2fl(Geo g, Init2fl a, const double* __restrict__ sph, const double* __restrict__ zc,
                          double* __restrict__ psi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > g.nx + 1) return;
  const int j = blockIdx.y, k = blockIdx.z;
  double v = a.zer ? 0. : 1.;
  const bool inner = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny && k >= 1 && k <= g.nz;
  if (inner && a.flm) v = smooth_step(zc[k] - a.l[2] / 2., a.seps);
  if (inner && a.sphere) {
    const double pos[3] = {((double)i - 0.5) * g.dx, ((double)j - 0.5) * g.dy, zc[k]};
    for (int q = 0; q < a.nsph; ++q) {
      const double* s = sph + 4 * q;
      const double r = s[3];
      bool far = false;
      for (int d = 0; d < 3; ++d) {
        if (!a.idir[d]) continue;
        double dd = pos[d] - s[d];
        if (a.iperiod[d]) dd = dd - a.l[d] * rint(dd / a.l[d]);
        if (fabs(dd) > r + a.reach) far = true;
      }
      if (far) continue;
      double sdistmin = a.lmax * 2.0;
      for (int kk = -1; kk <= 1; ++kk)
        for (int jj = -1; jj <= 1; ++jj)
          for (int ii = -1; ii <= 1; ++ii) {
            const double dx = pos[0] + ii * a.iperiod[0] * a.l[0] - s[0];
            const double dy = pos[1] + jj * a.iperiod[1] * a.l[1] - s[1];
            const double dz = pos[2] + kk * a.iperiod[2] * a.l[2] - s[2];
            const double sdist = sqrt(dx * dx * a.idir[0] + dy * dy * a.idir[1] + dz * dz * a.idir[2]) - r;
            if (fabs(sdist) <= sdistmin) sdistmin = sdist;
          }
      v = fmin(v, smooth_step(sdistmin, a.seps));
    }
  }
  if (a.swap) v = 1. - v;
  psi[g.h(i, j, k)] = v;
}

void launch_init2fl(const Launch& L, const Geo& g, const Init2fl& a, const double* sph, const double* zc,
                    double* psi) {
  dim3 b(g.nx + 2 >= 128 ? 128 : 64), gr((g.nx + 2 + b.x - 1) / b.x, g.ny + 2, g.nz + 2);
  k_init2fl<<<gr, b, 0, L.st>>>(g, a, sph, zc, psi);
}

// f = prof[k] on the interior, 0 on the ghosts (initflow's and initscal's
// z profiles)
__global__ void k_fill_zprofile(Geo g, const double* __restrict__ prof, double* __restrict__ f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > g.nx + 1) return;
  const int j = blockIdx.y, k = blockIdx.z;
  const bool inner = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny && k >= 1 && k <= g.nz;
  f[g.h(i, j, k)] = inner ? prof[k] : 0.;
}

void launch_fill_zprofile(const Launch& L, const Geo& g, const double* prof, double* f) {
  dim3 b(g.nx + 2 >= 128 ? 128 : 64), gr((g.nx + 2 + b.x - 1) / b.x, g.ny + 2, g.nz + 2);
  k_fill_zprofile<<<gr, b, 0, L.st>>>(g, prof, f);
}

// initscal 'dhc' (src/initflow.f90:414-424): the linear x profile between the
// x boundary values, xx = (ii-0.5)*dl(1)/l(1) with ii-0.5 a default-real
// difference (exact here); ghosts 0
__global__ void k_fill_xprofile(Geo g, double b0, double b1, double lx, double* __restrict__ f) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > g.nx + 1) return;
  const int j = blockIdx.y, k = blockIdx.z;
  const bool inner = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny && k >= 1 && k <= g.nz;
  const double xx = (double)((float)i - 0.5f) * g.dx / lx;
  f[g.h(i, j, k)] = inner ? ((1. - xx) * b0 + xx * b1) : 0.;
}

void launch_fill_xprofile(const Launch& L, const Geo& g, double b0, double b1, double lx, double* f) {
  dim3 b(g.nx + 2 >= 128 ? 128 : 64), gr((g.nx + 2 + b.x - 1) / b.x, g.ny + 2, g.nz + 2);
  k_fill_xprofile<<<gr, b, 0, L.st>>>(g, b0, b1, lx, f);
}

}  // namespace cansfz
