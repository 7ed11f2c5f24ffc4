"""Seeded synthetic workloads of the benchmark configurations.

Each builder returns (params, fields) with fields = (u, v, w, p, psi) in the
halo layout.  No public dataset is involved: every input comes from
numpy.random.default_rng(seed).

  rising_bubble_3d  64x64x128, domain 1x1x2, periodic x,y, no-slip z walls,
                    bubble D = 0.5 at (0.5,0.5,0.5), rho 1000/100, mu 10/1,
                    sigma 24.5, g = 0.98, ACDI, fluid at rest.
  poisson_256       256^3, PP/PP/NN, RHS ~ N(0,1) (seed 2026), mean removed.
  droplets_acdi     256^3, unit box, 64 droplets R ~ U[0.03,0.06] (dis3,
                    droplets = dense phase), rho 1000/1, mu 100/1, sigma 1,
                    g = 1, random divergence-free u0 (|k| <= 4, rms 0.1), ACDI.
  droplets_thinc    512x512x256, box 2x2x1, same physics, THINC/QQ.
  ensemble_cases    64 rising-bubble cases (seed 4): 32 2-D (ny = 2, periodic
                    y) with (nx, nz) from 64x128 to 256x512 and 32 3-D from
                    32^3 to 96x96x192, sizes 2^a 3^b multiples of 16; rho
                    ratio in {10,100,1000}, mu ratio in {10,100}, sigma in
                    [1,30], bubble diameter in [0.25,0.5] of the box width.
  shear_stretched   512x256x256, gtype 1, gr 1.5, Poiseuille mean 1 with the
                    laminar pressure gradient, 1% seeded perturbation, 200
                    droplets R ~ U[0.04,0.08], rho ratio 10, mu ratio 1,
                    sigma 0.5, ACDI.
"""
from __future__ import annotations

import numpy as np

from . import init, namelist, params


def _walls_z(nx, ny, nz, l, rho, mu, sigma, gacc, vof=False, gr=0.0, bforce=(0.0, 0.0, 0.0), cfl=0.5, icheck=10):
    text = f"""
&dns
ng(1:3) = {nx}, {ny}, {nz}
l(1:3) = {l[0]}, {l[1]}, {l[2]}
gtype = 1, gr = {gr}
cfl = {cfl}, dtmax = 1.e9, dt_f = -1.
icheck = {icheck}
cbcvel(0:1,1:3,1) = 'P','P', 'P','P', 'D','D'
cbcvel(0:1,1:3,2) = 'P','P', 'P','P', 'D','D'
cbcvel(0:1,1:3,3) = 'P','P', 'P','P', 'D','D'
cbcpre(0:1,1:3)   = 'P','P', 'P','P', 'N','N'
bforce(1:3) = {bforce[0]}, {bforce[1]}, {bforce[2]}
gacc(1:3) = {gacc[0]}, {gacc[1]}, {gacc[2]}
/
&two_fluid
cbcpsi(0:1,1:3)   = 'P','P', 'P','P', 'N','N'
cbcnor(0:1,1:3,1) = 'P','P', 'P','P', 'N','N'
cbcnor(0:1,1:3,2) = 'P','P', 'P','P', 'N','N'
cbcnor(0:1,1:3,3) = 'P','P', 'P','P', 'D','D'
rho12(1:2) = {rho[0]}, {rho[1]}
mu12(1:2) = {mu[0]}, {mu[1]}
sigma = {sigma}
psi_thickness_factor = {0.5 if vof else 0.51}
/
&cansfz
interface_capturing_vof = {'T' if vof else 'F'}
/
"""
    return params.from_namelist(namelist.parse(text))


def rising_bubble_3d():
    p = _walls_z(64, 64, 128, (1.0, 1.0, 2.0), (1000.0, 100.0), (10.0, 1.0), 24.5, (0.0, 0.0, -0.98))
    psi = init.init2fl(p, "bub3", np.array([[0.5, 0.5, 0.5, 0.25]]))
    u, v, w, pr = init.initflow(p, "zer")
    return p, (u, v, w, pr, psi)


def droplets(n=(256, 256, 256), l=(1.0, 1.0, 1.0), vof=False, count=64, rmin=0.03, rmax=0.06, seed=2026):
    p = _walls_z(n[0], n[1], n[2], l, (1000.0, 1.0), (100.0, 1.0), 1.0, (0.0, 0.0, -1.0), vof=vof)
    rng = np.random.default_rng(seed)
    eps = init.seps(p)
    sph = init.place_droplets(rng, count, rmin, rmax, list(l), eps)
    psi = init.init2fl(p, "dis3", sph, eps=eps)
    u, v, w = init.divfree_velocity(p, rng, 4, 0.1)
    return p, (u, v, w, np.zeros_like(u), psi)


def droplets_acdi(seed=2026):
    return droplets((256, 256, 256), (1.0, 1.0, 1.0), False, seed=seed)


def droplets_thinc(seed=2026):
    return droplets((512, 512, 256), (2.0, 2.0, 1.0), True, seed=seed)


def shear_stretched(seed=5):
    mu2, rho2, h, ub = 1.0, 1.0, 1.0, 1.0
    bf = 12.0 * mu2 * ub / (rho2 * h * h)   # laminar balance of the Poiseuille profile
    p = _walls_z(512, 256, 256, (2.0, 1.0, 1.0), (10.0, 1.0), (1.0, 1.0), 0.5, (0.0, 0.0, 0.0), gr=1.5,
                 bforce=(bf, 0.0, 0.0))
    rng = np.random.default_rng(seed)
    eps = init.seps(p)
    sph = init.place_droplets(rng, 200, 0.04, 0.08, [2.0, 1.0, 1.0], eps)
    psi = init.init2fl(p, "dis3", sph, eps=eps)
    u, v, w, pr = init.initflow(p, "poi")
    du, dv, dw = init.divfree_velocity(p, rng, 4, 0.01)
    return p, (u + du, v + dv, w + dw, pr, psi)


def poisson_rhs(n=256, seed=2026):
    p = _walls_z(n, n, n, (1.0, 1.0, 1.0), (1.0, 1.0), (0.01, 0.01), 0.0, (0.0, 0.0, 0.0))
    rng = np.random.default_rng(seed)
    rhs = np.zeros((n + 2, n + 2, n + 2), order="F")
    r = rng.standard_normal((n, n, n))
    rhs[1:-1, 1:-1, 1:-1] = r - r.mean()
    return p, rhs


BUILDERS = {
    "rising_bubble_3d": rising_bubble_3d,
    "droplets_acdi": droplets_acdi,
    "droplets_thinc": droplets_thinc,
    "shear_stretched": shear_stretched,
}


def _bubble_case(nx, ny, nz, lx, ly, lz, rho_ratio, mu_ratio, sigma, diam, two_d):
    p = _walls_z(nx, ny, nz, (lx, ly, lz), (1000.0, 1000.0 / rho_ratio), (10.0, 10.0 / mu_ratio), sigma,
                 (0.0, 0.0, -0.98))
    if two_d:
        psi = init.init2fl(p, "bub2", np.array([[0.5 * lx, 0.0, 0.5 * lz, 0.5 * diam]]))
    else:
        psi = init.init2fl(p, "bub3", np.array([[0.5 * lx, 0.5 * ly, 0.5 * lz, 0.5 * diam]]))
    u, v, w, pr = init.initflow(p, "zer")
    return p, (u, v, w, pr, psi)


def ensemble_cases(seed=4, count2d=32, count3d=32):
    """The batched-ensemble configuration: a list of (params, fields)."""
    rng = np.random.default_rng(seed)
    sizes2d = [64, 96, 128, 192, 256]      # nx; nz = 2 nx (box 1 x 2)
    sizes3d = [32, 48, 64, 96]             # nx = ny; nz = 2 nx (box 1 x 1 x 2)
    out = []
    for q in range(count2d + count3d):
        two_d = q < count2d
        n = int(rng.choice(sizes2d if two_d else sizes3d))
        rho_ratio = float(rng.choice([10.0, 100.0, 1000.0]))
        mu_ratio = float(rng.choice([10.0, 100.0]))
        sigma = float(rng.uniform(1.0, 30.0))
        diam = float(rng.uniform(0.25, 0.5))
        if two_d:
            out.append(_bubble_case(n, 2, 2 * n, 1.0, 2.0 / n, 2.0, rho_ratio, mu_ratio, sigma, diam, True))
        else:
            out.append(_bubble_case(n, n, 2 * n, 1.0, 1.0, 2.0, rho_ratio, mu_ratio, sigma, diam, False))
    return out
