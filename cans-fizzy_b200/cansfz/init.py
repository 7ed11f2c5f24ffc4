"""Initial conditions on the host (numpy), halo layout, Fortran order.

* ``init2fl``: the volume-fraction initialisation of src/two_fluid.f90:247-437
  for the sphere/cylinder/film cases ('bub3','bub2','bub1','drp*','dis*',
  'flm','uni','zer').  The 27-image scan of the reference is evaluated as the
  nearest periodic image inside a bounding box per sphere (outside the box
  tanh saturates, so psi_aux == 1 exactly there).
* ``initflow``: the velocity profiles of src/initflow.f90:16-361 used here
  ('zer','uni','cou','poi' with set_mean, 'voy','vox').
* Seeded synthetic inputs (no reference counterpart; the reference's own
  ``add_noise`` uses the compiler's RNG and is not reproducible): droplet
  placement by rejection sampling, and a random divergence-free velocity
  built as the discrete curl of a random vector potential on the staggered
  grid (so div_h u = 0 to round-off, with w = 0 on z walls).
"""
from __future__ import annotations

import ctypes as ct

import numpy as np

from . import lib as _L
from .params import Params


# A host routine with the signature of cansfz_initgrid that replaces the
# library's (None: the library's).  A process that must not load libcansfz
# (the timed CPU run of the reference's algorithm) generates its inputs with
# its own initgrid through this hook.
_initgrid = None


def use_initgrid(fn) -> None:
    """Route zgrid through `fn(gtype, nz, gr, lz, dzc, dzf, zc, zf) -> int`
    (ctypes-callable, double* outputs of nz+2 values); None restores the
    library's cansfz_initgrid."""
    global _initgrid
    _initgrid = fn


def zgrid(p: Params) -> dict:
    """initgrid (src/initgrid.f90:14-78) through the library's host routine
    (or the routine set with use_initgrid)."""
    nz = p.ng[2]
    arrs = [np.zeros(nz + 2) for _ in range(4)]
    fn = _initgrid if _initgrid is not None else _L.load().cansfz_initgrid
    _L.check(fn(int(p.gtype), int(nz), float(p.gr), float(p.l[2]), *[a.ctypes.data_as(_L.PD) for a in arrs]),
             "initgrid")
    dzc, dzf, zc, zf = arrs
    return {"dzc": dzc, "dzf": dzf, "zc": zc, "zf": zf, "dzci": 1.0 / dzc, "dzfi": 1.0 / dzf}


def seps(p: Params) -> float:
    """acdi_set_epsilon (src/acdi.f90:16-30)."""
    g = zgrid(p)
    dl = [p.l[q] / p.ng[q] for q in range(3)]
    dlmax = max(max(dl[0], dl[1]), float(np.max(1.0 / g["dzfi"])))
    return dlmax * p.psi_thickness_factor


def read_spheres(path: str) -> np.ndarray:
    """read_sphere_file (src/two_fluid.f90:439-471): one sphere per line,
    x y z r (list-directed); no file: no spheres (init2fl then uses its
    default sphere).  Returns an (nspheres, 4) array."""
    import os

    if not os.path.exists(path):
        return np.zeros((0, 4))
    rows = []
    with open(path) as f:
        for line in f:
            toks = line.replace(",", " ").split()
            if toks:
                rows.append([float(t.replace("d", "e").replace("D", "e")) for t in toks[:4]])
    return np.array(rows, dtype=np.float64).reshape(-1, 4)


def smooth_step_tanh(r, eps):
    return 0.5 * (1.0 + np.tanh(r / (2.0 * eps)))


def init2fl(p: Params, inipsi: str, spheres=None, eps: float | None = None) -> np.ndarray:
    nx, ny, nz = p.n
    l = [p.l[0], p.l[1], p.l[2]]
    dl = [l[q] / p.ng[q] for q in range(3)]
    g = zgrid(p)
    eps = seps(p) if eps is None else eps
    psi = np.ones((nx + 2, ny + 2, nz + 2), order="F")
    name = inipsi.strip()
    is_dim = [True, True, True]
    is_sphere = is_swap = False
    if name == "zer":
        psi[...] = 0.0
    elif name in ("bub3", "drp3", "dis3"):
        is_sphere, is_swap = True, name != "bub3"
    elif name in ("bub2", "drp2", "dis2"):
        is_dim = [True, False, True]
        is_sphere, is_swap = True, name != "bub2"
    elif name in ("bub1", "drp1", "dis1"):
        is_dim = [False, False, True]
        is_sphere, is_swap = True, name != "bub1"
    elif name == "flm":
        psi[1:-1, 1:-1, 1:-1] = smooth_step_tanh(g["zc"][1:-1] - l[2] / 2.0, eps)[None, None, :]
    elif name != "uni":
        raise ValueError(f"unsupported inipsi {inipsi!r}")
    if is_sphere:
        sph = np.zeros((0, 4)) if spheres is None else np.asarray(spheres, dtype=float).reshape(-1, 4)
        if sph.shape[0] == 0:
            lmin = min(l[q] for q in range(3) if is_dim[q])
            sph = np.array([[l[0] / 2, l[1] / 2, l[2] / 2, 0.25 * lmin]])
        cbcpsi = bytes(p.cbcpsi).decode()
        iperiod = [cbcpsi[2 * q] == "P" and cbcpsi[2 * q + 1] == "P" for q in range(3)]
        xc = (np.arange(1, nx + 1) - 0.5) * dl[0]
        yc = (np.arange(1, ny + 1) - 0.5) * dl[1]
        zc = g["zc"][1:-1]
        reach = 40.0 * eps  # tanh(r/(2 eps)) == 1 in FP64 beyond ~38.1 eps
        coords = [xc, yc, zc]
        inner = psi[1:-1, 1:-1, 1:-1]
        for xs, ys, zs, r in sph:
            ctr = [xs, ys, zs]
            idx, dsq = [], []
            for q in range(3):
                c = coords[q]
                if not is_dim[q]:
                    idx.append(np.arange(c.size))
                    dsq.append(np.zeros(c.size))
                    continue
                d = c - ctr[q]
                if iperiod[q]:
                    d = d - l[q] * np.round(d / l[q])
                sel = np.nonzero(np.abs(d) <= r + reach)[0]
                idx.append(sel)
                dsq.append(d[sel] ** 2)
            if any(s.size == 0 for s in idx):
                continue
            dist = np.sqrt(dsq[0][:, None, None] + dsq[1][None, :, None] + dsq[2][None, None, :])
            aux = smooth_step_tanh(dist - r, eps)
            ix = np.ix_(*idx)
            inner[ix] = np.minimum(inner[ix], aux)
    if is_swap:
        psi = 1.0 - psi
    return np.asfortranarray(psi)


def initflow(p: Params, inivel: str, time: float = 0.0):
    """u, v, w, p (halo layout; ghosts zero) as initflow sets the interior."""
    nx, ny, nz = p.n
    l = [p.l[0], p.l[1], p.l[2]]
    dl = [l[q] / p.ng[q] for q in range(3)]
    g = zgrid(p)
    shp = (nx + 2, ny + 2, nz + 2)
    u, v, w, pr = (np.zeros(shp, order="F") for _ in range(4))
    name = inivel.strip()
    zcn = g["zc"][1:-1] / l[2]
    if name in ("zer", "uni", "cou", "poi"):
        if name == "zer":
            u1d = np.zeros(nz)
        elif name == "uni":
            u1d = np.ones(nz)
        elif name == "cou":
            bcv = np.array(p.bcvel[:]).reshape((2, 3, 3), order="F")
            u1d = 0.5 * (1.0 - 2.0 * zcn) * (bcv[0, 2, 0] - bcv[1, 2, 0])
        else:
            u1d = 6.0 * zcn * (1.0 - zcn) * 1.0
        u[1:-1, 1:-1, 1:-1] = u1d[None, None, :]
        if name == "poi":  # set_mean, src/initflow.f90:464-485
            gv = g["dzf"][1:-1] / l[2] * (dl[0] / l[0]) * (dl[1] / l[1])
            meanold = float(np.sum(u[1:-1, 1:-1, 1:-1] * gv[None, None, :]))
            if meanold != 0.0:
                u[1:-1, 1:-1, 1:-1] = u[1:-1, 1:-1, 1:-1] / meanold * 1.0
    elif name in ("voy", "vox"):
        zff = g["zf"][1:-1] / l[2]
        xc = (np.arange(1, nx + 1) - 0.5) * dl[0] / l[0]
        xf = np.arange(1, nx + 1) * dl[0] / l[0]
        yc = (np.arange(1, ny + 1) - 0.5) * dl[1] / l[1]
        yf = np.arange(1, ny + 1) * dl[1] / l[1]
        ct_ = np.cos(np.pi * time / 4.0)
        if name == "voy":
            u[1:-1, 1:-1, 1:-1] = (np.sin(np.pi * xf)[:, None, None] ** 2 * np.sin(2 * np.pi * zcn)[None, None, :] * ct_)
            w[1:-1, 1:-1, 1:-1] = (-(np.sin(np.pi * zff)[None, None, :] ** 2) * np.sin(2 * np.pi * xc)[:, None, None] * ct_)
        else:
            v[1:-1, 1:-1, 1:-1] = (np.sin(np.pi * yf)[None, :, None] ** 2 * np.sin(2 * np.pi * zcn)[None, None, :] * ct_)
            w[1:-1, 1:-1, 1:-1] = (-(np.sin(np.pi * zff)[None, None, :] ** 2) * np.sin(2 * np.pi * yc)[None, :, None] * ct_)
    else:
        raise ValueError(f"unsupported inivel {inivel!r}")
    return u, v, w, pr


def initscal(p: Params, inisca: str) -> np.ndarray:
    """The scalar s (halo layout; ghosts zero) as initscal sets the interior
    (src/initflow.f90:363-429): 'cou' and 'dhc' start from the Couette
    profile between the z boundary values bcsca(0:1,3); 'dhc' then takes the
    linear profile between the x boundary values; 'uni' is their z mean,
    'zer' zero."""
    nx, ny, nz = p.n
    bc = np.array(p.bcsca[:]).reshape((2, 3), order="F")
    g = zgrid(p)
    zcn = g["zc"][1:-1] / p.l[2]
    name = inisca.strip()
    if name in ("cou", "dhc"):
        s1d = 0.5 * (1.0 - 2.0 * zcn) * 1.0
        s1d = s1d + 0.5
        s1d = bc[0, 2] * s1d + bc[1, 2] * (1.0 - s1d)
    elif name == "uni":
        s1d = np.full(nz, 0.5 * (bc[0, 2] + bc[1, 2]))
    elif name == "zer":
        s1d = np.zeros(nz)
    else:
        raise ValueError(f"invalid name for initial scalar field {inisca!r}")
    s = np.zeros((nx + 2, ny + 2, nz + 2), order="F")
    s[1:-1, 1:-1, 1:-1] = s1d[None, None, :]
    if name == "dhc":
        xx = (np.arange(1, nx + 1) - 0.5) * (p.l[0] / p.ng[0]) / p.l[0]
        s[1:-1, 1:-1, 1:-1] = ((1.0 - xx) * bc[0, 0] + xx * bc[1, 0])[:, None, None]
    return s


# ---------------------------------------------------------------------------
# seeded synthetic inputs
# ---------------------------------------------------------------------------
def place_droplets(rng: np.random.Generator, count: int, rmin: float, rmax: float, l, eps: float,
                   periodic=(True, True, False), max_tries: int = 200000) -> np.ndarray:
    """Rejection sampler: radii U[rmin,rmax], centres uniform; accepted when the
    gap to every other droplet exceeds 4*eps (minimum image in periodic
    directions) and, in wall directions, the droplet keeps 2*eps off the wall."""
    out = []
    tries = 0
    while len(out) < count:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("droplet placement did not converge")
        r = rng.uniform(rmin, rmax)
        c = np.array([rng.uniform(0.0, l[q]) if periodic[q] else rng.uniform(r + 2 * eps, l[q] - r - 2 * eps)
                      for q in range(3)])
        ok = True
        for (x, y, z, rr) in out:
            d = c - np.array([x, y, z])
            for q in range(3):
                if periodic[q]:
                    d[q] -= l[q] * np.round(d[q] / l[q])
            if np.sqrt(np.sum(d * d)) <= r + rr + 4 * eps:
                ok = False
                break
        if ok:
            out.append((c[0], c[1], c[2], r))
    return np.array(out)


def divfree_velocity(p: Params, rng: np.random.Generator, kmax: int = 4, rms: float = 0.1):
    """Random velocity with Fourier modes |k| <= kmax as the discrete curl of a
    vector potential A on cell edges (Ax at (xc,yf,zf), Ay at (xf,yc,zf), Az at
    (xf,yf,zc)); A_x, A_y vanish on the z walls, so w = 0 there and the
    discrete divergence of fillps is zero to round-off.  x and y periodic."""
    nx, ny, nz = p.n
    l = [p.l[0], p.l[1], p.l[2]]
    dl = [l[q] / p.ng[q] for q in range(3)]
    g = zgrid(p)
    xc = (np.arange(nx) + 0.5) * dl[0]
    xf = (np.arange(nx) + 1.0) * dl[0]
    yc = (np.arange(ny) + 0.5) * dl[1]
    yf = (np.arange(ny) + 1.0) * dl[1]
    zc = g["zc"][1:-1]
    zf = g["zf"]  # 0..nz+1, zf[0] = 0, zf[nz] = lz
    # A_c = Re sum_{kx,ky,kz} C_c exp(2 pi i (kx x/Lx + ky y/Ly)) S_c,kz(z): for each
    # kz the (x,y) sum is two small matrix products, then one outer product in z.
    ks = np.arange(-kmax, kmax + 1)
    Ex = {nm: np.exp(2j * np.pi * np.outer(xs, ks) / l[0]) for nm, xs in (("c", xc), ("f", xf))}
    Ey = {nm: np.exp(2j * np.pi * np.outer(ys, ks) / l[1]) for nm, ys in (("c", yc), ("f", yf))}
    kk = ks[:, None] ** 2 + ks[None, :] ** 2
    grids = (("c", "f", zf[: nz + 1], "s"), ("f", "c", zf[: nz + 1], "s"), ("f", "f", zc, "c"))
    A = []
    for comp, (gx, gy, zs, kind) in enumerate(grids):
        acc = np.zeros((nx, ny, zs.size))
        for kz in range(0, kmax + 1):
            mask = (kk + kz * kz <= kmax * kmax) & (kk + kz * kz > 0)
            coef = (rng.standard_normal(kk.shape) + 1j * rng.standard_normal(kk.shape)) / (1.0 + kk + kz * kz)
            coef = np.where(mask, coef, 0.0)
            plane = np.real(Ex[gx] @ coef @ Ey[gy].T)  # (nx, ny)
            if kind == "s":
                prof = np.sin(np.pi * max(kz, 1) * zs / l[2])  # vanishes on both walls
            else:
                prof = np.cos(np.pi * kz * zs / l[2])
            acc += plane[:, :, None] * prof[None, None, :]
        A.append(acc)
    Ax, Ay, Az = A
    dzf = g["dzf"][1:-1]
    dzc = g["dzc"]
    # u(i+1/2, j, k) = (Az(j+1/2) - Az(j-1/2))/dy - (Ay(k+1/2) - Ay(k-1/2))/dzf
    u = (Az - np.roll(Az, 1, axis=1)) / dl[1] - (Ay[:, :, 1:] - Ay[:, :, :-1]) / dzf[None, None, :]
    # v(i, j+1/2, k) = (Ax(k+1/2) - Ax(k-1/2))/dzf - (Az(i+1/2) - Az(i-1/2))/dx
    v = (Ax[:, :, 1:] - Ax[:, :, :-1]) / dzf[None, None, :] - (Az - np.roll(Az, 1, axis=0)) / dl[0]
    # w(i, j, k+1/2) = (Ay(i+1/2) - Ay(i-1/2))/dx - (Ax(j+1/2) - Ax(j-1/2))/dy, k = 0..nz
    w = (Ay - np.roll(Ay, 1, axis=0)) / dl[0] - (Ax - np.roll(Ax, 1, axis=1)) / dl[1]
    cur = np.sqrt(np.mean(np.concatenate([u.ravel() ** 2, v.ravel() ** 2, w[:, :, 1:nz].ravel() ** 2])))
    s = rms / cur
    shp = (nx + 2, ny + 2, nz + 2)
    U, V, W = (np.zeros(shp, order="F") for _ in range(3))
    U[1:-1, 1:-1, 1:-1] = u * s
    V[1:-1, 1:-1, 1:-1] = v * s
    W[1:-1, 1:-1, 0:nz + 1] = w * s
    _ = dzc
    return U, V, W
