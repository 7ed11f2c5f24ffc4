"""Per-procedure parity of the C ABI entries that the whole step fuses away
(rk_2fl, rk, clip_field, updatep, cmpt_mean_mass, bulk_mean_12_stag,
updt_rhs_b), each called through libcansfz on device fields and compared
with the oracle's restatement on the same seeded inputs; and whole steps
of the two step paths that the other parity cases do not reach: gravity
along a periodic direction (bulk_mean_12_stag inside the step,
src/main.f90:470-477) and a non-zero Dirichlet pressure BC (fillps +
updt_rhs_b + the unfused solve, src/main.f90:490-493).

Tolerances, relative to the field's maximum: rk_2fl 1e-13 (psi and the
three face fluxes), rk 1e-12 (u, v, w; the GPU contracts products into
FMAs, the oracle does not), clip_field and updatep bit-equal, the
reductions 1e-13, updt_rhs_b bit-equal on the interior planes it touches
and unchanged elsewhere; whole steps 1e-11 after 10 steps as in
test_gpu_parity.py.
"""
import numpy as np
import pytest

import oracle as O
from cansfz import case as C
from cansfz import init, namelist, params

from test_gpu_parity import _check_step, _nml, _oracle_sensitivity, _rand_fields, _rel, _run_pair

pytestmark = pytest.mark.gpu


@pytest.fixture()
def pair():
    """A fresh case on both sides: the AB2 entries keep `save` histories."""
    p = _nml(24, 16, 20, "PPPPNN", l=(1.0, 0.75, 1.2))
    return p, C.Case(p), O.Case(p)


def test_rk_2fl_two_calls(pair):
    """rk_2fl (src/rk.f90:193-254): the first call seeds the history with the
    current right-hand side (forward Euler), the second is a true AB2 step."""
    p, g, o = pair
    rng, f, psi = _rand_fields(p, 21)
    u, v, w, nx, ny, nz, phi = (f(0.3) for _ in range(7))
    dev = {k: g.field(a) for k, a in dict(u=u, v=v, w=w, nx=nx, ny=ny, nz=nz, phi=phi).items()}
    psig = g.field(psi)
    psio_ = psi.copy(order="F")
    fg = [g.field() for _ in range(3)]
    fo = [o.empty() for _ in range(3)]
    gam, seps, beta = 0.7, 0.013, 1.0
    for call, rkpar, dt in ((0, [1.0, 0.0], 2e-3), (1, [1.45, -0.45], 1.7e-3)):
        g.call("rk_2fl", list(rkpar), dt, gam, seps, beta, dev["u"], dev["v"], dev["w"], dev["nx"], dev["ny"],
               dev["nz"], dev["phi"], psig, *fg)
        o.call("rk_2fl", np.array(rkpar), dt, gam, seps, beta, u, v, w, nx, ny, nz, phi, psio_, *fo)
        assert _rel(psig.get(), psio_) < 1e-13, call
        for a, b in zip(fg, fo):
            assert _rel(a.get()[1:-1, 1:-1, 1:-1], b[1:-1, 1:-1, 1:-1]) < 1e-13, call
        assert psig.get().min() >= 0.0 and psig.get().max() <= 1.0  # clip_field(psi, 0, 1)


def test_rk_two_calls(pair):
    """rk (src/rk.f90:16-131): momentum AB2 with the density ratio, then the
    pressure-split, surface-tension and gravity terms; two calls so that
    the second reads the history the first left."""
    p, g, o = pair
    rng, f, psi = _rand_fields(p, 22)
    psio_ = np.asfortranarray(np.clip(psi + 0.05 * rng.standard_normal(psi.shape), 0, 1))
    u, v, w, fx, fy, fz, pp, pn, po, kap = (f(0.2) for _ in range(10))
    dev = {k: g.field(a) for k, a in dict(psi=psi, psio=psio_, fx=fx, fy=fy, fz=fz, p=pp, pn=pn, po=po,
                                          k=kap).items()}
    ug, vg, wg = g.field(u), g.field(v), g.field(w)
    uo, vo, wo = u.copy(order="F"), v.copy(order="F"), w.copy(order="F")
    rho_av = [0.0, 0.0, 0.0]
    for call, rkpar, dt, dt_r in ((0, [1.0, 0.0], 1e-3, 1.0), (1, [1.4, -0.4], 1.2e-3, 1.2)):
        g.call("rk", list(rkpar), dt, dt_r, rho_av, dev["psi"], dev["k"], dev["p"], dev["pn"], dev["po"], None,
               dev["psio"], dev["fx"], dev["fy"], dev["fz"], ug, vg, wg)
        o.call("rk", np.array(rkpar), dt, dt_r, np.array(rho_av), psi, kap, pp, pn, po, None, psio_, fx, fy, fz,
               uo, vo, wo)
        for a, b in zip((ug, vg, wg), (uo, vo, wo)):
            assert _rel(a.get()[1:-1, 1:-1, 1:-1], b[1:-1, 1:-1, 1:-1]) < 1e-12, call


def test_clip_field_and_updatep(pair):
    p, g, o = pair
    rng, f, _ = _rand_fields(p, 23)
    a = f()
    ag = g.field(a)
    g.call("clip_field", -0.5, 0.75, ag)
    o.call("clip_field", -0.5, 0.75, a)
    assert np.array_equal(ag.get(), a)  # clip_field (src/two_fluid.f90:35-58), whole halo array
    pp, pr = f(), f()
    ppg, prg = g.field(pp), g.field(pr)
    g.call("updatep", ppg, prg)
    o.call("updatep", pp, pr)
    assert np.array_equal(prg.get(), pr)  # updatep (src/updatep.f90:13-24): p = pp + p


def test_reductions_mass_and_bulk_mean(pair):
    """cmpt_mean_mass (src/output.f90:759-790) and bulk_mean_12_stag
    (src/utils.f90:68-136) for the three directions."""
    p, g, o = pair
    rng, f, psi = _rand_fields(p, 24)
    psig = g.field(psi)
    m = np.zeros(2)
    g.call("cmpt_mean_mass", psig, m)
    mo = np.zeros(2)
    o.call("cmpt_mean_mass", psi, mo)
    assert np.all(np.abs(m - mo) <= 1e-13 * np.abs(mo)), (m, mo)
    for idir in (1, 2, 3):
        mean = np.zeros(1)
        g.call("bulk_mean_12_stag", idir, psig, mean)
        ref = o.call("bulk_mean_12_stag", idir, psi)
        assert abs(mean[0] - ref) <= 1e-13 * abs(ref), (idir, mean[0], ref)


_DIRICHLET = """
&dns
ng(1:3) = 32, 24, 28
l(1:3) = 1., 0.75, 1.
cfl = 0.5, dtmax = 1.e9, icheck = 5
cbcvel(0:1,1:3,1) = 'N','N', 'P','P', 'D','D'
cbcvel(0:1,1:3,2) = 'N','N', 'P','P', 'D','D'
cbcvel(0:1,1:3,3) = 'N','N', 'P','P', 'D','D'
cbcpre(0:1,1:3)   = 'D','D', 'P','P', 'N','N'
bcpre(0:1,1:3)    = 1.5, -0.5, 0., 0., 0., 0.
gacc(1:3) = 0., 0., -0.98
/
&two_fluid
cbcpsi(0:1,1:3)   = 'N','N', 'P','P', 'N','N'
cbcnor(0:1,1:3,1) = 'D','D', 'P','P', 'N','N'
cbcnor(0:1,1:3,2) = 'N','N', 'P','P', 'N','N'
cbcnor(0:1,1:3,3) = 'N','N', 'P','P', 'D','D'
rho12(1:2) = 1000., 100.
mu12(1:2) = 10., 1.
sigma = 24.5
psi_thickness_factor = 0.51
/
"""


def test_updt_rhs_b_nonzero_dirichlet():
    """updt_rhs_b (src/bound.f90:341-396) with p = 1.5 and -0.5 on the two x
    faces: the boundary values enter the first and last interior planes
    of the right-hand side."""
    p = params.from_namelist(namelist.parse(_DIRICHLET))
    g, o = C.Case(p), O.Case(p)
    rng = np.random.default_rng(25)
    rhs = o.empty()
    rhs[1:-1, 1:-1, 1:-1] = rng.standard_normal(p.n)
    rhs0 = rhs.copy(order="F")
    rg = g.field(rhs)
    g.call("updt_rhs_b", rg)
    o.call("updt_rhs_b", rhs)
    a = rg.get()
    assert np.array_equal(a[1:-1, 1:-1, 1:-1], rhs[1:-1, 1:-1, 1:-1])
    # the x faces' values entered the first and last planes, nothing else moved
    assert not np.array_equal(a[1], rhs0[1]) and not np.array_equal(a[-2], rhs0[-2])
    assert np.array_equal(a[2:-2, 1:-1, 1:-1], rhs0[2:-2, 1:-1, 1:-1])


def test_step_dirichlet_pressure():
    """10 steps with a non-zero Dirichlet pressure BC in x: the step's
    fillps + updt_rhs_b + unfused solve path.  After one step the GPU
    matches the oracle to 1e-12.  Over ten steps the case amplifies
    round-off in the reference algorithm itself: far from the bubble psi
    lies within ~1e-12 of 1, where the SDF phi = eps*log((psi+e)/(1-psi+e))
    turns a one-ulp change of psi into a ~1e-4 change of phi, and through
    the normals and curvature into the velocity; moving psi by one ulp at
    random changes the oracle's own u, v, w by ~1e-6 after 10 steps (the
    GPU's FMA-rounded transport differs from the oracle by one ulp in some
    cells).  The bar is 1e-11 or four times that self-sensitivity."""
    p = params.from_namelist(namelist.parse(_DIRICHLET))
    psi = init.init2fl(p, "bub3", np.array([[0.5, 0.375, 0.5, 0.2]]))
    u, v, w, pr = init.initflow(p, "zer")
    g1, o1, rg, ro = _run_pair(p, u, v, w, pr, psi, 1)
    assert rg == 0 and ro == 0
    for nm in ("u", "v", "w", "p", "psi"):
        assert _rel(g1.get(nm), o1.get(nm)) < 1e-12, nm
    g, o, rg, ro = _run_pair(p, u, v, w, pr, psi, 10)
    assert rg == 0 and ro == 0
    sens = _oracle_sensitivity(p, u, v, w, pr, psi, 10, names=("u", "v", "w", "p"), mode="ulp")
    tol = max(1e-11, 4.0 * sens)
    errs = _check_step(g, o, tol=tol)
    # the Dirichlet BC fixes the pressure level: compare p itself as well
    pa, pb = g.get("p")[1:-1, 1:-1, 1:-1], o.get("p")[1:-1, 1:-1, 1:-1]
    assert _rel(pa, pb) < tol, (errs, sens)


def test_step_gravity_along_periodic_x():
    """10 steps with gravity components along periodic x and walled z: the
    step subtracts the mean density bulk_mean_12_stag(idir = 1) from the
    x buoyancy (src/main.f90:470-477)."""
    p = _nml(32, 24, 28, "PPPPNN", l=(1.0, 0.75, 1.0))
    p.gacc[:] = [-0.98, 0.0, -0.3]
    rng = np.random.default_rng(7)
    sph = init.place_droplets(rng, 5, 0.1, 0.15, [1, 0.75, 1], init.seps(p))
    psi = init.init2fl(p, "dis3", sph)
    u, v, w = init.divfree_velocity(p, rng, 3, 0.1)
    g, o, rg, ro = _run_pair(p, u, v, w, np.zeros_like(u), psi, 10)
    assert rg == 0 and ro == 0
    _check_step(g, o)


_WALLS = """
&dns
ng(1:3) = 20, 18, 16
l(1:3) = 1., 0.9, 0.8
gtype = 1, gr = 1.2
cbcvel(0:1,1:3,1) = 'D','D', 'D','N', 'D','D'
cbcvel(0:1,1:3,2) = 'N','D', 'D','D', 'N','D'
cbcvel(0:1,1:3,3) = 'D','N', 'N','D', 'D','D'
bcvel(0:1,1:3,1)  = 0.3, -0.2, 0.1, 0.05, 0., 0.7
bcvel(0:1,1:3,2)  = 0.2, 0.4, -0.1, 0.3, 0.6, -0.5
bcvel(0:1,1:3,3)  = 0.1, 0.25, 0.35, -0.45, 0.15, 0.
cbcpre(0:1,1:3)   = 'N','N', 'D','D', 'N','N'
bcpre(0:1,1:3)    = 0.5, -0.25, 1.5, -0.5, 0.75, 0.
/
&two_fluid
cbcpsi(0:1,1:3)   = 'N','D', 'D','N', 'N','N'
bcpsi(0:1,1:3)    = 0.1, 0.9, 0.2, 0.3, 0.4, 0.5
cbcnor(0:1,1:3,1) = 'D','D', 'N','N', 'N','N'
cbcnor(0:1,1:3,2) = 'N','N', 'D','D', 'N','N'
cbcnor(0:1,1:3,3) = 'N','N', 'N','N', 'D','D'
rho12(1:2) = 1000., 100.
mu12(1:2) = 10., 1.
/
"""


@pytest.mark.parametrize("text", [_DIRICHLET, _WALLS], ids=["x-walls", "all-walls"])
def test_boundary_fills_with_walls(text):
    """boundp for every field kind and bounduvw (after momentum and after
    correc) against the oracle, bit for bit, with walls in x (and y, z),
    centered and non-centered Dirichlet and Neumann faces with non-zero
    values, and periodic y: every ghost cell's value depends on the order of
    the fills (src/bound.f90:15-124), which the one-launch fill composes."""
    p = params.from_namelist(namelist.parse(text))
    g, o = C.Case(p), O.Case(p)
    rng = np.random.default_rng(31)
    shp = tuple(x + 2 for x in p.n)
    for which in range(6):
        a = np.asfortranarray(rng.standard_normal(shp))
        ag = g.field(a)
        g.call("boundp", which, ag)
        o.call("boundp", which, a)
        assert np.array_equal(ag.get(), a), which
    for is_correc in (0, 1):
        fs = [np.asfortranarray(rng.standard_normal(shp)) for _ in range(3)]
        gs = [g.field(a) for a in fs]
        g.call("bounduvw", is_correc, *gs)
        o.call("bounduvw", is_correc, *fs)
        for q, (a, b) in enumerate(zip(gs, fs)):
            assert np.array_equal(a.get(), b), (is_correc, q)
