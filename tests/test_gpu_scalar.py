"""The scalar transport (_SCALAR: rk_scal, src/rk.f90:133-191, with scal_ad,
src/scal.f90:13-66) and the Boussinesq buoyancy (_BOUSSINESQ_BUOYANCY,
src/mom.f90:1017-1024) on the GPU against the oracle:

* per procedure (scal_ad, rk_scal over two calls, mom_xyz_oth with the
  buoyancy term, boundp of cbcsca) on random fields, 1e-12 relative;
* whole steps: 10 steps of a two-fluid Rayleigh-Benard-like case (periodic
  x, y; the scalar Dirichlet below and Neumann above, a source term,
  unequal rho*cp, conductivities and expansion coefficients), a 2-D THINC
  case without buoyancy, and the reference's differentially heated cavity
  (tests/differentially_heated_cavity, fixture in tests/golden): 1e-11
  relative in u, v, w, p, psi and s, as the other FP64 steps; the mixed form
  within its 1e-6 bound;
* the differentially heated cavity run to the reference test's 50000 steps:
  the hot-wall Nusselt number within that test's tolerance of its
  acceptance value and close to the oracle's own 50000-step value;
* checkpoint files with the scalar, and a batched ensemble of scalar cases
  bit for bit equal to the cases' own runs.
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from cansfz import case as C
from cansfz import checkpoint as K
from cansfz import init, namelist, params

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _rb_params(nx=32, ny=24, nz=32, buoy=True, vof=False, form=0):
    """Periodic x, y; walls in z; gravity -z; the scalar held at 1 below and
    with a fixed gradient above; two fluids with different heat capacities."""
    lines = [
        "&dns", f"ng(1:3) = {nx}, {ny}, {nz}", f"l(1:3) = 1., {ny / nx}, 1.",
        "cfl = 0.5, dtmax = 1.e9, dt_f = -1., icheck = 5",
        "is_solve_ns = T, is_track_interface = T",
        "cbcvel(0:1,1:3,1) = 'P','P', 'P','P', 'D','D'",
        "cbcvel(0:1,1:3,2) = 'P','P', 'P','P', 'D','D'",
        "cbcvel(0:1,1:3,3) = 'P','P', 'P','P', 'D','D'",
        "cbcpre(0:1,1:3) = 'P','P', 'P','P', 'N','N'",
        "gacc(1:3) = 0., 0., -1.", "/",
        "&scalar", "cbcsca(0:1,1:3) = 'P','P', 'P','P', 'D','N'",
        "bcsca(0:1,1:3) = 0.,0., 0.,0., 1.,0.2", "ssource = 0.3", "/",
        "&two_fluid", "cbcpsi(0:1,1:3) = 'P','P', 'P','P', 'N','N'",
        "cbcnor(0:1,1:3,1) = 'P','P', 'P','P', 'N','N'",
        "cbcnor(0:1,1:3,2) = 'P','P', 'P','P', 'N','N'",
        "cbcnor(0:1,1:3,3) = 'P','P', 'P','P', 'D','D'",
        "rho12(1:2) = 2., 1.", "mu12(1:2) = 0.02, 0.01", "sigma = 0.05",
        "ka12(1:2) = 0.03, 0.01", "cp12(1:2) = 1.5, 1.", "beta12(1:2) = 0.5, 1.2",
        "psi_thickness_factor = 0.51", "/",
        "&cansfz", "scalar = T", f"boussinesq_buoyancy = {'T' if buoy else 'F'}",
        f"interface_capturing_vof = {'T' if vof else 'F'}", "/",
    ]
    p = params.from_namelist(namelist.parse("\n".join(lines)))
    p.form = form
    return p


def _rb_fields(p, seed=7):
    rng = np.random.default_rng(seed)
    eps = init.seps(p)
    sph = init.place_droplets(rng, 4, 0.1, 0.16, [p.l[0], p.l[1], p.l[2]], eps)
    psi = init.init2fl(p, "dis3", sph)
    u, v, w = init.divfree_velocity(p, rng, 3, 0.1)
    s = init.initscal(p, "cou")
    s[1:-1, 1:-1, 1:-1] += 0.05 * rng.standard_normal(p.n)
    return (u, v, w, np.zeros_like(u), psi), s


def _dhc_params():
    return params.from_namelist(namelist.read(os.path.join(GOLDEN, "dhc_case.nml")))


def _dhc_fields(p):
    nl = namelist.read(os.path.join(GOLDEN, "dhc_case.nml"))
    psi = init.init2fl(p, str(nl["inipsi"]))
    u, v, w, pr = init.initflow(p, str(nl["inivel"]))
    return (u, v, w, pr, psi), init.initscal(p, str(nl["inisca"]))


def _rel(a, b):
    s = np.abs(b).max()
    return np.abs(a - b).max() / (s if s > 0 else 1.0)


def _pair(p, f, s):
    g, o = C.Case(p), O.Case(p)
    g.set_fields(*f)
    g.set_scalar(s)
    for nm, a in zip(("u", "v", "w", "p", "psi"), f):
        o.set(nm, a)
    o.set("s", s)
    g.prepare()
    o.prepare()
    return g, o


def _check(g, o, tol):
    errs = {nm: _rel(g.get(nm), o.get(nm)) for nm in ("u", "v", "w", "psi", "s")}
    pa, pb = g.get("p")[1:-1, 1:-1, 1:-1], o.get("p")[1:-1, 1:-1, 1:-1]
    errs["p"] = _rel(pa - pa.mean(), pb - pb.mean())
    for k, e in errs.items():
        assert e < tol, f"{k}: rel err {e:.3e} ({errs})"
    dg, do = g.diag(), o.diag()
    assert dg.istep == do.istep and abs(dg.dt - do.dt) <= max(1e-13, tol) * do.dt
    return errs


# ---------------------------------------------------------------------------
# per procedure
# ---------------------------------------------------------------------------
@pytest.fixture(scope="module")
def small():
    p = _rb_params(24, 16, 20)
    return p, C.Case(p), O.Case(p)


def _rand(p, seed):
    rng = np.random.default_rng(seed)
    shp = tuple(x + 2 for x in p.n)
    f = lambda: np.asfortranarray(rng.standard_normal(shp))  # noqa: E731
    psi = np.asfortranarray(np.clip(0.5 + 0.45 * np.tanh(rng.standard_normal(shp)), 0, 1))
    return f, psi


def test_scal_ad_and_rk_scal(small):
    p, g, o = small
    f, psi = _rand(p, 1)
    u, v, w, fx, fy, fz, s = (f() for _ in range(7))
    psio = np.asfortranarray(np.clip(psi + 0.01 * f(), 0, 1))
    dev = {k: g.field(a) for k, a in dict(u=u, v=v, w=w, fx=fx, fy=fy, fz=fz, s=s, psi=psi, psio=psio).items()}
    dg = g.interior()
    do = np.zeros(p.n, order="F")
    g.call("scal_ad", dev["fx"], dev["fy"], dev["fz"], dev["psi"], dev["u"], dev["v"], dev["w"], dev["s"], dg)
    o.call("scal_ad", fx, fy, fz, psi, u, v, w, s, do)
    assert _rel(dg.get(), do) < 1e-13
    # rk_scal twice: the first call takes dsdtrko = dsdtrk, the second the history
    so = s.copy(order="F")
    for rkpar, dt in (([1.0, 0.0], 0.01), ([1.6, -0.6], 0.012)):
        g.call("rk_scal", rkpar, dt, dev["psi"], dev["u"], dev["v"], dev["w"], dev["psio"], dev["fx"], dev["fy"],
               dev["fz"], dev["s"])
        o.call("rk_scal", np.array(rkpar), dt, psi, u, v, w, psio, fx, fy, fz, so)
        a, b = dev["s"].get(), so
        assert _rel(a[1:-1, 1:-1, 1:-1], b[1:-1, 1:-1, 1:-1]) < 1e-13


def test_mom_xyz_oth_buoyancy(small):
    p, g, o = small
    f, psi = _rand(p, 2)
    pp, pn, po, kap, s = (f() for _ in range(5))
    dev = {k: g.field(a) for k, a in dict(p=pp, pn=pn, po=po, k=kap, s=s, psi=psi).items()}
    outg = [g.interior() for _ in range(3)]
    outo = [np.zeros(p.n, order="F") for _ in range(3)]
    rho_av = [0.0, 0.0, 0.0]
    g.call("mom_xyz_oth", 0.8, rho_av, dev["p"], dev["psi"], dev["k"], dev["s"], dev["pn"], dev["po"], *outg)
    o.call("mom_xyz_oth", 0.8, np.array(rho_av), pp, psi, kap, s, pn, po, *outo)
    for a, b in zip(outg, outo):
        assert _rel(a.get(), b) < 1e-12
    # the buoyancy term is there: without s the z component changes
    nob = [np.zeros(p.n, order="F") for _ in range(3)]
    o.call("mom_xyz_oth", 0.8, np.array(rho_av), pp, psi, kap, None, pn, po, *nob)
    assert _rel(nob[2], outo[2]) > 1e-3
    # a case with the buoyancy refuses a missing scalar
    with pytest.raises(Exception):
        g.call("mom_xyz_oth", 0.8, rho_av, dev["p"], dev["psi"], dev["k"], None, dev["pn"], dev["po"], *outg)


def test_boundp_scalar(small):
    p, g, o = small
    f, _ = _rand(p, 3)
    a = f()
    ag = g.field(a)
    g.call("boundp", 6, ag)
    o.call("boundp", 6, a)
    assert np.array_equal(ag.get(), a)


# ---------------------------------------------------------------------------
# whole steps
# ---------------------------------------------------------------------------
def test_step_rayleigh_benard_two_fluid():
    p = _rb_params()
    f, s = _rb_fields(p)
    g, o = _pair(p, f, s)
    assert g.step(10) == 0 and o.step(10) == 0
    _check(g, o, 1e-11)


def test_step_thinc_scalar_without_buoyancy_2d():
    p = _rb_params(64, 2, 48, buoy=False, vof=True)
    f, s = _rb_fields(p, seed=11)
    g, o = _pair(p, f, s)
    assert g.step(10) == 0 and o.step(10) == 0
    _check(g, o, 1e-11)


def test_step_dhc_reference_case():
    # the reference's differentially heated cavity, its first 10 steps
    p = _dhc_params()
    assert p.scalar == 1 and p.boussinesq == 1 and p.n == (128, 2, 128)
    f, s = _dhc_fields(p)
    g, o = _pair(p, f, s)
    assert g.step(10) == 0 and o.step(10) == 0
    _check(g, o, 1e-11)


def test_step_mixed_form():
    p = _rb_params(form=1)
    q = p.copy()
    q.form = 0
    f, s = _rb_fields(p)
    g = C.Case(p)
    g.set_fields(*f)
    g.set_scalar(s)
    g.prepare()
    o = O.Case(q)
    for nm, a in zip(("u", "v", "w", "p", "psi"), f):
        o.set(nm, a)
    o.set("s", s)
    o.prepare()
    assert g.step(10) == 0 and o.step(10) == 0
    _check(g, o, 1e-6)


def test_dhc_reference_acceptance():
    """tests/differentially_heated_cavity of the reference on the GPU: its
    50000 steps, then its Nusselt number of the hot wall (test.py) within its
    tolerance of its acceptance value, and within 1e-6 of the oracle's
    50000-step value recorded in the fixture."""
    gold = json.load(open(os.path.join(GOLDEN, "dhc_oracle.json")))
    p = _dhc_params()
    f, s = _dhc_fields(p)
    g = C.Case(p)
    g.set_fields(*f)
    g.set_scalar(s)
    g.prepare()
    nsteps = gold["steps"]
    assert g.step(500) == 0
    nu500 = _nusselt(g.get("s")[1:-1, 1:-1, 1:-1], p)
    assert abs(nu500 - gold["oracle"]["500"]["nusselt"]) <= 1e-9 * abs(gold["oracle"]["500"]["nusselt"])
    assert g.step(nsteps - 500) == 0
    d = g.diag()
    assert d.istep == nsteps
    nu = _nusselt(g.get("s")[1:-1, 1:-1, 1:-1], p)
    ref = gold["nusselt_reference"]
    assert abs(nu - ref) <= gold["atol"] + gold["rtol"] * abs(ref), (nu, ref)
    assert abs(nu - gold["oracle"][str(nsteps)]["nusselt"]) <= 1e-6 * abs(ref), (nu, gold["oracle"])
    assert abs(d.time - gold["oracle"][str(nsteps)]["time"]) <= 1e-9 * d.time


def _nusselt(s_interior, p):
    bc = np.array(p.bcsca[:]).reshape((2, 3), order="F")
    tw = bc[0, 0]
    xp0 = 0.5 * p.l[0] / p.ng[0]
    zp0 = 0.5 * p.l[2] / p.ng[2]
    return float((1.0 / p.l[0]) * np.sum((s_interior[0, 0, :] - tw) / (2.0 * xp0) * (2.0 * zp0)) * p.l[0] / (-tw))


# ---------------------------------------------------------------------------
# checkpoint and ensemble
# ---------------------------------------------------------------------------
def test_checkpoint_with_scalar(tmp_path):
    p = _rb_params(24, 16, 20)
    f, s = _rb_fields(p, seed=5)
    a = C.Case(p)
    a.set_fields(*f)
    a.set_scalar(s)
    a.prepare()
    assert a.step(6) == 0
    K.save(a, str(tmp_path), "fld")
    assert os.path.getsize(tmp_path / "fld_s.bin") == (np.prod(p.n) + 2) * 8
    b = C.Case(p)
    time, istep = K.restore(b, str(tmp_path), "fld")
    b.prepare()
    assert istep == 6
    for nm in ("u", "v", "w", "p", "psi", "s"):
        assert np.array_equal(a.get(nm)[1:-1, 1:-1, 1:-1], b.get(nm)[1:-1, 1:-1, 1:-1]), nm
    assert b.step(2) == 0


def test_ensemble_batched_scalar_cases():
    specs = []
    for seed, rho in ((1, 2.0), (2, 3.0), (3, 1.5)):
        p = _rb_params(32, 16, 24)
        p.rho12[0] = rho
        specs.append((p, _rb_fields(p, seed)))

    def build():
        out = []
        for p, (f, s) in specs:
            c = C.Case(p, own_stream=True)
            c.set_fields(*f)
            c.set_scalar(s)
            c.prepare()
            out.append(c)
        return out

    single = build()
    for c in single:
        assert c.step(7) == 0
    batch = build()
    ens = C.Ensemble(batch, batch=4)
    rc, st = ens.step(7)
    assert rc == 0 and st == [0, 0, 0]
    assert ens.groups() == (1, 3)
    for a, b in zip(single, batch):
        for nm in ("u", "v", "w", "p", "psi", "s"):
            assert np.array_equal(a.get(nm), b.get(nm)), nm
    ens.close()


def test_step_scalar_without_interface_tracking():
    # is_track_interface = F: the phase fluxes are zero and psi stays as set
    # (src/main.f90:453-458), so the scalar is advected by rho2*cp2*u only
    p = _rb_params(24, 16, 20)
    p.is_track_interface = 0
    f, s = _rb_fields(p, seed=13)
    g, o = _pair(p, f, s)
    assert g.step(10) == 0 and o.step(10) == 0
    _check(g, o, 1e-11)
