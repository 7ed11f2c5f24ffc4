"""Pins of the CPU oracle (oracle/cansfz_oracle.cpp) before it is trusted as
the parity checker of the CUDA path.

* FFTW r2r kinds restated vs scipy.fft (FFTW's published definitions).
* Known-answer tests built from the reference's own checks: the discrete
  Poisson residual (chk_poisson, src/debug.f90:81-114) and the projection
  test that the reference keeps disabled (src/sanity.f90:211-242).
* The reference's regression tests tests/rising_bubble and
  tests/lid_driven_cavity, run through the oracle with the reference's own
  input files and acceptance criteria (read from the reference checkout at
  test time; skipped where it is absent).
* tests/differentially_heated_cavity (the scalar with Boussinesq buoyancy):
  its 50000 steps take the oracle about five minutes, so the full run is
  recorded in tests/golden/dhc_oracle.json by tests/golden/make_dhc.py and
  checked there against the test's acceptance value; the default suite
  re-runs its first 500 steps against that record, and the full run repeats
  with CANSFZ_LONG_TESTS=1.
"""
import json
import os

import numpy as np
import pytest
import scipy.fft as sf
from scipy.spatial.distance import directed_hausdorff

import oracle as O
from cansfz import namelist, params

# FFTW kind numbers (src/fftw.f90:39-62)
R2HC, HC2R, REDFT01, REDFT10, REDFT11, RODFT01, RODFT10, RODFT11 = 0, 1, 4, 5, 6, 8, 9, 10
SMALL = np.finfo(np.float64).eps * 1e7   # src/param.f90:21


@pytest.mark.parametrize("n", [2, 4, 6, 12, 32, 48, 64, 96, 128, 256])
def test_r2r_kinds_vs_scipy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((5, n))
    X = np.fft.fft(x, axis=-1)
    hc = np.zeros_like(x)
    hc[:, : n // 2 + 1] = X[:, : n // 2 + 1].real
    for k in range(1, (n + 1) // 2):
        hc[:, n - k] = X[:, k].imag
    tol = 1e-13 * n
    assert np.abs(O.r2r(R2HC, x) - hc).max() <= tol * np.abs(hc).max()
    assert np.abs(O.r2r(HC2R, hc) - n * x).max() <= tol * n * np.abs(x).max()
    assert np.abs(O.r2r(REDFT10, x) - sf.dct(x, type=2)).max() <= tol
    assert np.abs(O.r2r(REDFT01, x) - sf.dct(x, type=3)).max() <= tol
    assert np.abs(O.r2r(RODFT10, x) - sf.dst(x, type=2)).max() <= tol
    assert np.abs(O.r2r(RODFT01, x) - sf.dst(x, type=3)).max() <= tol
    assert np.abs(O.r2r(REDFT11, x) - sf.dct(x, type=4)).max() <= tol
    assert np.abs(O.r2r(RODFT11, x) - sf.dst(x, type=4)).max() <= tol


def test_initgrid_uniform_and_stretched():
    nz, lz = 96, 2.0
    dzc, dzf, zc, zf = (np.zeros(nz + 2) for _ in range(4))
    O.lib().orc_initgrid(1, nz, 0.0, lz, *[O.ptr(a) for a in (dzc, dzf, zc, zf)])
    # z0 = (k-0.)/(1.*n) is a default-kind (single) quotient in the reference
    z0 = (np.arange(1, nz + 1, dtype=np.float32) / np.float32(nz)).astype(np.float64)
    assert np.array_equal(zf[1:nz + 1], z0 * lz)
    O.lib().orc_initgrid(1, nz, 1.5, lz, *[O.ptr(a) for a in (dzc, dzf, zc, zf)])
    assert abs(zf[nz] - lz) < 1e-14 and np.all(np.diff(zf[: nz + 1]) > 0)
    assert dzf[1] < dzf[nz // 2]  # clustered at the two walls


def _case(nx, ny, nz, cbcpre="PPPPNN", l=(1.0, 1.0, 1.0), gr=0.0):
    nl = namelist.defaults()
    nl.set("ng", np.array([nx, ny, nz]))
    nl.set("l", np.array(l, dtype=float))
    nl.set("gr", gr)
    cp = np.array(list(cbcpre), dtype=object).reshape((2, 3), order="F")
    nl.set("cbcpre", cp)
    cv = np.empty((2, 3, 3), dtype=object)
    for d in range(3):
        pp = cp[0, d] == "P"
        for ivel in range(3):
            cv[:, d, ivel] = "P" if pp else ("D" if ivel == d else ("D" if cp[0, d] == "N" else "N"))
    nl.set("cbcvel", cv)
    nl.set("cbcpsi", cp.copy())
    return O.Case(params.from_namelist(nl)), nl


def _laplacian(c, f):
    """7-point Laplacian of the reference (chk_poisson, src/debug.f90:100-106)."""
    g = c.grid()
    nx, ny, nz = c.n
    dxi, dyi = nx / c.params.l[0], ny / c.params.l[1]
    dzci, dzfi = g["dzci"], g["dzfi"]
    lap = np.zeros_like(f)
    ff = f
    lap[1:-1, 1:-1, 1:-1] = (
        (ff[2:, 1:-1, 1:-1] - 2 * ff[1:-1, 1:-1, 1:-1] + ff[:-2, 1:-1, 1:-1]) * dxi**2
        + (ff[1:-1, 2:, 1:-1] - 2 * ff[1:-1, 1:-1, 1:-1] + ff[1:-1, :-2, 1:-1]) * dyi**2
        + ((ff[1:-1, 1:-1, 2:] - ff[1:-1, 1:-1, 1:-1]) * dzci[None, None, 1:-1]
           - (ff[1:-1, 1:-1, 1:-1] - ff[1:-1, 1:-1, :-2]) * dzci[None, None, :-2]) * dzfi[None, None, 1:-1]
    )
    return lap


@pytest.mark.parametrize("cbcpre,gr", [("PPPPNN", 0.0), ("PPPPPP", 0.0), ("NNPPNN", 0.0),
                                        ("PPNNNN", 0.0), ("PPPPNN", 1.5), ("DDPPNN", 0.0)])
def test_poisson_known_answer(cbcpre, gr):
    """Solve lap(p) = lap(f) for a random f with the BC ghosts of cbcpre:
    the solution is f up to the constant of the all-Neumann/periodic null
    space; the residual is checked the way chk_poisson does."""
    c, _ = _case(24, 16, 20, cbcpre, l=(1.0, 0.75, 1.2), gr=gr)
    rng = np.random.default_rng(7)
    f = c.empty()
    f[1:-1, 1:-1, 1:-1] = rng.standard_normal(c.n)
    c.call("boundp", 0, f)
    rhs = _laplacian(c, f)
    p = rhs.copy(order="F")
    c.call("solver", p)
    c.call("boundp", 0, p)
    inner = (slice(1, -1),) * 3
    singular = "D" not in cbcpre
    e = p[inner] - f[inner]
    if singular:
        e = e - e.mean()
    assert np.abs(e).max() < 1e-10 * np.abs(f).max()
    res = np.abs(_laplacian(c, p)[inner] - rhs[inner]).max()
    assert res < 1e-9 * np.abs(rhs).max()


def test_projection_known_answer():
    """fillps -> solver -> correc leaves max|div| below `small`
    (the disabled test_sanity_solver, src/sanity.f90:211-242)."""
    c, _ = _case(32, 24, 16, "PPPPNN")
    rng = np.random.default_rng(11)
    u, v, w = (c.empty() for _ in range(3))
    for a in (u, v, w):
        a[1:-1, 1:-1, 1:-1] = rng.uniform(-0.5, 0.5, c.n)
    c.call("bounduvw", 0, u, v, w)
    d0t, d0m = np.zeros(1), np.zeros(1)
    c.call("chkdiv_fields", u, v, w, d0t, d0m)
    dt = np.pi
    p = c.empty()
    c.call("fillps", 1.0 / dt, u, v, w, p)
    c.call("updt_rhs_b", p)
    c.call("solver", p)
    c.call("boundp", 0, p)
    c.call("correc", dt, p, u, v, w)
    c.call("bounduvw", 1, u, v, w)
    divtot, divmax = np.zeros(1), np.zeros(1)
    c.call("chkdiv_fields", u, v, w, divtot, divmax)
    assert divmax[0] < SMALL
    assert divmax[0] < 1e-12 * d0m[0]  # round-off of the FP64 solve


def test_uniform_phase_known_answers():
    """psi = const: zero normals/curvature/phase RHS; u = 0: zero advection."""
    c, _ = _case(16, 16, 16, "PPPPNN")
    psi = c.empty() + 0.3
    phi = c.empty()
    c.call("acdi_cmpt_phi", c.seps, psi, phi)
    nx, ny, nz, kap = (c.empty() for _ in range(4))
    c.call("cmpt_norm_curv_youngs", phi, nx, ny, nz, kap)
    for a in (nx, ny, nz, kap):
        assert np.abs(a[1:-1, 1:-1, 1:-1]).max() == 0.0
    u, v, w = (c.empty() for _ in range(3))
    dpsidt = np.zeros(c.n, order="F")
    fx, fy, fz = (c.empty() for _ in range(3))
    c.call("acdi_transport_pf", 1.0, c.seps, u, v, w, nx, ny, nz, phi, psi, dpsidt, fx, fy, fz)
    assert np.abs(dpsidt).max() == 0.0


def _run_reference_case(case_dir):
    nl = namelist.read(os.path.join(case_dir, "input.nml"))
    conf = os.path.join(case_dir, "build.conf")
    if os.path.exists(conf):
        namelist.apply_build_conf(nl, conf)
    p = params.from_namelist(nl)
    c = O.Case(p)
    sph_file = os.path.join(case_dir, "spheres.in")
    sph = np.loadtxt(sph_file, ndmin=2) if os.path.exists(sph_file) else None
    c.init2fl(str(nl["inipsi"]), sph)
    c.initflow(str(nl["inivel"]))
    if p.scalar:
        c.initscal(str(nl["inisca"]))
    c.prepare()
    stop = nl["stop_type"]
    while True:
        rc = c.step(1)
        d = c.diag()
        assert rc == 0, f"oracle aborted with status {rc} at step {d.istep}"
        if (stop[0] and d.istep >= nl["nstep"]) or (stop[1] and d.time >= nl["time_max"]):
            break
    return c, nl, d


def _zero_level_points(f, xs, zs):
    """psi = 0.5 crossings on grid edges (the vertices matplotlib's contour
    puts on its path), linear interpolation."""
    g = f - 0.5
    pts = []
    for i in range(len(xs) - 1):
        s = g[i] * g[i + 1] < 0
        t = g[i][s] / (g[i][s] - g[i + 1][s])
        pts += list(zip(xs[i] + t * (xs[i + 1] - xs[i]), zs[s]))
    for k in range(len(zs) - 1):
        s = g[:, k] * g[:, k + 1] < 0
        t = g[s, k] / (g[s, k] - g[s, k + 1])
        pts += list(zip(xs[s], zs[k] + t * (zs[k + 1] - zs[k])))
    return np.array(pts)


@pytest.mark.slow
def test_reference_rising_bubble(reference_dir):
    """tests/rising_bubble of the reference: 2-D bubble, t = 3 (6000 steps);
    psi = 0.5 contour within directed Hausdorff distance 0.1 of the
    benchmark contour shipped with that test (its test.py criterion)."""
    case = os.path.join(reference_dir, "tests", "rising_bubble")
    c, nl, d = _run_reference_case(case)
    assert d.istep == 6000 and abs(d.time - 3.0) < 1e-9
    psi = c.get("psi")[1:-1, 1, 1:-1]
    nx = c.n[0]
    xs = (np.arange(nx) + 0.5) * c.params.l[0] / nx
    zs = c.grid()["zc"][1:-1]
    pts = _zero_level_points(psi, xs, zs)
    ref = np.loadtxt(os.path.join(case, "c1g2l3s.txt"))
    err = directed_hausdorff(pts, ref)[0]
    assert err < 1e-1
    assert err < 2e-2  # what this restatement achieves (0.0088)


@pytest.mark.slow
def test_reference_lid_driven_cavity(reference_dir):
    """tests/lid_driven_cavity of the reference (20000 steps): centre-line
    velocity profiles vs the tables shipped with that test, rtol/atol 0.1."""
    case = os.path.join(reference_dir, "tests", "lid_driven_cavity")
    c, nl, d = _run_reference_case(case)
    v = c.get("v")[1:-1, 1:-1, 1:-1]
    w = c.get("w")[1:-1, 1:-1, 1:-1]
    ny, nz = c.n[1], c.n[2]
    yp = (np.arange(ny) + 0.5) / ny * c.params.l[1]
    zp = c.grid()["zc"][1:-1]
    islice = nz // 2
    ref_u = np.loadtxt(os.path.join(case, "ghiau.txt"))
    data = v[0]
    interp = np.interp(ref_u[:, 0], zp, 0.5 * (data[islice, :] + data[islice + 1, :]))
    np.testing.assert_allclose(interp, ref_u[:, 1], rtol=1e-1, atol=1e-1)
    islice = ny // 2
    ref_v = np.loadtxt(os.path.join(case, "ghiav.txt"))
    data = w[0]
    interp = np.interp(ref_v[:, 0], yp, 0.5 * (data[:, islice] + data[:, islice + 1]))
    np.testing.assert_allclose(interp, ref_v[:, 1], rtol=1e-1, atol=1e-1)


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _dhc_nusselt(c):
    """The Nusselt number of tests/differentially_heated_cavity/test.py:9-13:
    (s - tw)/(2*xp(1)) * (2*zp(1)) summed over the hot wall's first column."""
    p = c.params
    s = c.get("s")[1:-1, 1:-1, 1:-1]
    tw = p.bcsca[0]
    xp0, zp0 = 0.5 * p.l[0] / p.ng[0], 0.5 * p.l[2] / p.ng[2]
    return float((1.0 / p.l[0]) * np.sum((s[0, 0, :] - tw) / (2.0 * xp0) * (2.0 * zp0)) * p.l[0] / (-tw))


def test_dhc_record_and_first_steps():
    """The recorded 50000-step oracle run meets the reference test's
    acceptance value; the oracle still reproduces the record's 500th step."""
    gold = json.load(open(os.path.join(GOLDEN, "dhc_oracle.json")))
    nu = gold["oracle"][str(gold["steps"])]["nusselt"]
    ref = gold["nusselt_reference"]
    assert abs(nu - ref) <= gold["atol"] + gold["rtol"] * abs(ref)
    nl = namelist.read(os.path.join(GOLDEN, "dhc_case.nml"))
    p = params.from_namelist(nl)
    c = O.Case(p)
    c.init2fl(str(nl["inipsi"]))
    c.initflow(str(nl["inivel"]))
    c.initscal(str(nl["inisca"]))
    c.prepare()
    assert c.step(500) == 0
    rec = gold["oracle"]["500"]
    assert abs(_dhc_nusselt(c) - rec["nusselt"]) <= 1e-12 * abs(rec["nusselt"])
    assert c.diag().time == rec["time"]


def test_dhc_fixture_is_the_reference_input(reference_dir):
    case = os.path.join(reference_dir, "tests", "differentially_heated_cavity")
    nl = namelist.read(os.path.join(case, "input.nml"))
    namelist.apply_build_conf(nl, os.path.join(case, "build.conf"))
    a = params.from_namelist(nl)
    b = params.from_namelist(namelist.read(os.path.join(GOLDEN, "dhc_case.nml")))
    assert bytes(a) == bytes(b)


@pytest.mark.slow
@pytest.mark.skipif(not os.environ.get("CANSFZ_LONG_TESTS"), reason="five minutes of oracle steps; the record "
                    "in tests/golden/dhc_oracle.json holds this run (CANSFZ_LONG_TESTS=1 repeats it)")
def test_reference_differentially_heated_cavity(reference_dir):
    """tests/differentially_heated_cavity of the reference (50000 steps,
    _SCALAR and _BOUSSINESQ_BUOYANCY from its build.conf): the hot wall's
    Nusselt number vs the acceptance value of its test.py, rtol = atol = 1e-2."""
    import re

    case = os.path.join(reference_dir, "tests", "differentially_heated_cavity")
    c, nl, d = _run_reference_case(case)
    assert d.istep == int(nl["nstep"])
    txt = open(os.path.join(case, "test.py")).read()
    ref = float(re.search(r"nusselt_ref\s*=\s*([0-9.eE+-]+)", txt).group(1))
    np.testing.assert_allclose([_dhc_nusselt(c)], [ref], rtol=1e-2, atol=1e-2)


def test_balanced_split_known_answers():
    """_BALANCED_CAPILLARY_PRESSURE_SPLIT (src/mom.f90:982-1032): without
    surface tension the split moves nothing (the same step bit for bit);
    with it, the surf?_n arrays hold the last step's force and surf?_o the
    one before, and the step differs from the unsplit one."""
    from cansfz import workloads as W

    for sigma in (0.0, 1.0):
        runs = []
        for bal in (0, 1):
            p, f = W.droplets((16, 16, 16), (1.0, 1.0, 1.0), False, count=2, rmin=0.15, rmax=0.2, seed=3)
            p.sigma = sigma
            p.balanced = bal
            c = O.Case(p)
            for nm, a in zip(("u", "v", "w", "p", "psi"), f):
                c.set(nm, a)
            c.prepare()
            assert c.step(4) == 0
            runs.append(c)
        same = all(np.array_equal(runs[0].get(nm), runs[1].get(nm)) for nm in ("u", "v", "w", "p", "psi"))
        assert same == (sigma == 0.0)
        if sigma > 0:
            b = runs[1]
            assert np.abs(b.get("surfz_n")).max() > 0 and np.abs(b.get("surfz_o")).max() > 0
            assert not np.array_equal(b.get("surfz_n"), b.get("surfz_o"))
