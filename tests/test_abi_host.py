"""CPU checks of the boundary and the host logic: the C-ABI library loads and
exports every entry point declared in include/cansfz.h, the params layout
matches the C struct, the namelist reader, and the host-side initial
conditions against the oracle's restatement of init2fl/initflow."""
import ctypes as ct
import os
import re
import subprocess

import numpy as np

import oracle as O
from cansfz import init, lib, namelist, params

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "cansfz.h")).read()
    return sorted(set(re.findall(r"\b(cansfz_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = lib.load()
    names = _declared()
    assert len(names) > 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # every declared entry has a ctypes signature in the host binding
    assert set(names) <= set(lib.SIGNATURES)


def _c_layout(tmp_path, struct, fields):
    """sizeof and offsetof of the header's struct, from a C program built
    against include/cansfz.h."""
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "cansfz.h"', "int main(void) {",
             f'  printf("%zu\\n", sizeof({struct}));']
    lines += [f'  printf("%zu\\n", offsetof({struct}, {f}));' for f in fields]
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    return [int(x) for x in out]


def test_params_layout_matches_c(tmp_path):
    for cls, struct in ((params.Params, "cansfz_params"), (lib.Diag, "cansfz_diag"), (lib.Plan, "cansfz_plan")):
        names = [f[0] for f in cls._fields_]
        got = _c_layout(tmp_path, struct, names)
        assert got[0] == ct.sizeof(cls), struct
        assert got[1:] == [getattr(cls, n).offset for n in names], struct


def test_status_strings_and_no_device_error():
    L = lib.load()
    assert L.cansfz_version() >= 100
    assert b"divergence" in L.cansfz_status_string(5)
    out = ct.c_void_p()
    p = params.from_namelist(namelist.defaults())
    rc = L.cansfz_create(ct.byref(p), None, ct.byref(out))
    import torch

    if not torch.cuda.is_available():
        assert rc == 9  # CANSFZ_ERR_NOT_FOUND: no silent CPU path
        assert not out.value


def test_namelist_reference_inputs(reference_dir):
    for case in ("rising_bubble", "lid_driven_cavity", "deforming_circle"):
        nl = namelist.read(os.path.join(reference_dir, "tests", case, "input.nml"))
        p = params.from_namelist(nl)
        assert all(x > 0 for x in p.n)
    nl = namelist.read(os.path.join(reference_dir, "tests", "rising_bubble", "input.nml"))
    assert list(nl["ng"]) == [64, 2, 128]
    assert nl["cbcvel"][0, 0, 0] == "D" and nl["cbcvel"][0, 1, 0] == "P"
    assert nl["cbcpre"][:, 0].tolist() == ["N", "N"]
    assert nl["stop_type"].tolist() == [True, True, False]
    assert nl["inipsi"] == "bub2"


def test_namelist_defaults_single_precision_literals():
    nl = namelist.defaults()
    assert nl["cfl"] == float(np.float32(0.95))
    assert nl["acdi_gam_min"] == float(np.float32(1e-12))


def test_namelist_roundtrip():
    nl = namelist.defaults()
    nl.set("ng", np.array([10, 12, 14]))
    nl2 = namelist.parse(namelist.write(nl))
    assert list(nl2["ng"]) == [10, 12, 14]


def _case_params(nx, ny, nz, cbc="PPPPNN", l=(1.0, 1.0, 1.0), gr=0.0):
    nl = namelist.defaults()
    nl.set("ng", np.array([nx, ny, nz]))
    nl.set("l", np.array(l))
    nl.set("gr", gr)
    cp = np.array(list(cbc), dtype=object).reshape((2, 3), order="F")
    nl.set("cbcpre", cp)
    nl.set("cbcpsi", cp.copy())
    return params.from_namelist(nl)


def test_initgrid_matches_oracle():
    for gtype, gr in ((1, 0.0), (1, 1.5), (2, 1.2), (3, 0.8), (4, 2.0)):
        p = _case_params(8, 8, 48, gr=gr)
        p.gtype = gtype
        g = init.zgrid(p)
        o = O.Case(p).grid()
        for k in ("dzc", "dzf", "zc", "zf"):
            assert np.array_equal(g[k], o[k]), (gtype, k)


def test_init2fl_matches_oracle():
    p = _case_params(32, 24, 40, "PPPPNN", l=(1.0, 0.75, 1.25))
    rng = np.random.default_rng(0)
    eps = init.seps(p)
    sph = init.place_droplets(rng, 5, 0.08, 0.14, [1.0, 0.75, 1.25], eps)
    for name in ("bub3", "dis3", "bub2", "drp2", "bub1", "flm", "uni"):
        a = init.init2fl(p, name, sph)
        c = O.Case(p)
        c.init2fl(name, sph)
        b = c.get("psi")
        assert np.abs(a - b)[1:-1, 1:-1, 1:-1].max() <= 1e-15, name


def test_initflow_matches_oracle():
    p = _case_params(16, 12, 24, "PPPPNN", l=(1.0, 1.0, 2.0), gr=1.2)
    for name in ("zer", "uni", "poi", "voy", "vox"):
        u, v, w, pr = init.initflow(p, name, 0.37)
        c = O.Case(p)
        c.initflow(name, 0.37)
        for a, nm in zip((u, v, w), ("u", "v", "w")):
            # set_mean sums in a different order: round-off only
            assert np.abs(a - c.get(nm))[1:-1, 1:-1, 1:-1].max() <= 1e-14, (name, nm)


def test_divfree_velocity_is_discretely_solenoidal():
    p = _case_params(24, 20, 16, "PPPPNN", gr=1.3)
    u, v, w = init.divfree_velocity(p, np.random.default_rng(1), 4, 0.1)
    c = O.Case(p)
    c.call("bounduvw", 0, u, v, w)
    t, m = np.zeros(1), np.zeros(1)
    c.call("chkdiv_fields", u, v, w, t, m)
    rms = np.sqrt(np.mean(u[1:-1, 1:-1, 1:-1] ** 2))
    assert 0.05 < rms < 0.2
    assert m[0] < 1e-12


def test_initscal_matches_oracle():
    p = _case_params(16, 6, 20, "NNPPNN", l=(1.0, 0.5, 1.5), gr=1.1)
    p.scalar = 1
    p.bcsca[:] = [-0.5, 0.5, 0.0, 0.0, 0.25, 0.75]
    for name in ("zer", "uni", "cou", "dhc"):
        a = init.initscal(p, name)
        c = O.Case(p)
        c.initscal(name)
        assert np.array_equal(a[1:-1, 1:-1, 1:-1], c.get("s")[1:-1, 1:-1, 1:-1]), name
    # 'dhc' is the x profile between the x boundary values, centred cells
    s = init.initscal(p, "dhc")[1:-1, 1, 1]
    assert np.allclose(s, -0.5 + (np.arange(16) + 0.5) / 16)
    try:
        init.initscal(p, "xyz")
        raise AssertionError("invalid name accepted")
    except ValueError:
        pass


def test_build_conf_switches(reference_dir, tmp_path):
    # the reference's differentially heated cavity builds with _SCALAR and
    # _BOUSSINESQ_BUOYANCY; its &scalar group and ka12/cp12 fill the params
    case = os.path.join(reference_dir, "tests", "differentially_heated_cavity")
    nl = namelist.read(os.path.join(case, "input.nml"))
    namelist.apply_build_conf(nl, os.path.join(case, "build.conf"))
    p = params.from_namelist(nl)
    assert p.scalar == 1 and p.boussinesq == 1 and p.interface_capturing == params.ACDI
    assert bytes(p.cbcsca) == b"DDPPNN" and list(p.bcsca)[:2] == [-0.5, 0.5]
    assert nl["inisca"] == "dhc" and p.ka12[0] == p.ka12[1] > 0 and list(p.cp12) == [1.0, 1.0]
    # _BOUSSINESQ_BUOYANCY without _SCALAR has no effect, as in the reference
    conf = tmp_path / "build.conf"
    conf.write_text("SCALAR=0   # off\nBOUSSINESQ_BUOYANCY=1\nINTERFACE_CAPTURING_VOF=1\nSDF_NORMALS=0\n")
    nl = namelist.apply_build_conf(namelist.defaults(), str(conf))
    p = params.from_namelist(nl)
    assert p.scalar == 0 and p.boussinesq == 0 and p.interface_capturing == params.VOF_THINC
    assert p.sdf_normals == 0 and p.brackbill == 1  # absent: flags.mk's default 1
    for bad in ("CONSTANT_COEFFS_POISSON=0\n", "SINGLE_PRECISION=1\n"):
        conf.write_text(bad)
        try:
            namelist.apply_build_conf(namelist.defaults(), str(conf))
            raise AssertionError(bad)
        except ValueError:
            pass


def test_read_spheres(reference_dir, tmp_path):
    found = 0
    for root in ("tests", "examples"):
        for dirpath, _, files in os.walk(os.path.join(reference_dir, root)):
            if "spheres.in" in files:
                path = os.path.join(dirpath, "spheres.in")
                a = init.read_spheres(path)
                assert a.shape[1] == 4 and np.allclose(a, np.loadtxt(path, ndmin=2)[:, :4], rtol=0, atol=0)
                found += 1
    assert found > 0
    assert init.read_spheres(str(tmp_path / "none.in")).shape == (0, 4)


def test_xform_matrices_match_the_r2r_kinds():
    """The dense matrices of the FP32 solve's tensor-core transforms against
    the oracle's restatement of FFTW's kinds (R2HC/HC2R in the packed order
    (r0, r_{n/2}, r1, i1, ...), REDFT10/01, RODFT10/01)."""
    L = lib.load()
    R2HC, HC2R, REDFT01, REDFT10, RODFT01, RODFT10 = 0, 1, 4, 5, 8, 9
    rng = np.random.default_rng(11)
    for n in (64, 128, 256, 96):
        x = rng.standard_normal((3, n))

        def mat(kind, d):
            F = np.zeros(n * n)
            assert L.cansfz_xform_matrix(kind, d, n, F.ctypes.data_as(lib.PD)) == 0
            return F.reshape(n, n)

        # periodic: FFTW's half-complex order -> the packed order
        hc = O.r2r(R2HC, x)
        h = n // 2
        packed = np.zeros_like(hc)
        packed[:, 0], packed[:, 1] = hc[:, 0], hc[:, h]
        for k in range(1, h):
            packed[:, 2 * k], packed[:, 2 * k + 1] = hc[:, k], hc[:, n - k]
        tol = 1e-12 * n
        assert np.abs(x @ mat(0, 1).T - packed).max() <= tol * np.abs(packed).max()
        assert np.abs(packed @ mat(0, -1).T - O.r2r(HC2R, hc)).max() <= tol * n * np.abs(x).max()
        for kind, fw, bw in ((1, REDFT10, REDFT01), (2, RODFT10, RODFT01)):
            assert np.abs(x @ mat(kind, 1).T - O.r2r(fw, x)).max() <= tol * np.abs(O.r2r(fw, x)).max()
            assert np.abs(x @ mat(kind, -1).T - O.r2r(bw, x)).max() <= tol * np.abs(O.r2r(bw, x)).max()
