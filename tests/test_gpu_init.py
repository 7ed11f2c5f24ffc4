"""Initial conditions computed on the device (cansfz_init2fl, _initflow,
_initscal) against the oracle's restatement of init2fl
(src/two_fluid.f90:247-437), initflow (src/initflow.f90:16-361) and
initscal (:363-429): every name, spheres across periodic boundaries, the
default sphere, the film; then a case initialised on the device steps as
the oracle's case initialised on the host (1e-11 after 10 steps).  The
device's tanh and sqrt differ from the host's by an ulp, hence 1e-15."""
import numpy as np
import pytest

import oracle as O
from cansfz import case as C
from cansfz import init, namelist, params

pytestmark = pytest.mark.gpu


def _params(n=(40, 32, 36), cbc="PPPPNN", l=(1.0, 0.8, 0.9), gr=0.0, scalar=False):
    nl = namelist.defaults()
    nl.set("ng", np.array(n))
    nl.set("l", np.array(l))
    nl.set("gr", gr)
    cp = np.array(list(cbc), dtype=object).reshape((2, 3), order="F")
    nl.set("cbcpre", cp)
    nl.set("cbcpsi", cp.copy())
    p = params.from_namelist(nl)
    if scalar:
        p.scalar = 1
        p.bcsca[:] = [-0.5, 0.5, 0.0, 0.0, 0.25, 0.75]
    return p


SPHERES = np.array([[0.02, 0.4, 0.45, 0.12],    # across the periodic x boundary
                    [0.5, 0.78, 0.3, 0.1],      # across the periodic y boundary
                    [0.7, 0.2, 0.6, 0.15],
                    [0.3, 0.3, 0.2, 0.08]])


@pytest.mark.parametrize("name", ["bub3", "drp3", "dis3", "bub2", "dis2", "bub1", "drp1", "flm", "uni", "zer"])
@pytest.mark.parametrize("default_sphere", [False, True])
def test_init2fl(name, default_sphere):
    p = _params(gr=1.2)
    sph = None if default_sphere else SPHERES
    g, o = C.Case(p), O.Case(p)
    g.init2fl(name, sph)
    o.init2fl(name, sph)
    a, b = g.get("psi"), o.get("psi")
    assert np.abs(a - b).max() <= 1e-15, name
    assert np.abs(a - init.init2fl(p, name, sph)).max() <= 1e-15, name


@pytest.mark.parametrize("name", ["zer", "uni", "cou", "poi", "voy", "vox"])
def test_initflow(name):
    p = _params(gr=1.3)
    p.bcvel[4:6] = [0.3, -0.7]  # bcvel(0:1,3,1): the Couette wall velocities
    g, o = C.Case(p), O.Case(p)
    g.set_time(0.37, 0)
    g.initflow(name)
    o.initflow(name, 0.37)
    for nm in ("u", "v", "w", "p"):
        a, b = g.get(nm), o.get(nm)
        assert np.abs(a - b)[1:-1, 1:-1, 1:-1].max() <= 1e-14 * max(1.0, np.abs(b).max()), (name, nm)


@pytest.mark.parametrize("name", ["zer", "uni", "cou", "dhc"])
def test_initscal(name):
    p = _params(cbc="NNPPNN", scalar=True)
    g, o = C.Case(p), O.Case(p)
    g.initscal(name)
    o.initscal(name)
    assert np.array_equal(g.get("s")[1:-1, 1:-1, 1:-1], o.get("s")[1:-1, 1:-1, 1:-1]), name


def test_unknown_names_refused():
    p = _params()
    g = C.Case(p)
    for call in (lambda: g.init2fl("xyz"), lambda: g.initflow("xyz"), lambda: g.initscal("cou")):
        with pytest.raises(Exception):
            call()


def test_device_init_then_steps():
    p = _params((32, 32, 32), l=(1.0, 1.0, 1.0))
    p.rho12[:] = [10.0, 1.0]
    p.mu12[:] = [0.05, 0.01]
    p.sigma = 0.5
    p.gacc[:] = [0.0, 0.0, -1.0]
    g, o = C.Case(p), O.Case(p)
    g.init2fl("dis3", SPHERES[2:])
    g.initflow("zer")
    o.init2fl("dis3", SPHERES[2:])
    o.initflow("zer")
    g.prepare()
    o.prepare()
    assert g.step(10) == 0 and o.step(10) == 0
    for nm in ("u", "v", "w", "psi"):
        a, b = g.get(nm), o.get(nm)
        assert np.abs(a - b).max() <= 1e-11 * np.abs(b).max(), nm
