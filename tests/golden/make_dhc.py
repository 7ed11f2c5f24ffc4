"""Writes the differentially-heated-cavity fixtures from the reference's own
regression test (tests/differentially_heated_cavity: input.nml, build.conf
and the acceptance value in test.py), so that the GPU box, which has no
reference checkout, can run that test against the library:

* dhc_case.nml -- the test's parameters as this library's namelist reader
  sees them (every variable, rendered by cansfz.namelist.write), with the
  build.conf switches (_SCALAR, _BOUSSINESQ_BUOYANCY) in &cansfz;
* dhc_oracle.json -- the oracle's run of that case: the Nusselt number of
  the hot wall after 500 steps and after the test's 50000 steps, computed as
  the test computes it, and the test's acceptance value and tolerances.

Run from the repository root:  python tests/golden/make_dhc.py
(about five minutes: 50000 oracle steps on 128 x 2 x 128 cells).
"""
import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "cans-fizzy_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from cansfz import namelist, params  # noqa: E402

# the reference's test case directory (reference checkout from
# CANSFZ_REFERENCE_DIR, default the build container's read-only copy)
CASE = os.path.join(os.environ.get("CANSFZ_REFERENCE_DIR", "/root/reference"), "tests",
                    "differentially_heated_cavity")


def nusselt(s_interior, p):
    """The test's Nusselt number (test.py:9-13): hot-wall gradient of the
    first cell column, (s - tw)/(2*xp(1)) * (2*zp(1)), summed over z."""
    bc = np.array(p.bcsca[:]).reshape((2, 3), order="F")
    tw = bc[0, 0]
    lx = p.l[0]
    xp0 = 0.5 * p.l[0] / p.ng[0]
    zp0 = 0.5 * p.l[2] / p.ng[2]
    col = s_interior[0, 0, :]
    return float((1.0 / lx) * np.sum((col - tw) / (2.0 * xp0) * (2.0 * zp0)) * lx / (-tw))


def run(p, nl, steps):
    c = O.Case(p)
    c.init2fl(str(nl["inipsi"]))
    c.initflow(str(nl["inivel"]))
    c.initscal(str(nl["inisca"]))
    c.prepare()
    out = {}
    done = 0
    for k in steps:
        rc = c.step(k - done)
        assert rc == 0, rc
        done = k
        d = c.diag()
        out[k] = {"nusselt": nusselt(c.get("s")[1:-1, 1:-1, 1:-1], p), "time": d.time, "dt": d.dt}
    return out


def main():
    nl = namelist.read(os.path.join(CASE, "input.nml"))
    namelist.apply_build_conf(nl, os.path.join(CASE, "build.conf"))
    with open(os.path.join(HERE, "dhc_case.nml"), "w") as f:
        f.write("! tests/differentially_heated_cavity of the reference (input.nml + build.conf),\n")
        f.write("! rendered by tests/golden/make_dhc.py\n")
        f.write(namelist.write(nl))
    test_py = open(os.path.join(CASE, "test.py")).read()
    ref = float(re.search(r"nusselt_ref\s*=\s*([0-9.eE+-]+)", test_py).group(1))
    tol = re.search(r"assert_allclose\(\[nusselt\],\s*\[nusselt_ref\],\s*rtol=([0-9.eE+-]+),\s*atol=([0-9.eE+-]+)\)",
                    test_py)
    p = params.from_namelist(namelist.read(os.path.join(HERE, "dhc_case.nml")))
    nsteps = int(nl["nstep"])
    res = run(p, nl, [500, nsteps])
    data = {"steps": nsteps, "nusselt_reference": ref, "rtol": float(tol.group(1)), "atol": float(tol.group(2)),
            "oracle": {str(k): v for k, v in res.items()}}
    with open(os.path.join(HERE, "dhc_oracle.json"), "w") as f:
        json.dump(data, f, indent=1)
    print(json.dumps(data, indent=1))


if __name__ == "__main__":
    main()
