"""Checkpoint files in the reference's restart format (load_one,
src/load.f90:13-170): layout, size check and round trips.  The format tests
run on the CPU; the round trip through a GPU case is marked gpu."""
import os

import numpy as np
import pytest

from cansfz import checkpoint as K


def test_layout_is_the_reference_one(tmp_path):
    ng = (6, 4, 5)
    rng = np.random.default_rng(1)
    a = rng.standard_normal(ng)
    K.write_field(str(tmp_path / "fld_u.bin"), a, 1.25, 37)
    raw = np.fromfile(tmp_path / "fld_u.bin", dtype=np.float64)
    # interior in Fortran order (x fastest), then [time, istep]
    assert raw.size == a.size + 2
    assert np.array_equal(raw[:-2], a.reshape(-1, order="F"))
    assert raw[-2] == 1.25 and raw[-1] == 37.0
    assert os.path.getsize(tmp_path / "fld_u.bin") == (np.prod(ng) + 2) * 8


def test_round_trip_and_size_check(tmp_path):
    ng = (8, 6, 4)
    rng = np.random.default_rng(2)
    halo = [rng.standard_normal(tuple(n + 2 for n in ng)) for _ in range(5)]
    K.save_fields(str(tmp_path), "fld", halo, 0.5, 12)
    back, time, istep = K.load_fields(str(tmp_path), ng)
    assert time == 0.5 and istep == 12
    for a, b in zip(halo, back):
        assert np.array_equal(a[1:-1, 1:-1, 1:-1], b[1:-1, 1:-1, 1:-1])
        assert not b[0].any() and not b[-1].any()
    # a file of the wrong size is refused, as the reference aborts on it
    with open(tmp_path / "fld_p.bin", "ab") as f:
        f.write(b"\0" * 8)
    with pytest.raises(K.CheckpointError):
        K.load_fields(str(tmp_path), ng)


@pytest.mark.gpu
def test_gpu_case_save_restore(tmp_path):
    from cansfz import case as C
    from cansfz import workloads as W

    p, f = W.droplets((32, 32, 32), (1.0, 1.0, 1.0), False, count=4, rmin=0.1, rmax=0.15, seed=5)
    a = C.Case(p)
    a.set_fields(*f)
    a.prepare()
    assert a.step(7) == 0
    t = K.save(a, str(tmp_path), "fld", background=True)
    t.join()
    b = C.Case(p)
    time, istep = K.restore(b, str(tmp_path), "fld")
    b.prepare()
    assert istep == 7 and time == a.diag().time
    for nm in ("u", "v", "w", "p", "psi"):
        assert np.array_equal(a.get(nm)[1:-1, 1:-1, 1:-1], b.get(nm)[1:-1, 1:-1, 1:-1]), nm
    d = b.diag()
    assert d.istep == 7 and d.time == time
    # the restarted case takes an Euler first step (no AB2 history in the
    # files, as in the reference); it must step on from the restored count
    assert b.step(3) == 0 and b.diag().istep == 10


@pytest.mark.gpu
def test_gpu_status_is_diag_without_masses():
    # cansfz_get_status: the per-step scalars of cansfz_get_diag, no mass reduction
    from cansfz import case as C
    from cansfz import workloads as W

    p, f = W.droplets((32, 32, 32), (1.0, 1.0, 1.0), False, count=3, rmin=0.1, rmax=0.15, seed=7)
    a = C.Case(p)
    a.set_fields(*f)
    a.prepare()
    assert a.step(11) == 0  # past an icheck step: dt and divergence updated
    s, d = a.status(), a.diag()
    for nm in ("time", "istep", "dt", "dto", "dt_cfl", "gam", "seps", "divtot", "divmax", "status"):
        assert getattr(s, nm) == getattr(d, nm), nm
    assert np.isnan(s.mass12[0]) and np.isnan(s.mass12[1])
    assert d.mass12[0] > 0 and d.mass12[1] > 0
