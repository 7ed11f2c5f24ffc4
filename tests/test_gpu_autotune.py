"""The launch plans and their autotuner (cansfz_get_plan / cansfz_set_plan /
cansfz_autotune), through the C ABI.

* The tile kernels' z split is a launch shape only: steps with other splits
  are bit-equal.  The z-solve variant changes the elimination order
  (round-off), the y-transform variant the FFT factorisation (round-off),
  the FP32 solve's transforms change the FP32 result before refinement; all
  stay within the FP64 whole-step bar.
* The autotuner times on a copy: the case itself neither advances nor
  changes.  Its choice is written to the cache file and read back, without
  timing, by the next case with the same key.
"""
import numpy as np
import pytest

from cansfz import case as C
from cansfz import lib, workloads

pytestmark = pytest.mark.gpu


def _case(n=(32, 32, 64), **kw):
    p, f = workloads.droplets(n, (1.0, 1.0, 1.0), False, count=6, rmin=0.1, rmax=0.15, seed=3)
    for k, v in kw.items():
        setattr(p, k, v)
    g = C.Case(p)
    g.set_fields(*f)
    g.prepare()
    return g


def _state(g):
    return [g.get(nm) for nm in ("u", "v", "w", "p", "psi")]


def test_tile_splits_are_bit_equal():
    # 256 x 256 x 64: the default split gives blocks of 8 levels, one slot
    # per SM gives blocks of 64
    a, b = _case((256, 256, 64)), _case((256, 256, 64))
    q = b.plan()
    q.phase_slots, q.momentum_slots = 1, 1
    b.set_plan(q)
    assert a.step(6) == 0 and b.step(6) == 0
    for x, y in zip(_state(a), _state(b)):
        assert np.array_equal(x, y)


_AUX = ("phi", "kappa", "normx", "normy", "normz", "psiflx_x", "psiflx_y", "psiflx_z", "pn", "po", "pcorr")


@pytest.mark.parametrize("kind", ["walls-z", "periodic", "mixed", "thinc"])
def test_ghost_images_are_bit_equal(kind):
    """The producing kernels' periodic ghost images (ghost_images = 1) and
    the fill stages (0) leave the same bits in every field, ghosts included."""
    kw = {}
    if kind == "mixed":
        kw["form"] = 1
    if kind == "thinc":
        kw["interface_capturing"] = 1
    if kind == "periodic":
        kw.update(cbcvel=b"P" * 18, cbcpre=b"P" * 6, cbcpsi=b"P" * 6, cbcnor=b"P" * 18)
    a, b = _case((64, 32, 48), **kw), _case((64, 32, 48), **kw)
    q = b.plan()
    assert q.ghost_images == 1
    q.ghost_images = 0
    b.set_plan(q)
    assert a.step(5) == 0 and b.step(5) == 0
    for nm, x, y in zip(("u", "v", "w", "p", "psi"), _state(a), _state(b)):
        assert np.array_equal(x, y), nm
    for nm in _AUX:
        assert np.array_equal(a.get(nm), b.get(nm)), nm


def test_zsolve_variants_agree():
    # 256 x 128 columns: the partitioned z solve applies (nz = 64 = 8 x 8)
    a, b = _case((256, 128, 64)), _case((256, 128, 64))
    q = b.plan()
    assert q.zsolve == 0
    q.zsolve = 1
    b.set_plan(q)
    assert a.step(5) == 0 and b.step(5) == 0
    for nm, x, y in zip(("u", "v", "w", "p", "psi"), _state(a), _state(b)):
        if nm == "p":
            x, y = x[1:-1, 1:-1, 1:-1] - x[1:-1, 1:-1, 1:-1].mean(), y[1:-1, 1:-1, 1:-1] - y[1:-1, 1:-1, 1:-1].mean()
        assert np.abs(x - y).max() <= 1e-11 * np.abs(y).max(), nm


@pytest.mark.parametrize("form", [0, 1])
def test_tile_staging_is_bit_equal(form):
    """The momentum tile's planes staged by TMA tensor copies (tile_tma = 1;
    in the mixed form the FP64 planes, with the FP32 ones as element copies)
    or all by element copies (0): the same values in shared memory, the same
    arithmetic, the same bits."""
    a, b = _case((64, 32, 48), form=form), _case((64, 32, 48), form=form)
    q = b.plan()
    assert q.tile_tma == 1
    q.tile_tma = 0
    b.set_plan(q)
    assert a.step(6) == 0 and b.step(6) == 0
    for nm, x, y in zip(("u", "v", "w", "p", "psi"), _state(a), _state(b)):
        assert np.array_equal(x, y), nm


@pytest.mark.parametrize("n", [(256, 128, 64), (64, 64, 32), (48, 256, 32)])
def test_line_transform_variants_agree(n):
    # periodic y of 128, 64 and 256 points: the two-pass register y
    # transforms (line_transforms = 0) against the Stockham kernels (1)
    a, b = _case(n), _case(n)
    q = b.plan()
    assert q.line_transforms == 0
    q.line_transforms = 1
    b.set_plan(q)
    assert b.plan().line_transforms == 1
    assert a.step(5) == 0 and b.step(5) == 0
    for nm, x, y in zip(("u", "v", "w", "p", "psi"), _state(a), _state(b)):
        if nm == "p":
            x, y = x[1:-1, 1:-1, 1:-1] - x[1:-1, 1:-1, 1:-1].mean(), y[1:-1, 1:-1, 1:-1] - y[1:-1, 1:-1, 1:-1].mean()
        assert np.abs(x - y).max() <= 1e-11 * np.abs(y).max(), nm


def test_autotune_runs_on_a_copy_and_caches(tmp_path):
    cache = str(tmp_path / "plans.txt")
    g = _case((64, 64, 64))
    before = _state(g)
    d0 = g.diag()
    q, rep = g.autotune(cache)
    assert rep.startswith("tuned"), rep
    assert q.ms_per_step > 0 and q.phase_slots in (12, 24, 48) and q.momentum_slots in (24, 48, 96)
    d1 = g.diag()
    assert d1.istep == d0.istep and d1.time == d0.time
    for x, y in zip(before, _state(g)):
        assert np.array_equal(x, y)
    cur = g.plan()
    assert (cur.phase_slots, cur.momentum_slots, cur.zsolve) == (q.phase_slots, q.momentum_slots, q.zsolve)
    lines = open(cache).read().splitlines()
    assert len(lines) == 1 and "grid=64x64x64" in lines[0]
    # the same key: read back, not timed again
    h = _case((64, 64, 64))
    q2, rep2 = h.autotune(cache)
    assert rep2.startswith("cached"), rep2
    assert (q2.phase_slots, q2.momentum_slots, q2.zsolve, q2.fp32_transforms) == \
        (q.phase_slots, q.momentum_slots, q.zsolve, q.fp32_transforms)
    assert len(open(cache).read().splitlines()) == 1
    assert g.step(3) == 0 and h.step(3) == 0


def test_autotune_mixed_with_refined_solve(tmp_path):
    """The mixed form with the FP32 solve: the transform choice is one of the
    knobs; the tuned case then steps."""
    g = _case((64, 64, 64), form=1, refine_sweeps=1)
    q, rep = g.autotune(str(tmp_path / "p.txt"))
    assert rep.startswith("tuned") and q.fp32_transforms in (0, 1), rep
    assert g.step(4) == 0


def test_set_plan_rejects_bad_values():
    g = _case()
    q = g.plan()
    q.phase_slots = 0
    with pytest.raises(lib.CansfzError):
        g.set_plan(q)
