"""Batched ensemble (cansfz_ensemble_*): independent cases of different sizes
and parameters advanced by one graph launch per step must compute exactly
what each case computes on its own, and an aborting case must stop the
ensemble with its own status while the others report OK.  Cases of the same
grid (different densities, viscosities, surface tension and bubble sizes)
share batched launches; the others run as branches of their own.
"""
import numpy as np
import pytest

from cansfz import case as C
from cansfz import workloads as W

pytestmark = pytest.mark.gpu


def _small_cases():
    return [
        W._bubble_case(64, 2, 128, 1.0, 2.0 / 64, 2.0, 100.0, 10.0, 5.0, 0.4, True),
        W._bubble_case(64, 2, 128, 1.0, 2.0 / 64, 2.0, 1000.0, 100.0, 20.0, 0.3, True),
        W._bubble_case(96, 2, 192, 1.0, 2.0 / 96, 2.0, 1000.0, 100.0, 20.0, 0.3, True),
        W._bubble_case(32, 32, 64, 1.0, 1.0, 2.0, 10.0, 10.0, 1.5, 0.45, False),
        W._bubble_case(32, 32, 64, 1.0, 1.0, 2.0, 100.0, 100.0, 8.0, 0.35, False),
        W._bubble_case(32, 32, 64, 1.0, 1.0, 2.0, 1000.0, 10.0, 25.0, 0.25, False),
        W._bubble_case(48, 48, 96, 1.0, 1.0, 2.0, 1000.0, 10.0, 12.0, 0.3, False),
    ]


def _build(specs, form=0):
    out = []
    for p, f in specs:
        q = p.copy()
        q.form = form
        c = C.Case(q, own_stream=True)
        c.set_fields(*f)
        c.prepare()
        out.append(c)
    return out


@pytest.mark.parametrize("form,batching", [(0, 1), (0, 4), (1, 4)])
def test_ensemble_matches_individual_runs(form, batching):
    specs = _small_cases()
    single = _build(specs, form)
    for c in single:
        assert c.step(12) == 0
    batch = _build(specs, form)
    ens = C.Ensemble(batch, batch=batching)
    rc, st = ens.step(5)  # odd count: the next call starts on the other parity
    assert rc == 0 and st == [0] * len(specs)
    rc, st = ens.step(7)
    assert rc == 0
    # batched: two groups (2 and 3 cases) and two cases on their own
    assert ens.groups() == ((4, 5) if batching > 1 else (len(specs), 0))
    for a, b in zip(single, batch):
        for nm in ("u", "v", "w", "p", "psi"):
            assert np.array_equal(a.get(nm), b.get(nm)), nm
        assert a.diag().istep == b.diag().istep == 12
    ens.close()


def test_ensemble_stops_on_abort():
    # cases 0 and 1 share batched launches; case 1 aborts
    specs = _small_cases()[:3]
    p, f = specs[1]
    u = f[0].copy()
    u[10, 1, 10] = np.nan
    specs[1] = (p, (u,) + tuple(f[1:]))
    batch = _build(specs)
    ens = C.Ensemble(batch, batch=4)
    rc, st = ens.step(25)  # icheck = 10: the NaN is caught at step 10
    assert ens.groups() == (2, 2)
    assert rc in (4, 5)
    assert st[0] == 0 and st[2] == 0 and st[1] == rc
    assert batch[1].diag().istep == 10
    assert batch[0].diag().istep == 25
    # the grouped case that did not abort matches its run on its own
    alone = _build(_small_cases()[:1])[0]
    assert alone.step(25) == 0
    for nm in ("u", "v", "w", "p", "psi"):
        assert np.array_equal(alone.get(nm), batch[0].get(nm)), nm
    rc2, _ = ens.step(1)
    assert rc2 == rc  # the ensemble stays stopped
    ens.close()


def test_batched_two_pass_line_transforms():
    """Same-shape cases with periodic x and y lines of 64 and 128 points: their
    batched launches run the two-pass register transforms (y both ways, x
    backward, and x forward with fillps for the 64-point lines) and compute
    bit for bit what each case computes alone."""
    specs = [W._bubble_case(64, 64, 32, 1.0, 1.0, 0.5, 100.0, 10.0, 8.0, 0.3, False),
             W._bubble_case(64, 64, 32, 1.0, 1.0, 0.5, 1000.0, 100.0, 20.0, 0.35, False),
             W._bubble_case(128, 128, 16, 1.0, 1.0, 0.125, 10.0, 10.0, 2.0, 0.1, False),
             W._bubble_case(128, 128, 16, 1.0, 1.0, 0.125, 100.0, 10.0, 5.0, 0.12, False)]
    single = _build(specs)
    for c in single:
        assert c.step(6) == 0
    batch = _build(specs)
    ens = C.Ensemble(batch, batch=2)
    rc, _ = ens.step(6)
    assert rc == 0
    assert ens.groups() == (2, 4)
    for a, b in zip(single, batch):
        for nm in ("u", "v", "w", "p", "psi"):
            assert np.array_equal(a.get(nm), b.get(nm)), nm
    ens.close()
