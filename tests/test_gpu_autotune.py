"""The solver autotuner: every candidate (tile depth x multigrid sweep schedule x, in mixed
precision, inner tolerance) is timed on a complete Poisson solve of the case's own right-hand
side, the fastest converged one is returned, and it leaves the case's state untouched (the next
step equals a run without tuning)."""
import numpy as np
import pytest

import impact_b200 as I
from impact_b200 import autotune as A
from impact_b200 import geometry as G

pytestmark = pytest.mark.gpu


def _case(precision):
    g = I.Grid((33, 33, 65), (1.0, 1.0, 2.0))
    c = I.Case(g, precision=precision)
    c.set_labels(G.straight_vessel(g, stenoses=[(1.0, 0.5, 0.125)]))
    return c


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_autotune_picks_a_converged_candidate(precision):
    p = I.step_params(Re=300.0, tol_rel=1e-8, omega=0.8, precond=1, max_it=200 if precision == 0 else 40)
    ref = _case(precision)
    ref.step(p, 3)
    c = _case(precision)
    c.step(p, 2)  # the first step from rest leaves a zero right-hand side
    itols = (1e-3, 1e-2) if precision == 1 else ()  # inner tolerances: mixed precision only
    best, report = A.tune(c, p.poisson, tile_kc=(8, 32), sweeps=((2, 2, 2), (4, 4, 4)), use_cache=False,
                          inner_tol=itols)
    assert len(report) == 4 * max(1, len(itols)) and all(r["converged"] for r in report)
    assert all(r["iterations"] > 0 for r in report)
    fastest = min(report, key=lambda r: r["ms"])
    assert (best.tile_kc, [best.mg_down, best.mg_up, best.mg_bottom]) == (fastest["tile_kc"], fastest["sweeps"])
    if precision == 1:
        assert best.inner_tol_rel == fastest["inner_tol"]
    # tuning only wrote the scratch field: the next step matches the untuned run
    c.step(p, 1)
    for f in ("vel1", "vel2", "vel3", "pre"):
        assert np.array_equal(c.download(f), ref.download(f))


def test_autotune_leaves_a_zero_right_hand_side_untuned():
    p = I.step_params(Re=300.0, tol_rel=1e-8, omega=0.8, precond=1, max_it=200)
    c = _case(0)
    c.step(p, 1)  # from rest: the Poisson right-hand side of the last substep is zero
    best, report = A.tune(c, p.poisson, tile_kc=(8, 32), sweeps=((2, 2, 2),), use_cache=False)
    assert report == [{"skipped": "zero right-hand side"}]
    assert (best.tile_kc, best.mg_down) == (p.poisson.tile_kc, p.poisson.mg_down)
