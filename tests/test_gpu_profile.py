"""The in-library profiler and launch counter: with profiling on, the solver's kernels are timed
(CUDA events inside the replayed graphs) and counted; with it off, nothing is recorded."""
import pytest

import impact_b200 as I
from impact_b200 import geometry as G

pytestmark = pytest.mark.gpu


def test_profiler_counts_graph_replays():
    g = I.Grid((33, 33, 65), (1.0, 1.0, 2.0))
    c = I.Case(g, precision=1)
    c.set_labels(G.straight_vessel(g))
    p = I.step_params(Re=300.0, tol_rel=1e-8, omega=0.8, precond=1, max_it=30, inner_tol_rel=1e-3)
    c.step(p, 1)  # engines built, graphs captured without profiling
    I.profile(True)
    n0 = I.launch_count()
    c.step(p, 1)
    prof = I.profile_read()
    I.profile(False)
    assert I.launch_count() > n0
    for k in ("mg_sweep", "div_grad_dot", "x_update", "nl_rhs", "mx_residual", "mx_apply"):
        launches, ms, byts = prof[k]
        assert launches > 0 and ms > 0 and byts > 0, k
    I.profile(False, reset=True)
    c.step(p, 1)
    assert all(v[0] == 0 for v in I.profile_read().values())
