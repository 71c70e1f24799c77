"""The continuous-batching request loop: requests of different grids arrive over time, are
admitted by HBM budget while others run, share batched launches, and every result equals the
same request run alone (bit for bit: a batch keeps each case's arithmetic separate)."""
import numpy as np
import pytest

import impact_b200 as I
from impact_b200 import geometry as G
from impact_b200 import serve as S

pytestmark = pytest.mark.gpu


def _requests(precision):
    rng = np.random.default_rng(3)
    specs = [((17, 17, 33), 3, 0.0), ((25, 25, 49), 2, 0.0), ((17, 25, 33), 3, 0.02), ((33, 33, 65), 2, 0.05),
             ((21, 17, 41), 2, 0.08)]
    reqs = []
    for rid, (N, nsteps, t) in enumerate(specs):
        seed = int(rng.integers(1 << 30))
        radius = float(rng.uniform(0.15, 0.3))
        Re = float(rng.uniform(100, 800))
        U0 = float(rng.uniform(0.5, 1.5))

        def labels(g, seed=seed, radius=radius):
            return G.curved_tube(g, np.random.default_rng(seed), radius, stenoses=[(1.0, 0.5, 0.125)])

        p = I.step_params(Re=Re, U0=U0, tol_rel=1e-8, omega=0.8, precond=1,
                          max_it=200 if precision == 0 else 30, inner_tol_rel=1e-3)
        reqs.append(S.Request(rid, N, (1.0, 1.0, 2.0), labels, p, nsteps, t))
    return reqs


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_served_results_equal_alone(precision):
    reqs = _requests(precision)
    sizes = sorted(S.case_bytes(r.N, precision) for r in reqs)
    budget = sizes[-1] + sizes[-2]  # room for the two largest at once, so some requests wait
    srv = S.Server(budget, precision=precision, keep=("vel1", "vel2", "vel3", "pre"))
    done = srv.run(reqs)
    assert sorted(d.rid for d in done) == [r.rid for r in reqs]
    assert srv.peak_bytes <= budget
    assert srv.peak_cases >= 2          # work of several requests overlapped in one batch
    for d in done:
        assert all(s == 0 for s in d.status)
        assert d.finished >= d.admitted >= d.arrival - 1e-9
        r = reqs[d.rid]
        g = I.Grid(r.N, r.L)
        c = I.Case(g, precision=precision)
        c.set_labels(r.labels(g))
        c.step(r.params, r.nsteps)
        for f in ("vel1", "vel2", "vel3", "pre"):
            assert np.array_equal(d.fields[f], c.download(f)), (d.rid, f)
        c.close()
    stats = S.summarize(done, max(d.finished for d in done))
    assert stats["latency_p99_s"] >= stats["latency_p50_s"] > 0
