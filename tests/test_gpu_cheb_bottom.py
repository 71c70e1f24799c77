"""The Chebyshev bottom of the V-cycle (solver parameter bottom_cheb): on a grid whose hierarchy
stops at a large coarsest level (n = 8 x 13: the coarsening of mod_setup.f90:95-143 halves an
axis only while its cell count is even, so the coarsest level is 13 x 13 x 13) the reference's
relax_bottom (mod_solvers.f90:420-450: a few Jacobi sweeps) leaves the smooth coarse modes in
place and BiCGstab needs many iterations; d Chebyshev steps of the Jacobi-scaled coarsest
operator in the one-block tail remove them.  The solve still ends at the 1e-8 FP64 residual, with
fewer iterations, and a case in a batch stays bit-identical to the same case alone."""
import numpy as np
import pytest

import impact_b200 as I
from impact_b200 import geometry as G

pytestmark = pytest.mark.gpu

N = (105, 105, 209)  # 104 x 104 x 208 cells: levels 104 -> 52 -> 26 -> 13 per axis (z 208 -> 13)


def _params(precision, cheb):
    return I.solver_params(tol_rel=1e-8, max_it=200 if precision == 0 else 40, precond=1, omega=0.8,
                           mg_down=3, mg_up=3, mg_bottom=3, init_yes=1, check_every=2,
                           inner_tol_rel=3e-3, inner_max_it=400, bottom_cheb=cheb)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_chebyshev_bottom_converges_in_fewer_iterations(precision):
    g = I.Grid(N, (1.0, 1.0, 2.0))
    case = I.Case(g, precision=precision)
    assert case.mg_levels == 5
    rng = np.random.default_rng(11)
    x_true = g.zeros()
    g.interior(x_true)[...] = rng.uniform(-1.0, 1.0, g.interior(x_true).shape)
    case.upload("pre", x_true)
    case.apply("pre", "res", 0)  # b = A x_true (zero mean by construction)
    b = case.download("res")
    its = {}
    for cheb in (0, 24):
        case.upload("pre", g.zeros())
        r = case.poisson("res", "pre", _params(precision, cheb))
        assert r.status == 0, (cheb, r.status)
        case.apply("pre", "nl1", 0)
        res = g.interior(b) - g.interior(case.download("nl1"))
        assert np.sqrt((res ** 2).sum()) <= 1.5e-8 * np.sqrt((g.interior(b) ** 2).sum())
        its[cheb] = r.inner_iterations if precision == 1 else r.iterations
    assert its[24] < its[0], its
    case.close()


def _vessel(n, precision, cheb, Re=400.0):
    g = I.Grid((n + 1, n + 1, 2 * n + 1), (1.0, 1.0, 2.0))
    case = I.Case(g, precision=precision)
    case.set_labels(G.straight_vessel(g, stenoses=[(1.0, 0.5, 0.1)]))
    p = I.step_params(Re=Re, U0=1.0, tol_rel=1e-8, omega=0.8, precond=1, mg_down=3, mg_up=3, mg_bottom=3,
                      max_it=200 if precision == 0 else 40, inner_tol_rel=3e-3, bottom_cheb=cheb)
    return case, p


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_chebyshev_bottom_batch_equals_alone(precision):
    sizes = (104, 40)  # a one-level tail (13^3) and a multi-level one
    alone = []
    for n in sizes:
        case, p = _vessel(n, precision, 16)
        case.step(p, 2)
        alone.append([case.download(f) for f in ("vel1", "vel2", "vel3", "pre")])
        assert all(s == 0 for s in case.state.poisson_status)
        case.close()
    made = [_vessel(n, precision, 16) for n in sizes]
    batch = I.Batch([c for c, _ in made])
    for _ in range(2):
        batch.step([p for _, p in made])
    for (case, _), ref in zip(made, alone):
        assert all(s == 0 for s in case.state.poisson_status)
        for f, want in zip(("vel1", "vel2", "vel3", "pre"), ref):
            assert np.array_equal(case.download(f), want)
    batch.close()


def test_chebyshev_bottom_step_agrees_with_jacobi_bottom():
    """Two preconditioners, one 1e-8 solve: the velocities after two steps agree far inside the
    solve's tolerance."""
    out = []
    for cheb in (0, 16):
        case, p = _vessel(104, 1, cheb)
        case.step(p, 2)
        out.append([case.download(f) for f in ("vel1", "vel2", "vel3")])
        case.close()
    for a, b in zip(*out):
        assert np.abs(a - b).max() <= 1e-6 * max(np.abs(b).max(), 1e-30)
