"""The autotuner's host logic (impact_b200.autotune.tune) with the device solve replaced by a
stand-in whose cost and convergence depend on the candidate, and a virtual clock: the fastest
converged candidate wins, candidates that do not converge are never chosen, the inner tolerance
is tuned in mixed precision only, without the multigrid only the tile depth is tuned, a zero
right-hand side leaves the base parameters, and results are cached per grid and parameters."""
import pytest

import impact_b200 as I
from impact_b200 import autotune as A


class Clock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t


class Result:
    def __init__(self, status, b_two=1.0):
        self.status, self.b_two, self.iterations, self.inner_iterations = status, b_two, 5, 9


class FakeGrid:
    N = (65, 65, 129)


class FakeCase:
    """Cost in ms of one solve = cost(tile_kc, sweeps, inner_tol); `bad` candidates fail."""

    def __init__(self, clock, precision, cost, bad=(), b_two=1.0):
        self.grid, self.precision = FakeGrid(), precision
        self.clock, self.cost, self.bad, self.b_two = clock, cost, set(bad), b_two
        self.calls = []

    def poisson(self, rhs, scratch, p):
        key = (p.tile_kc, (p.mg_down, p.mg_up, p.mg_bottom), p.inner_tol_rel if self.precision == 1 else None)
        self.calls.append(key)
        self.clock.t += self.cost(*key) / 1e3
        return Result(2 if key in self.bad else 0, self.b_two)


@pytest.fixture
def clock(monkeypatch):
    c = Clock()
    monkeypatch.setattr(A.time, "perf_counter", c)
    A._cache.clear()
    yield c
    A._cache.clear()


def test_fastest_converged_candidate_wins(clock):
    def cost(kc, sw, it):
        return 100 - kc + 10 * abs(sw[0] - 3) + {3e-3: 0, 1e-3: 7, 1e-2: 8}[it]
    bad = {(64, (3, 3, 3), 3e-3)}  # the fastest one does not converge
    case = FakeCase(clock, 1, cost, bad)
    base = I.solver_params(precond=1, inner_tol_rel=1e-3)
    best, report = A.tune(case, base)
    # the next fastest: same depth and sweeps, inner tolerance 1e-3 (7 ms more; 1e-2: 8 ms more)
    assert (best.tile_kc, (best.mg_down, best.mg_up, best.mg_bottom), best.inner_tol_rel) == (64, (3, 3, 3), 1e-3)
    assert len(report) == len(A.TILE_KC) * len(A.SWEEPS) * len(A.INNER_TOL)
    assert sum(1 for r in report if not r["converged"]) == 1
    # each candidate: one untimed solve (engine build) and one timed one
    assert len(case.calls) == 2 * len(report)
    # cached per grid and parameters
    again, _ = A.tune(case, base)
    assert again.tile_kc == best.tile_kc and len(case.calls) == 2 * len(report)


def test_fp64_and_jacobi_restrict_the_candidates(clock):
    case = FakeCase(clock, 0, lambda kc, sw, it: 50 + kc)
    best, report = A.tune(case, I.solver_params(precond=1))
    assert {r["inner_tol"] for r in report} == {None} and best.tile_kc == 8
    A._cache.clear()
    case = FakeCase(clock, 1, lambda kc, sw, it: 50 + kc)
    base = I.solver_params(precond=0, n_sweeps=4, mg_down=4, mg_up=4, mg_bottom=4)
    best, report = A.tune(case, base, inner_tol=())
    assert {tuple(r["sweeps"]) for r in report} == {(4, 4, 4)} and len(report) == len(A.TILE_KC)


def test_zero_rhs_keeps_the_base(clock):
    case = FakeCase(clock, 1, lambda kc, sw, it: 10.0, b_two=0.0)
    base = I.solver_params(precond=1, tile_kc=16)
    best, report = A.tune(case, base)
    assert report == [{"skipped": "zero right-hand side"}] and best.tile_kc == 16


def test_nothing_converges_keeps_the_base(clock):
    case = FakeCase(clock, 0, lambda kc, sw, it: 10.0)
    case.bad = {(kc, sw, None) for kc in A.TILE_KC for sw in A.SWEEPS}
    base = I.solver_params(precond=1, tile_kc=16, mg_down=2, mg_up=2, mg_bottom=2)
    best, report = A.tune(case, base)
    assert best.tile_kc == 16 and (best.mg_down, best.mg_up, best.mg_bottom) == (2, 2, 2)
    assert not any(r["converged"] for r in report)
