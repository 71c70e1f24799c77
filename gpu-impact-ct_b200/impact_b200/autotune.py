"""Autotuner of the pressure solve: tile depth of the solver kernels, multigrid sweep schedule and,
for mixed precision, the tolerance of each FP32 inner solve.

The kernels of the Poisson engine cut every grid into tiles of 32 x 8 columns and `tile_kc`
z-planes; deeper tiles stream longer columns (fewer tile start-ups), shallower ones give more
tiles to fill the 148 SMs on small grids and coarse levels.  The V-cycle's sweep counts trade
the cost of one preconditioner application against the number of BiCGstab iterations.  Both are
chosen here by timing complete Poisson solves of the case's own current right-hand side to the
requested tolerance, one per candidate, on the device, and keeping the fastest candidate that
converged.  In mixed precision a looser inner tolerance means cheaper inner solves and more FP64
refinement passes (each one an FP64 residual and correction over the whole grid); a tighter one
fewer passes and longer FP32 solves.  The best balance depends on the case, so it is one more
tuned dimension.  Tolerances below 1e-3 are not offered: the FP32 operator's rounding limits
what one refinement pass gains (on the 384 x 384 x 768 benchmark case, inner solves to 1e-4 still
took three or four passes and made the time step 20 % slower than 3e-3), and the candidates are
timed from a zero start, where tight inner solves look better than they are inside a time step.
Results are cached per (grid, precision, device) for the life of the process.
"""
from __future__ import annotations

import copy
import time

from . import Case, SolverParams

TILE_KC = (8, 16, 32, 64)
SWEEPS = ((2, 2, 2), (3, 3, 3), (4, 4, 4))
INNER_TOL = (1e-3, 3e-3, 1e-2)

_cache: dict = {}


def _with(base: SolverParams, kc: int, sw, itol=None) -> SolverParams:
    p = copy.copy(base)
    p.tile_kc = kc
    p.mg_down, p.mg_up, p.mg_bottom = sw
    if itol is not None:
        p.inner_tol_rel = itol
    return p


def tune(case: Case, base: SolverParams, tile_kc=TILE_KC, sweeps=SWEEPS, rhs="res", scratch="rhs1",
         repeats: int = 1, use_cache: bool = True, inner_tol=INNER_TOL):
    """Time Poisson solves A x = rhs (x from zero, written into `scratch`, which the next time step
    recomputes anyway) for every candidate and return (best SolverParams, report).  The case should
    hold a realistic right-hand side, e.g. after two time steps from rest (the first step of a
    flow at rest has a zero right-hand side; with one, nothing is tuned and `base` is returned).
    Multigrid candidates only when base.precond == 1; otherwise only the tile depth is tuned.
    inner_tol: candidate inner tolerances of a mixed-precision case (ignored in FP64; () keeps
    base.inner_tol_rel)."""
    key = (tuple(case.grid.N), case.precision, base.precond, base.tol_rel, base.omega)
    if use_cache and key in _cache:
        return _cache[key]
    sws = sweeps if base.precond == 1 else [(base.mg_down, base.mg_up, base.mg_bottom)]
    itols = list(inner_tol) if (case.precision == 1 and inner_tol) else [None]
    cands = [(kc, sw, it) for kc in tile_kc for sw in sws for it in itols]
    report = []
    best = None
    for kc, sw, it in cands:
        p = _with(base, kc, sw, it)
        p.init_yes = 1
        r0 = case.poisson(rhs, scratch, p)  # builds the engine and its graphs
        if r0.b_two == 0.0:
            # a zero right-hand side (e.g. a flow still at rest) solves in no iterations: timing
            # it says nothing about the candidates, so the base parameters stay
            return copy.copy(base), [{"skipped": "zero right-hand side"}]
        t0 = time.perf_counter()
        for _ in range(repeats):
            r = case.poisson(rhs, scratch, p)  # returns after the device has finished
        ms = 1e3 * (time.perf_counter() - t0) / repeats
        ok = r.status == 0
        report.append({"tile_kc": kc, "sweeps": list(sw), "inner_tol": it, "ms": round(ms, 3),
                       "iterations": r.iterations, "inner_iterations": r.inner_iterations, "converged": ok})
        if ok and (best is None or ms < best[0]):
            best = (ms, kc, sw, it)
    if best is None:
        chosen = copy.copy(base)
    else:
        chosen = _with(base, best[1], best[2], best[3])
    out = (chosen, report)
    if use_cache:
        _cache[key] = out
    return out
