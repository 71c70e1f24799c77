"""Full RK3 fractional steps (mod_timeint.f90:242-578) on the device against the CPU FP64 oracle.

Vessel geometry of the plain-step workload (straight cylinder, radius 0.25 L1, inflow buffer
label 5 and outlet label 9), reduced to a grid the oracle finishes in seconds.  Bars: time step
equal to 1e-12 in FP64; velocity within 1e-6 of max|u| (FP64 and mixed precision); Poisson
iteration counts within 3 of the oracle's.  The mixed-precision step with explicit_fp32 = 1
evaluates advection and Helmholtz in FP32 (the FP32 rhs_vel pass), so its velocity -- and the
CFL time step computed from it -- carry FP32 rounding: the mixed step's time step is held to the
velocity's 1e-6 bar.
"""
import numpy as np
import pytest

import oracle as O
import impact_b200 as I
from impact_b200 import geometry as G
from _util import rel_err

pytestmark = pytest.mark.gpu


def _run(precision, nsteps=3, N=(33, 33, 65), L=(1.0, 1.0, 2.0), Re=200.0, precond=0, explicit_fp32=0):
    og, ig = O.Grid(N, L), I.Grid(N, L)
    lab = G.straight_vessel(ig, stenoses=[(1.0, 0.6, 0.125)])
    mg = og.multigrid() if precond == 1 else None
    # oracle
    vel, nl, pre = og.zeros(3), og.zeros(3), og.zeros()
    st = O.OrcStepState()
    p = O.step_params(Re=Re, tol_rel=1e-8, n_sweeps=4, omega=0.8, mg=mg)
    hist = []
    for _ in range(nsteps):
        og.time_step(p, lab, vel, nl, pre, st)
        hist.append((st.dtime, list(st.poisson_iterations)))
    # device
    case = I.Case(ig, precision=precision)
    case.set_labels(lab)
    sp = I.step_params(Re=Re, tol_rel=1e-8, n_sweeps=4, omega=0.8, max_it=2000 if precision == 0 else 30,
                       precond=precond, inner_tol_rel=1e-3, explicit_fp32=explicit_fp32)
    dh = []
    for _ in range(nsteps):
        s = case.step(sp)
        dh.append((s.dtime, list(s.poisson_iterations), list(s.poisson_status)))
    got = [case.download(f) for f in ("vel1", "vel2", "vel3")]
    return og, vel, pre, hist, case, got, dh


def test_step_fp64_odd_rows_matches_oracle():
    """n1 odd: the staged FP64 operator (the vector operator needs whole 16-byte pairs) and, in every
    stencil, rows that are not 16-byte aligned."""
    og, vel, pre, hist, case, got, dh = _run(0, nsteps=2, N=(32, 33, 65))
    for (dt_o, it_o), (dt_g, it_g, stat) in zip(hist, dh):
        assert abs(dt_g - dt_o) <= 1e-12 * dt_o
        assert all(s == 0 for s in stat)
        assert all(abs(a - b) <= 3 for a, b in zip(it_o, it_g))
    umax = max(np.abs(og.interior(vel[m])).max() for m in range(3))
    for m in range(3):
        assert np.abs(og.interior(got[m]) - og.interior(vel[m])).max() <= 1e-6 * umax


@pytest.mark.parametrize("precond", [0, 1], ids=["jor4", "multigrid"])
def test_step_fp64_matches_oracle(precond):
    og, vel, pre, hist, case, got, dh = _run(0, precond=precond)
    for (dt_o, it_o), (dt_g, it_g, stat) in zip(hist, dh):
        assert abs(dt_g - dt_o) <= 1e-12 * dt_o
        assert all(s == 0 for s in stat)
        assert all(abs(a - b) <= 3 for a, b in zip(it_o, it_g))
    umax = max(np.abs(og.interior(vel[m])).max() for m in range(3))
    for m in range(3):
        assert np.abs(og.interior(got[m]) - og.interior(vel[m])).max() <= 1e-6 * umax
    p = case.download("pre")
    d = og.interior(p) - og.interior(pre)
    assert np.abs(d).max() <= 1e-6 * np.abs(og.interior(pre)).max()


@pytest.mark.parametrize("explicit_fp32", [0, 1], ids=["fp64-rhs", "fp32-rhs"])
@pytest.mark.parametrize("precond", [0, 1], ids=["jor4", "multigrid"])
def test_step_mixed_matches_oracle(precond, explicit_fp32):
    og, vel, pre, hist, case, got, dh = _run(1, precond=precond, explicit_fp32=explicit_fp32)
    for (dt_o, _), (dt_g, _, stat) in zip(hist, dh):
        assert abs(dt_g - dt_o) <= 1e-6 * dt_o
        assert all(s == 0 for s in stat)
    umax = max(np.abs(og.interior(vel[m])).max() for m in range(3))
    for m in range(3):
        assert np.abs(og.interior(got[m]) - og.interior(vel[m])).max() <= 1e-6 * umax


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_step_wide_grid_matches_oracle(precision):
    """A grid wide enough for thread blocks whose 3-point halos stay inside the box (the kernels'
    unwrapped fast path) next to blocks at the periodic boundary (the wrapped path)."""
    og, vel, pre, hist, case, got, dh = _run(precision, nsteps=2, N=(97, 25, 33), L=(4.0, 1.0, 1.0), precond=1)
    for (dt_o, _), (dt_g, _, stat) in zip(hist, dh):
        assert abs(dt_g - dt_o) <= 1e-6 * dt_o
        assert all(s == 0 for s in stat)
    umax = max(np.abs(og.interior(vel[m])).max() for m in range(3))
    for m in range(3):
        assert np.abs(og.interior(got[m]) - og.interior(vel[m])).max() <= 1e-6 * umax
