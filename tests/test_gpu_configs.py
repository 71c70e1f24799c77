"""Parity at the benchmark configurations' own sizes, against the CPU FP64 oracle.

Plain step (64 x 64 x 128 cells): straight cylindrical vessel of radius 0.25 L1 (label-5 inflow
buffer on the first 10 planes, label-9 outlet on the last 10), pulsatile plug inflow
U0 (1 + 0.5 sin(2 pi t / T)), Re = 200, dt = 0.2 x the CFL limit, 10 FP64 RK3 steps from rest,
every Poisson solve BiCGstab with the JOR preconditioner (omega = 0.8, 4 sweeps) to a 1e-8
relative residual (mod_timeint.f90:242-578, mod_solvers.f90:1509-1935).  Bars: time step equal
to 1e-10 (it follows the velocity, whose last bits differ); iteration counts within 10 % of the
oracle's; velocity and pressure within 1e-6 of their
maxima; the discrete divergence of the reference's in-code check (test_divergence,
mod_test.f90:300-345: max |div2(u)| and max |div2(u) weight|) equal to 1e-6.

Operator microbench (256 x 256 x 512 cells, x and y stretched by x_i = sinh(2 (i/N - 1/2)) /
sinh 1, z uniform, i.i.d. U[-1, 1] fields from fixed seeds): gradient, divergence2, explicit
Helmholtz (multL = 1e-3), the nine upwind terms, both interpolations and 50 JOR sweeps
(omega = 0.8), each through the reference's launcher FFI (FP64) and its _sp FP32 counterpart.
Bars: max |gpu - oracle| / max |oracle| <= 1e-12 (FP64) and <= 1e-5 (FP32, inputs and tables
rounded to FP32, against the FP64 oracle).
"""
import numpy as np
import pytest

import oracle as O
import impact_b200 as I
from impact_b200 import geometry as G
from _util import dev, host, ptr, rel_err

pytestmark = pytest.mark.gpu

TOL64, TOL32 = 1e-12, 1e-5


# ------------------------------------------------------------------------------------------
# plain step, 64 x 64 x 128, 10 FP64 steps
# ------------------------------------------------------------------------------------------
def test_plain_step_config_10_steps_matches_oracle():
    N, L = (65, 65, 129), (1.0, 1.0, 2.0)
    og, ig = O.Grid(N, L), I.Grid(N, L)
    lab = G.straight_vessel(ig, radius_frac=0.25, n_in=10, n_out=10)
    vel, nl, pre = og.zeros(3), og.zeros(3), og.zeros()
    st = O.OrcStepState()
    p = O.step_params(Re=200.0, CFL=0.2, tol_rel=1e-8, n_sweeps=4, omega=0.8)
    case = I.Case(ig, precision=0)
    case.set_labels(lab)
    sp = I.step_params(Re=200.0, CFL=0.2, tol_rel=1e-8, n_sweeps=4, omega=0.8, max_it=2000, precond=0)
    for step in range(10):
        og.time_step(p, lab, vel, nl, pre, st)
        s = case.step(sp)
        assert abs(s.dtime - st.dtime) <= 1e-10 * st.dtime, step
        assert all(x == 0 for x in s.poisson_status), (step, list(s.poisson_status))
        # about 105 JOR-preconditioned iterations per solve: rounding moves the count by a few
        assert all(abs(a - b) <= max(3, 0.1 * a) for a, b in zip(st.poisson_iterations, s.poisson_iterations)), \
            (step, list(st.poisson_iterations), list(s.poisson_iterations))
    got = np.stack([case.download(f) for f in ("vel1", "vel2", "vel3")])
    umax = max(np.abs(og.interior(vel[m])).max() for m in range(3))
    for m in range(3):
        assert np.abs(og.interior(got[m]) - og.interior(vel[m])).max() <= 1e-6 * umax
    gp = case.download("pre")
    assert np.abs(og.interior(gp) - og.interior(pre)).max() <= 1e-6 * np.abs(og.interior(pre)).max()
    want_div, got_div = og.test_divergence(vel), og.test_divergence(got)
    for a, b in zip(got_div, want_div):
        assert abs(a - b) <= 1e-6 * b
    # the same metric on the fluid points away from the mask (labels 1 whose divergence stencil,
    # 3 points each way, sees fluid only): the solver's own divergence error
    fl = og.interior(lab) == G.FLUID
    inner = fl.copy()
    for ax in range(3):
        for sh in (-3, -2, -1, 1, 2, 3):
            inner &= np.roll(fl, sh, axis=ax)
    # (the oracle reaches about 2.5e-10 here; both runs stop at a 1e-8 relative residual, so the
    # bar is that tolerance on the velocity-gradient scale umax / dx, about 7e-7)
    dx = 1.0 / 64
    want_in, got_in = og.test_divergence(vel, inner), og.test_divergence(got, inner)
    assert want_in[0] <= 1e-8 * umax / dx
    assert got_in[0] <= 1e-8 * umax / dx
    case.close()


# ------------------------------------------------------------------------------------------
# operator microbench, 256 x 256 x 512 stretched
# ------------------------------------------------------------------------------------------
N2 = (257, 257, 513)


@pytest.fixture(scope="module")
def big():
    L, kinds = (2.0, 2.0, 4.0), (1, 1, 0)
    og, ig = O.Grid(N2, L, kinds), I.Grid(N2, L, kinds)
    return og, ig


def _dims(og):
    return tuple(n + 7 for n in og.N)


def _t(ig, name, a, f32):
    t = ig.tab[name][a]
    return dev(t.astype(np.float32) if f32 else t)


def _f(a, f32):
    return dev(a.astype(np.float32) if f32 else a)


def _check(og, got, want, f32):
    assert rel_err(og.interior(host(got)), og.interior(want)) <= (TOL32 if f32 else TOL64)


@pytest.mark.parametrize("f32", [False, True], ids=["fp64", "fp32"])
def test_operators_gradient_and_divergence2_at_size(big, f32):
    og, ig = big
    nx, ny, nz = _dims(og)
    sfx = "_sp_" if f32 else "_"
    phi = og.random(1001)
    d_phi = _f(phi, f32)
    for m in (1, 2, 3):
        want = og.gradient(m, phi)
        d_out, t_g = _f(og.zeros(), f32), _t(ig, "cG", m - 1, f32)
        I.launchers.call("gradient_launcher" + sfx, ("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 6),
                         ("i", og.N[m - 1] + 1), ("p", ptr(d_phi)), ("p", ptr(t_g)), ("p", ptr(d_out)))
        _check(og, d_out, want, f32)
    del d_phi
    vel = og.random(1002, n=3)
    want = og.divergence2(vel[0], vel[1], vel[2])
    d_vel, d_div = _f(vel, f32), _f(og.zeros(), f32)
    c = [_t(ig, "cD", a, f32) for a in range(3)]
    I.launchers.call("divergence2_launcher" + sfx, ("i", nx), ("i", ny), ("i", nz), ("i", 6), ("i", 6), ("i", 6),
                     ("p", ptr(d_vel)), ("p", ptr(d_div)), ("p", ptr(c[0])), ("p", ptr(c[1])), ("p", ptr(c[2])))
    _check(og, d_div, want, f32)


@pytest.mark.parametrize("f32", [False, True], ids=["fp64", "fp32"])
def test_operators_helmholtz_and_interpolations_at_size(big, f32):
    og, ig = big
    nx, ny, nz = _dims(og)
    sfx = "_sp_" if f32 else "_"
    scal = "f" if f32 else "d"
    vel, nl0 = og.random(1011), og.random(1012)
    d_vel = _f(vel, f32)
    for m in (1, 2, 3):
        want = og.helmholtz(m, 1e-3, vel, nl0.copy())
        names = [("cuu" if a == m - 1 else "cpp") for a in range(3)]
        c = [_t(ig, names[a], a, f32) for a in range(3)]
        d_nl = _f(nl0, f32)
        I.launchers.call("helmholtz_explicit_launcher" + sfx, ("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 7),
                         ("i", 7), ("i", 7), (scal, 1e-3), ("p", ptr(d_vel)), ("p", ptr(d_nl)), ("p", ptr(c[0])),
                         ("p", ptr(c[1])), ("p", ptr(c[2])))
        _check(og, d_nl, want, f32)
    for m in (1, 2, 3):
        d_out, t_pu, t_up = _f(og.zeros(), f32), _t(ig, "cIpu", m - 1, f32), _t(ig, "cIup", m - 1, f32)
        I.launchers.call("interpolate2_pre_vel_launcher" + sfx, ("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 6),
                         ("i", og.N[m - 1] + 1), ("p", ptr(d_vel)), ("p", ptr(t_pu)), ("p", ptr(d_out)))
        _check(og, d_out, og.interpolate_pre_vel(m, vel), f32)
        I.launchers.call("interpolate2_vel_pre_launcher" + sfx, ("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 6),
                         ("i", og.N[m - 1] + 1), ("p", ptr(d_vel)), ("p", ptr(t_up)), ("p", ptr(d_out)))
        _check(og, d_out, og.interpolate_vel_pre(m, vel), f32)


@pytest.mark.parametrize("f32", [False, True], ids=["fp64", "fp32"])
def test_operators_upwind_nine_terms_at_size(big, f32):
    og, ig = big
    nx, ny, nz = _dims(og)
    sfx = "_sp_" if f32 else "_"
    vel, pp = og.random(1021), og.random(1022)  # mixed signs exercise both upwind tables
    d_vel, d_pp = _f(vel, f32), _f(pp, f32)
    for cid in range(1, 10):
        m, a = (cid - 1) // 3 + 1, (cid - 1) % 3 + 1
        nl = og.random(1030 + cid)
        want = og.nonlinear_upwind(cid, pp, vel, nl.copy())
        up, dn = ("cNuU", "cNuD") if a == m else ("cNpU", "cNpD")
        d_nl = _f(nl, f32)
        t_up, t_dn = _t(ig, up, a - 1, f32), _t(ig, dn, a - 1, f32)  # both tables alive during the launch
        I.launchers.call("nonlinear_upwind_launcher" + sfx, ("i", cid), ("i", nx), ("i", ny), ("i", nz), ("i", 7),
                         ("i", og.N[a - 1] + 1), ("p", ptr(d_pp)), ("p", ptr(d_vel)), ("p", ptr(d_nl)),
                         ("p", ptr(t_up)), ("p", ptr(t_dn)))
        _check(og, d_nl, want, f32)


@pytest.mark.parametrize("f32", [False, True], ids=["fp64", "fp32"])
def test_operators_fifty_jor_sweeps_at_size(big, f32):
    og, ig = big
    nx, ny, nz = _dims(og)
    sfx = "_sp_" if f32 else "_"
    scal = "f" if f32 else "d"
    bb, rel = og.random(1041), og.random(1042)
    want = og.jacobi(bb.copy(), rel.copy(), 50, 0.8, init_yes=False)
    c = [_t(ig, "cdg", a, f32) for a in range(3)]
    d_bb, d_rel, d_comp = _f(bb, f32), _f(rel, f32), _f(og.zeros(), f32)
    for _ in range(50):
        I.launchers.call("jacobi_launcher" + sfx, ("i", 1), ("i", nx), ("i", ny), ("i", nz), ("i", og.N[0]),
                         ("i", og.N[1]), ("i", og.N[2]), ("i", 3), (scal, 0.8), ("p", ptr(c[0])), ("p", ptr(c[1])),
                         ("p", ptr(c[2])), ("p", ptr(d_rel)), ("p", ptr(d_bb)), ("p", ptr(d_comp)))
        d_rel, d_comp = d_comp, d_rel
    _check(og, d_rel, want, f32)
