"""Device Poisson solvers against the CPU FP64 oracle (mod_solvers.f90 restatement).

* BiCGstab_orig with the Jacobi preconditioner: a fixed number of iterations must track the
  oracle's iterates (the only difference is the order of the FP64 inner-product sums);
* a converged solve reaches ||b - A x||_2 <= 1e-8 ||b||_2 measured with the oracle's operator;
* the mixed-precision solve (FP32 inner BiCGstab, FP64 refinement) reaches the same residual;
* the device_jacobi_solver replacement equals the same number of oracle JOR sweeps;
* failures (non-finite input, iteration cap) come back as status codes, never as a hang.
"""
import numpy as np
import pytest

import oracle as O
import impact_b200 as I
from _util import rel_err

pytestmark = pytest.mark.gpu


def _rhs(og, seed):
    """a right-hand side in the range of A (on stretched periodic grids the left null vector of
    A is not the constant, so a merely mean-free vector would be inconsistent)"""
    x = og.random(seed)
    return og.product_div_grad(x)


def _case(N, L=(1.0, 1.0, 2.0), kinds=(0, 0, 0), precision=0):
    og, ig = O.Grid(N, L, kinds), I.Grid(N, L, kinds)
    return og, ig, I.Case(ig, precision=precision)


@pytest.mark.parametrize("init_yes", [1, 0])
@pytest.mark.parametrize("n_sweeps", [0, 1, 4])
def test_bicgstab_iterates_track_oracle(init_yes, n_sweeps):
    og, ig, case = _case((17, 25, 33), kinds=(1, 0, 0))
    b = _rhs(og, 1)
    x0 = og.random(2) if not init_yes else og.zeros()
    want = x0.copy()
    r_o = og.bicgstab(b.copy(), want, tol_rel=0.0, max_it=8, n_sweeps=n_sweeps, omega=0.8, init_yes=bool(init_yes))
    case.upload("res", b)
    case.upload("pre", x0)
    r = case.poisson("res", "pre", I.solver_params(tol_rel=0.0, max_it=8, n_sweeps=n_sweeps, omega=0.8,
                                                   init_yes=init_yes, check_every=3))
    got = case.download("pre")
    assert r.iterations == r_o.iterations == 8
    assert rel_err(og.interior(got), og.interior(want)) <= 1e-9


@pytest.mark.parametrize("kinds", [(0, 0, 0), (1, 1, 0)])
def test_bicgstab_converges_to_1e8(kinds):
    og, ig, case = _case((33, 33, 65), kinds=kinds)
    x_true = og.random(3)
    b = og.product_div_grad(x_true.copy())
    case.upload("res", b)
    case.upload("pre", og.zeros())
    r = case.poisson("res", "pre", I.solver_params(tol_rel=1e-8, max_it=2000, n_sweeps=4, omega=0.8, init_yes=1))
    assert r.status == 0
    x = case.download("pre")
    Ax = og.product_div_grad(x.copy())
    res = og.interior(b) - og.interior(Ax)
    assert np.sqrt((res ** 2).sum()) <= 1.5e-8 * np.sqrt((og.interior(b) ** 2).sum())
    want = og.zeros()
    r_o = og.bicgstab(b.copy(), want, tol_rel=1e-8, max_it=2000, n_sweeps=4, omega=0.8, init_yes=True)
    # same algorithm: iteration counts agree up to the drift of the FP64 inner-product order
    assert abs(r.iterations - r_o.iterations) <= max(3, 0.15 * r_o.iterations)

    def err(sol):  # distance to the known solution, up to the periodic constant
        d = og.interior(sol) - og.interior(x_true)
        return np.abs(d - d.mean()).max()

    assert err(x) <= 3.0 * err(want) + 1e-12


def test_mixed_precision_solve_reaches_fp64_residual():
    og, ig, case = _case((33, 33, 65), precision=1)
    x_true = og.random(4)
    b = og.product_div_grad(x_true.copy())
    case.upload("res", b)
    case.upload("pre", og.zeros())
    r = case.poisson("res", "pre", I.solver_params(tol_rel=1e-8, max_it=20, n_sweeps=4, omega=0.8, init_yes=1,
                                                   inner_tol_rel=1e-3))
    assert r.status == 0, r.status
    assert r.inner_iterations > 0 and r.iterations >= 2
    x = case.download("pre")
    Ax = og.product_div_grad(x.copy())
    res = og.interior(b) - og.interior(Ax)
    assert np.sqrt((res ** 2).sum()) <= 1e-8 * np.sqrt((og.interior(b) ** 2).sum())
    want = og.zeros()
    og.bicgstab(b.copy(), want, tol_rel=1e-8, max_it=4000, n_sweeps=4, omega=0.8, init_yes=True)

    def err(sol):
        d = og.interior(sol) - og.interior(x_true)
        return np.abs(d - d.mean()).max()

    # the mixed-precision result is as close to the true solution as the FP64 solve at 1e-8
    assert err(x) <= 3.0 * err(want) + 1e-12


def test_jacobi_solve_matches_sweeps():
    og, ig = O.Grid((17, 17, 25)), I.Grid((17, 17, 25))
    b, rel = og.random(5), og.random(6)
    want = og.jacobi(b.copy(), rel.copy(), 37, 0.8, init_yes=False)
    got = rel.copy()
    sweeps, _ = I.jacobi_solve(ig, got, b, omega=0.8, mode_j=1000, max_sweeps=37)
    assert sweeps == 37
    assert rel_err(og.interior(got), og.interior(want)) <= 1e-12


def test_jacobi_solve_with_ct_pressure_condition():
    """Every iteration first sets the inlet / outlet planes (jacobi_solver_host_v4.f90:302-305),
    then sweeps: the oracle's pressure_bc and one JOR sweep, 29 times."""
    N = (17, 17, 25)
    og, ig = O.Grid(N), I.Grid(N)
    b, rel = og.random(9), og.random(10)
    lab = np.ones(og.shape, dtype=np.uint8)
    ks = 6
    lab[ks - 1 + 3, 6:12, 6:12] = 5   # inlet disc on plane ks - 1
    lab[ks - 1 + 3, 13:16, 4:8] = 9   # first outlet on the same plane
    lab[20 + 3, 6:10, 6:10] = 11      # second outlet (type_id3 = 1 here)
    lab[ks + 3, 6:12, 6:12] = 5       # label 5 off the plane: left alone
    pin, pout, pout2 = 0.31, -0.12, 0.05
    want = rel.copy()
    for _ in range(29):
        og.pressure_bc(lab, ks, pin, pout, pout2, want)
        want = og.jacobi(b.copy(), want, 1, 0.8, init_yes=False)
    got = rel.copy()
    sweeps, _ = I.jacobi_solve(ig, got, b, omega=0.8, mode_j=1000, max_sweeps=29, labels=lab, k_start_index=ks,
                               type_ids=(1, 1, 1), pressures=(pin, pout, pout2))
    assert sweeps == 29
    assert rel_err(og.interior(got), og.interior(want)) <= 1e-12
    # without the condition the result differs
    plain = rel.copy()
    I.jacobi_solve(ig, plain, b, omega=0.8, mode_j=1000, max_sweeps=29)
    assert rel_err(og.interior(plain), og.interior(want)) > 1e-6


def test_jacobi_solve_heuristic_stop_terminates():
    og, ig = O.Grid((17, 17, 17)), I.Grid((17, 17, 17))
    b = _rhs(og, 7)
    rel = og.zeros()
    sweeps, res = I.jacobi_solve(ig, rel, b, omega=0.8, mode_j=20, max_sweeps=20000)
    assert 0 < sweeps < 20000 and np.isfinite(res)


def test_nonfinite_rhs_reports_status():
    og, ig, case = _case((17, 17, 17))
    b = _rhs(og, 8)
    og.interior(b)[3, 4, 5] = np.nan
    case.upload("res", b)
    case.upload("pre", og.zeros())
    r = case.poisson("res", "pre", I.solver_params(tol_rel=1e-8, max_it=50, init_yes=1))
    assert r.status == 3


def test_iteration_cap_reports_status():
    og, ig, case = _case((17, 17, 33))
    b = _rhs(og, 9)
    case.upload("res", b)
    case.upload("pre", og.zeros())
    r = case.poisson("res", "pre", I.solver_params(tol_rel=1e-14, max_it=3, init_yes=1))
    assert r.status == 1 and r.iterations == 3
