"""The multigrid V-cycle preconditioner (multigridV, mod_solvers.f90:456-585) on the device
against the oracle's restatement, and BiCGstab with it.

Level sizes, level coordinates, per-level compact Laplacians and interpolation weights follow
mod_setup.f90:95-143, mod_geometry.f90:66-103, get_stencil and interp_coeffs; restriction and
interpolation follow restrict / interpolate.  One V-cycle must agree with the oracle to 1e-12
(FP64), including a grid whose axes stop coarsening at different levels and a stretched grid.
"""
import numpy as np
import pytest

import oracle as O
import impact_b200 as I
from _util import rel_err

pytestmark = pytest.mark.gpu

CASES = [((17, 17, 33), (1.0, 1.0, 2.0), (0, 0, 0)), ((33, 25, 17), (1.0, 0.8, 1.0), (1, 1, 0)),
         ((25, 13, 49), (1.0, 0.5, 2.0), (0, 0, 1))]


@pytest.mark.parametrize("N,L,kinds", CASES, ids=["16x16x32", "32x24x16-stretched", "24x12x48-semi"])
@pytest.mark.parametrize("omega", [0.98, 0.8])
def test_vcycle_matches_oracle(N, L, kinds, omega):
    og, ig = O.Grid(N, L, kinds), I.Grid(N, L, kinds)
    mg = og.multigrid()
    case = I.Case(ig, precision=0)
    assert case.mg_levels == mg.n_grids > 1
    b = og.random(5)
    want = mg.vcycle(b.copy(), og.zeros(), 4, 4, 4, omega)
    case.upload("res", b)
    case.precond("res", "pre", I.solver_params(precond=1, omega=omega, mg_down=4, mg_up=4, mg_bottom=4))
    got = case.download("pre")
    assert rel_err(og.interior(got), og.interior(want)) <= 1e-12


def test_jacobi_precond_matches_oracle():
    og, ig = O.Grid((17, 21, 13)), I.Grid((17, 21, 13))
    case = I.Case(ig, precision=0)
    b = og.random(6)
    want = og.jacobi(b.copy(), og.zeros(), 4, 0.8, init_yes=True)
    case.upload("res", b)
    case.precond("res", "pre", I.solver_params(precond=0, n_sweeps=4, omega=0.8))
    assert rel_err(og.interior(case.download("pre")), og.interior(want)) <= 1e-12


@pytest.mark.parametrize("precision", [0, 1])
def test_bicgstab_multigrid_converges(precision):
    N, L = (33, 33, 65), (1.0, 1.0, 2.0)
    og, ig = O.Grid(N, L), I.Grid(N, L)
    mg = og.multigrid()
    x_true = og.random(7)
    b = og.product_div_grad(x_true.copy())
    case = I.Case(ig, precision=precision)
    case.upload("res", b)
    case.upload("pre", og.zeros())
    r = case.poisson("res", "pre", I.solver_params(tol_rel=1e-8, max_it=60 if precision == 0 else 20, precond=1,
                                                   omega=0.8, init_yes=1, inner_tol_rel=1e-3))
    assert r.status == 0
    x = case.download("pre")
    res = og.interior(b) - og.interior(og.product_div_grad(x.copy()))
    assert np.sqrt((res ** 2).sum()) <= 1.5e-8 * np.sqrt((og.interior(b) ** 2).sum())
    r_o = mg.bicgstab(b.copy(), og.zeros(), tol_rel=1e-8, max_it=60, omega=0.8, init_yes=True)
    if precision == 0:
        assert abs(r.iterations - r_o.iterations) <= 2
        assert r.iterations <= 15  # mesh-independent: a handful of iterations instead of hundreds


@pytest.mark.parametrize("N,L,kinds", [((17, 17, 33), (1.0, 1.0, 2.0), (0, 0, 0)),
                                       ((33, 25, 17), (1.0, 0.8, 1.0), (1, 1, 0))],
                         ids=["16x16x32", "32x24x16-stretched"])
def test_product_div_grad_matches_oracle(N, L, kinds):
    """A x of the Poisson solve (product_div_grad, collapsed per axis to 11-point stencils on the
    device) against the oracle's gradient-then-divergence evaluation."""
    og, ig = O.Grid(N, L, kinds), I.Grid(N, L, kinds)
    case = I.Case(ig, precision=0)
    x = og.random(11)
    want = og.product_div_grad(x.copy())
    case.upload("pre", x)
    case.apply("pre", "res")
    got = case.download("res")
    scale = np.abs(og.interior(want)).max()
    assert np.abs(og.interior(got) - og.interior(want)).max() <= 1e-12 * scale


# Grids deep enough that the tile depth of the finest level stays at 16 planes, so that the
# prolongation runs whole blocks of 8 fine planes (in FP32 with every coarse plane of the block
# loaded up front); the second one is stretched in z (per-plane interpolation weights).
DEEP = [((257, 129, 257), (2.0, 1.0, 2.0), (0, 0, 0)), ((257, 129, 193), (2.0, 1.0, 1.5), (0, 0, 1))]


@pytest.mark.parametrize("precision,tol", [(0, 1e-12), (1, 1e-5)], ids=["fp64", "fp32"])
@pytest.mark.parametrize("N,L,kinds", DEEP, ids=["256x128x256", "256x128x192-z"])
def test_vcycle_deep_tiles_matches_oracle(N, L, kinds, precision, tol):
    og, ig = O.Grid(N, L, kinds), I.Grid(N, L, kinds)
    mg = og.multigrid()
    b = og.random(7)
    want = mg.vcycle(b.copy(), og.zeros(), 3, 3, 3, 0.8)
    case = I.Case(ig, precision=precision)
    case.upload("res", b)
    case.precond("res", "pre", I.solver_params(precond=1, omega=0.8, mg_down=3, mg_up=3, mg_bottom=3))
    got = og.interior(case.download("pre"))
    w = og.interior(want)
    assert np.abs(got - w).max() <= tol * np.abs(w).max()
    case.close()
