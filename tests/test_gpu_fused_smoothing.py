"""The fused V-cycle smoothing kernels: every pre-smoothing phase (init sweep, the remaining
sweeps and the residual before the restriction) and every post-smoothing phase (the sweeps after
the prolongation) of a level run as one z-marching kernel instead of one launch per sweep.

They must give the iterate of the one-sweep-per-launch schedule bit for bit (same operations per
point in the same order), for every sweep count that has a fused kernel (2..4), on equidistant,
stretched (z rows differ: the non-uniform path) and ragged grids whose sizes do not fill the
64 x 16 / 32 x 16 / x 8 column tiles, in FP64 and FP32 (one V-cycle) and in the inner solve of
the mixed-precision Poisson solve; and one V-cycle with 2 and 3 sweeps must agree with the
oracle's multigridV to 1e-12.
"""
import numpy as np
import pytest

import oracle as O
import impact_b200 as I
from _util import rel_err

pytestmark = pytest.mark.gpu

GRIDS = [((17, 17, 33), (1.0, 1.0, 2.0), (0, 0, 0)),     # 16 x 16 x 32
         ((33, 25, 17), (1.0, 0.8, 1.0), (1, 1, 0)),     # stretched x, y
         ((25, 13, 49), (1.0, 0.5, 2.0), (0, 0, 1)),     # stretched z (per-plane diagonal)
         ((70, 41, 150), (2.0, 1.0, 3.0), (0, 0, 0)),    # 69 x 40 x 149: ragged tiles and z chunks
         ((129, 65, 33), (1.0, 0.5, 0.25), (0, 0, 0))]   # 128 x 64 x 32: ragged x / y tiles of the fast path
GIDS = ["16x16x32", "32x24x16-xy", "24x12x48-z", "69x40x149", "128x64x32"]
SWEEPS = [(2, 2, 2), (3, 3, 3), (4, 4, 4), (2, 3, 4), (3, 2, 1)]


def _params(sw, unfused, omega=0.8, **kw):
    return I.solver_params(precond=1, omega=omega, mg_down=sw[0], mg_up=sw[1], mg_bottom=sw[2],
                           smooth_unfused=unfused, **kw)


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "fp32"])
@pytest.mark.parametrize("gi", range(len(GRIDS)), ids=GIDS)
@pytest.mark.parametrize("sw", SWEEPS, ids=lambda s: "%d%d%d" % s)
def test_fused_vcycle_equals_one_sweep_per_launch(gi, sw, precision):
    """precision 1: the FP32 V-cycle of the mixed solve's inner solve."""
    N, L, kinds = GRIDS[gi]
    og, ig = O.Grid(N, L, kinds), I.Grid(N, L, kinds)
    case = I.Case(ig, precision=precision)
    case.upload("res", og.random(21))
    case.precond("res", "pre", _params(sw, 1))
    want = case.download("pre")
    case.precond("res", "rhs1", _params(sw, 0))
    got = case.download("rhs1")
    assert np.array_equal(og.interior(got), og.interior(want)), rel_err(og.interior(got), og.interior(want))
    case.close()


@pytest.mark.parametrize("sw", [(2, 2, 2), (3, 3, 3)], ids=["222", "333"])
@pytest.mark.parametrize("gi", [0, 2], ids=[GIDS[0], GIDS[2]])
def test_fused_vcycle_matches_oracle(gi, sw):
    N, L, kinds = GRIDS[gi]
    og, ig = O.Grid(N, L, kinds), I.Grid(N, L, kinds)
    mg = og.multigrid()
    b = og.random(5)
    want = mg.vcycle(b.copy(), og.zeros(), sw[0], sw[1], sw[2], 0.8)
    case = I.Case(ig, precision=0)
    case.upload("res", b)
    case.precond("res", "pre", _params(sw, 0))
    assert rel_err(og.interior(case.download("pre")), og.interior(want)) <= 1e-12
    case.close()


@pytest.mark.parametrize("gi", [3, 4], ids=[GIDS[3], GIDS[4]])
@pytest.mark.parametrize("sw", [(3, 3, 3), (4, 2, 2)], ids=["333", "422"])
def test_fused_mixed_solve_equals_one_sweep_per_launch(sw, gi):
    """The FP32 inner solve of the mixed-precision Poisson solve with fused and unfused smoothing:
    same iteration counts, same solution bit for bit."""
    N, L, kinds = GRIDS[gi]
    og, ig = O.Grid(N, L, kinds), I.Grid(N, L, kinds)
    b = og.product_div_grad(og.random(9))
    out = []
    for unfused in (1, 0):
        case = I.Case(ig, precision=1)
        case.upload("res", b)
        case.upload("pre", og.zeros())
        r = case.poisson("res", "pre", _params(sw, unfused, tol_rel=1e-8, max_it=20, init_yes=1, inner_tol_rel=1e-3))
        assert r.status == 0
        out.append((r.iterations, r.inner_iterations, case.download("pre")))
        case.close()
    assert out[0][:2] == out[1][:2]
    assert np.array_equal(og.interior(out[0][2]), og.interior(out[1][2])), rel_err(og.interior(out[1][2]),
                                                                                   og.interior(out[0][2]))
