"""The operator of the Poisson solve (product_div_grad, mod_laplace.f90:38-197, collapsed to
11-point stencils per axis) in FP64 and in FP32 (the mixed-precision solve's inner BiCGstab: FP32
weights and arithmetic) against the oracle's FP64 gradient-then-divergence evaluation.

The staged kernels stage their plane ring in 16-byte chunks where the padded rows are 16-byte
aligned (nx a multiple of 4) and the chunk's points are interior, element by element from the
periodic images elsewhere; the vector kernels copy every chunk in 16 bytes, at the box ends from
its periodic image (a tile of a narrow grid wraps at both ends).  The grids cover aligned rows
with interior and wrapped chunks, unaligned rows (every chunk element-wise), ragged x / y tiles,
tile depths that the step depth does not divide, the smallest grid the library accepts and a
stretched z axis (per-plane weights).  Bar: 1e-12 of max|A x| in FP64; 1e-5 in FP32 (rounding of
the input, the weights and 33 products per point; an indexing error is of order one).  FP32 grids
with n1 divisible by 4 and uniform x and z spacing run the FP32 vector kernel (16x16x32,
100x41x26, 8x9x10, 64x56x102: one to several tiles along z, ragged last steps), grids with n1 even
the FP64 vector kernel, the others the staged kernels.
"""
import numpy as np
import pytest

import oracle as O
import impact_b200 as I

pytestmark = pytest.mark.gpu

GRIDS = [((17, 17, 33), (1.0, 1.0, 2.0), (0, 0, 0)),     # 16 x 16 x 32, nx 24: aligned rows
         ((31, 19, 23), (1.0, 1.0, 1.0), (0, 0, 0)),     # 30 x 18 x 22, nx 38: aligned for FP64 only
         ((101, 42, 27), (2.0, 1.0, 1.0), (0, 0, 0)),    # 100 x 41 x 26: aligned, ragged x and y tiles
         ((22, 15, 13), (1.0, 0.7, 0.9), (1, 0, 1)),     # 21 x 14 x 12: unaligned rows, stretched x and z
         ((9, 10, 11), (1.0, 1.0, 1.0), (0, 0, 0)),      # 8 x 9 x 10: the smallest grid, one tile
         ((33, 25, 49), (1.0, 0.8, 2.0), (0, 1, 1)),     # 32 x 24 x 48: aligned, stretched y and z
         ((70, 41, 150), (2.0, 1.0, 3.0), (0, 0, 0)),    # 69 x 40 x 149: unaligned, deep ragged tiles
         ((65, 57, 103), (1.0, 0.9, 1.6), (0, 0, 0))]    # 64 x 56 x 102: FP32 vector kernel, z tiles
IDS = ["16x16x32", "30x18x22", "100x41x26", "21x14x12-xz", "8x9x10", "32x24x48-yz", "69x40x149", "64x56x102"]


@pytest.mark.parametrize("op,tol", [(0, 1e-12), (2, 1e-5)], ids=["fp64", "fp32"])
@pytest.mark.parametrize("gi", range(len(GRIDS)), ids=IDS)
def test_operator_matches_oracle(gi, op, tol):
    N, L, kinds = GRIDS[gi]
    og, ig = O.Grid(N, L, kinds), I.Grid(N, L, kinds)
    case = I.Case(ig, precision=1 if op == 2 else 0)
    x = og.random(17)
    want = og.product_div_grad(x.copy())
    case.upload("pre", x)
    case.apply("pre", "res", op=op)
    got = og.interior(case.download("res"))
    w = og.interior(want)
    assert np.abs(got - w).max() <= tol * np.abs(w).max()
    case.close()
