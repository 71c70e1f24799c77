"""rhs_vel of each velocity component (mod_rhs.f90:35-140) on the device -- the z-marching
stencil pass of the time step: upwind advection by the interpolated velocities, explicit
Helmholtz and both RK updates -- against the CPU FP64 oracle (interpolate_vel, nonlinear and
Helmholtz_explicit restated from mod_diff.f90).

Grids: equidistant, sinh-stretched (every coefficient row different) and ragged ones: sizes
that do not fill the 32 x 8 column tiles, an x axis shorter than one tile (8 points, the
smallest grid the library accepts), and plane counts that the z chunks of a block do not
divide.  Fields are seeded U[-1, 1], so both upwind branches occur everywhere.  Bar: 1e-12 of
max|.| (FP64).
"""
import numpy as np
import pytest

import oracle as O
import impact_b200 as I
from _util import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12
MULTL, MULT_B, MULT_A = 2e-3, -0.01, 0.02  # the constants of kernel_bench ids 10..12
GRIDS = [
    ((17, 17, 33), (1.0, 1.0, 2.0), (0, 0, 0)),    # 16 x 16 x 32, equidistant
    ((33, 25, 17), (1.0, 1.0, 1.0), (1, 1, 0)),    # 32 x 24 x 16, stretched in x and y
    ((22, 15, 13), (1.0, 0.7, 0.9), (1, 0, 1)),    # 21 x 14 x 12, ragged, stretched in x and z
    ((9, 10, 11), (1.0, 1.0, 1.0), (0, 0, 0)),     # 8 x 9 x 10: x shorter than a tile, ragged y
    ((70, 41, 150), (2.0, 1.0, 3.0), (0, 1, 1)),   # 69 x 40 x 149: several ragged z chunks
]


@pytest.mark.parametrize("gi", range(len(GRIDS)), ids=lambda i: "x".join(str(n - 1) for n in GRIDS[i][0]))
def test_rhs_vel_matches_oracle(gi):
    N, L, kinds = GRIDS[gi]
    og, ig = O.Grid(N, L, kinds), I.Grid(N, L, kinds)
    vel = [og.random(100 + a) for a in range(3)]
    nl0 = [og.random(200 + a) for a in range(3)]
    case = I.Case(ig, precision=0)
    for a in range(3):
        case.upload(f"vel{a + 1}", vel[a])
        case.upload(f"nl{a + 1}", nl0[a])
    case.kernel_bench(13, 1)  # work_a = interpolate_vel(vel_a) (idempotent)
    work = [og.interpolate_vel_pre(a + 1, vel[a].copy()) for a in range(3)]
    for m in range(3):
        # two launches: the second takes the first one's nl_m as the old nonlinear term
        case.kernel_bench(10 + m, 1)
        nl = og.nonlinear(m + 1, vel[m].copy(), *[w.copy() for w in work])
        og.helmholtz(m + 1, MULTL, vel[m].copy(), nl)
        rhs = vel[m] - MULT_B * nl
        rhs = rhs - MULT_A * nl
        got_nl, got_rhs = case.download(f"nl{m + 1}"), case.download(f"rhs{m + 1}")
        assert rel_err(og.interior(got_nl), og.interior(nl)) <= TOL, f"nl{m + 1}"
        assert rel_err(og.interior(got_rhs), og.interior(rhs)) <= TOL, f"rhs{m + 1}"
    case.close()
