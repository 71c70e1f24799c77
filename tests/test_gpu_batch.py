"""Batched time steps: several vessel cases of different grid sizes and parameters advance
together (one launch per operator of the pressure solve over all cases) and every case must end
bit-identical to the same case stepped alone: each case's tiles, reductions and convergence
decisions are its own, whatever else is in the batch."""
import numpy as np
import pytest

import impact_b200 as I
from impact_b200 import geometry as G

pytestmark = pytest.mark.gpu

# the 22 x 20 x 40 case (n1 not divisible by 4) runs the FP32 operator's staged kernel, the others
# its vector kernel; the 19 x 20 x 40 case (n1 odd) also the FP64 operator's staged kernel (the
# FP64 batch and the mixed solve's outer residual): in a batch both kernels run, each on its own
# cases
SPECS = [((17, 17, 33), 200.0, 1.0, [(1.0, 0.5, 0.125)]),
         ((25, 21, 41), 500.0, 0.7, []),
         ((33, 33, 65), 350.0, 1.3, [(0.6, 0.4, 0.1), (1.4, 0.6, 0.15)]),
         ((23, 21, 41), 300.0, 0.9, []),
         ((20, 21, 41), 250.0, 1.1, [(1.0, 0.5, 0.1)])]


def _make(spec, precision, explicit_fp32=0):
    N, Re, U0, sten = spec
    g = I.Grid(N, (1.0, 1.0, 2.0))
    case = I.Case(g, precision=precision)
    case.set_labels(G.straight_vessel(g, stenoses=sten))
    p = I.step_params(Re=Re, U0=U0, tol_rel=1e-8, n_sweeps=4, omega=0.8, precond=1,
                      max_it=200 if precision == 0 else 30, inner_tol_rel=1e-3, explicit_fp32=explicit_fp32)
    return case, p


@pytest.mark.parametrize("precision,explicit_fp32", [(0, 0), (1, 0), (1, 1)], ids=["fp64", "mixed", "mixed-fp32-rhs"])
def test_batch_equals_alone(precision, explicit_fp32):
    nsteps = 2
    alone = []
    for spec in SPECS:
        case, p = _make(spec, precision, explicit_fp32)
        case.step(p, nsteps)
        alone.append((case, [case.download(f) for f in ("vel1", "vel2", "vel3", "pre")], case.state.dtime))
    made = [_make(spec, precision, explicit_fp32) for spec in SPECS]
    batch = I.Batch([c for c, _ in made])
    for _ in range(nsteps):
        batch.step([p for _, p in made])
    for (case, _), (_, ref, dt) in zip(made, alone):
        assert case.state.timestep == nsteps
        assert case.state.dtime == dt
        assert all(s == 0 for s in case.state.poisson_status)
        got = [case.download(f) for f in ("vel1", "vel2", "vel3", "pre")]
        for a, b in zip(got, ref):
            assert np.array_equal(a, b)
    batch.close()


def test_batch_rejects_mixed_precisions():
    a, _ = _make(SPECS[0], 0)
    b, _ = _make(SPECS[1], 1)
    with pytest.raises(I.ImpactError):
        I.Batch([a, b])


@pytest.mark.parametrize("precision,explicit_fp32", [(0, 0), (1, 1)], ids=["fp64", "mixed-fp32-rhs"])
def test_batch_rhs_depth_does_not_change_results(precision, explicit_fp32):
    """A batch's rhs_vel blocks take their z depth from the whole batch (10 planes for these three
    cases together, 8 for each alone): the pass's arithmetic per point does not depend on it."""
    specs = [((129, 129, 257), 400.0, 1.0, [(1.0, 0.5, 0.1)]),
             ((97, 97, 193), 300.0, 0.8, []),
             ((65, 65, 129), 500.0, 1.2, [(0.8, 0.4, 0.1)])]
    alone = []
    for spec in specs:
        case, p = _make(spec, precision, explicit_fp32)
        case.step(p, 1)
        alone.append([case.download(f) for f in ("vel1", "vel2", "vel3", "pre")])
        case.close()
    made = [_make(spec, precision, explicit_fp32) for spec in specs]
    batch = I.Batch([c for c, _ in made])
    batch.step([p for _, p in made])
    for (case, _), ref in zip(made, alone):
        assert all(s == 0 for s in case.state.poisson_status)
        for a, b in zip([case.download(f) for f in ("vel1", "vel2", "vel3", "pre")], ref):
            assert np.array_equal(a, b)
    batch.close()
