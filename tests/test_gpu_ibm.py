"""Immersed-boundary transfers on the device (impact_b200_case_set_markers / _ibm_interpolate /
_ibm_spread) against the oracle's restatement of interpolate_vel_to_ib and
spread_force_dens_to_vel_grid (mod_ibm.f90:428-737) on a stretched grid, with markers inside,
on the edges, outside the box and skipped:

* marker velocities bit for bit for the delta kernels built from +, -, *, / and sqrt (types 2-4)
  and within 1e-13 of the largest for the cosine kernel (type 1: the device cosine may differ
  from the host's in the last bits), in FP64 and mixed-precision cases;
* force densities within 1e-13 of the largest value (the device adds overlapping supports with
  atomics, in no fixed order), exact zeros away from every support;
* no markers: zero velocities' shape and zeroed force fields; growing the marker set; the errors
  for a reach wider than the kernels' support limit and for transfers before any markers.
"""
import numpy as np
import pytest

import impact_b200 as I
import oracle as O

pytestmark = pytest.mark.gpu

N = (17, 17, 25)
L = (1.0, 1.5, 2.0)
KINDS = (1, 0, 1)
REACH = 0.25  # about 2.7 y spacings, four x and three z spacings


def _markers(n, seed):
    rng = np.random.default_rng(seed)
    y = np.stack([rng.uniform(-0.05 * l, 1.05 * l, size=n) for l in L], axis=1)
    y[0] = [0.5, 0.75, 1.0]
    y[1] = [-1.0, 0.5, 0.5]  # outside along x: no vicinity
    return y


def _case(precision=0, seed=21):
    grid, og = I.Grid(N, L, KINDS), O.Grid(N, L, KINDS)
    case = I.Case(grid, precision=precision)
    vel = og.random(seed, n=3)
    for m in range(3):
        case.upload(f"vel{m + 1}", vel[m])
    return case, og, vel


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("dtype", [1, 2, 3, 4])
def test_marker_velocity_matches_oracle(dtype, precision):
    case, og, vel = _case(precision)
    n = 64
    yb = _markers(n, dtype)
    skip = np.zeros(n, dtype=np.uint8)
    skip[[3, 9]] = 1
    case.set_markers(yb, REACH, dtype, skip)
    got = case.ibm_interpolate()
    want = og.ibm_interpolate(yb, vel, dtype, REACH, skip)
    assert got.shape == (n, 3)
    if dtype == 1:
        assert np.max(np.abs(got - want)) <= 1e-13 * np.max(np.abs(want))
    else:
        assert np.array_equal(got, want)
    assert np.all(got[skip == 1] == 0.0) and np.all(got[1] == 0.0)
    case.close()


@pytest.mark.parametrize("dtype", [2, 4])
def test_force_density_matches_oracle(dtype):
    case, og, _ = _case()
    n = 80
    yb = _markers(n, 40 + dtype)
    rng = np.random.default_rng(dtype)
    fb = rng.uniform(-1.0, 1.0, size=(n, 3))
    vol = rng.uniform(0.5, 1.5, size=n) * 1e-3
    skip = np.zeros(n, dtype=np.uint8)
    skip[7] = 1
    case.set_markers(yb, REACH, dtype, skip)
    for into in ("rhs", "nl"):
        case.upload(f"{into}2", np.full(og.shape, 7.0))  # overwritten everywhere, ghosts included
        assert case.ibm_spread(fb, vol, into=into) == into + "1"
        fd = np.stack([case.download(f"{into}{c + 1}") for c in range(3)])
        want = og.ibm_spread(yb, fb, vol, dtype, REACH, skip)
        assert np.max(np.abs(fd - want)) <= 1e-13 * np.max(np.abs(want))
        assert np.all(fd[want == 0.0] == 0.0)
    case.close()


def test_empty_and_growing_marker_sets():
    case, og, vel = _case()
    with pytest.raises(I.ImpactError):
        case.ibm_interpolate()  # no markers yet
    case.set_markers(np.zeros((0, 3)), REACH)
    assert case.ibm_interpolate().shape == (0, 3)
    case.upload("rhs1", np.ones(og.shape))
    case.ibm_spread(np.zeros((0, 3)), np.zeros(0))
    assert not case.download("rhs1").any()
    for n in (10, 50):
        yb = _markers(n, n)
        case.set_markers(yb, REACH, 2)
        assert np.array_equal(case.ibm_interpolate(), og.ibm_interpolate(yb, vel, 2, REACH))
    with pytest.raises(I.ImpactError):
        case.set_markers(_markers(4, 1), 1.0, 2)  # a window of 2.0 holds all 24 points along z
    with pytest.raises(I.ImpactError):
        case.set_markers(_markers(4, 1), REACH, 5)  # no such delta kernel
    # a rejected set leaves the previous one in place
    assert np.array_equal(case.ibm_interpolate(), og.ibm_interpolate(_markers(50, 50), vel, 2, REACH))
    case.close()
