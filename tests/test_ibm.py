"""Immersed-boundary transfers (mod_ibm.f90) on the CPU: the arithmetic the device kernels use
(gpu-impact-ct_b200/csrc/ibm.cuh, compiled here for the host from the same source by
tests/ibm_host.cpp) against the oracle's literal restatement of discrete_delta,
find_vicinity_coordinates, interpolate_vel_to_ib and spread_force_dens_to_vel_grid:

* the four delta kernels bit for bit at distances across their pieces and edges, and the
  partition of unity of the hat (type 2) and four-point (type 4) kernels on a uniform grid;
* the binary-search vicinity equals the reference's linear scan, also for positions on grid
  points, exactly one reach away and outside the domain;
* marker velocities and spread force densities bit for bit on a stretched grid with markers
  inside, at the edges, outside (empty vicinity) and skipped, for every delta type;
* the transfers are adjoint: sum(fd u dV) = sum(fb vol ub);
* the support bound that set_markers enforces.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N = (17, 13, 21)
L = (1.0, 1.5, 2.0)
KINDS = (1, 0, 1)

_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    out = tmp_path_factory.mktemp("ibm") / "libibm_host.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared",
                    "-I", os.path.join(ROOT, "gpu-impact-ct_b200", "csrc"),
                    os.path.join(ROOT, "tests", "ibm_host.cpp"), "-o", str(out)], check=True)
    lib = C.CDLL(str(out))
    i, d = C.c_int, C.c_double
    lib.host_ibm_delta.restype, lib.host_ibm_delta.argtypes = d, [i, d, d]
    lib.host_ibm_vicinity.restype = None
    lib.host_ibm_vicinity.argtypes = [_dp, i, d, d, C.POINTER(i), C.POINTER(i)]
    lib.host_ibm_widest.restype, lib.host_ibm_widest.argtypes = i, [i, _dp, _dp, d]
    lib.host_ibm_interpolate.restype = i
    lib.host_ibm_interpolate.argtypes = [i, i, i, C.POINTER(_dp), C.POINTER(_dp), i, d, i, _dp, _u8p, _dp, _dp]
    lib.host_ibm_spread.restype = i
    lib.host_ibm_spread.argtypes = [i, i, i, C.POINTER(_dp), C.POINTER(_dp), i, d, i, _dp, _u8p, _dp, _dp, _dp]
    return lib


def _p(a):
    return a.ctypes.data_as(_dp)


def _markers(grid, n, seed):
    """Markers spread over the box and a little beyond, a few on grid points and one reach
    from a grid point; returns (n, 3) positions."""
    rng = np.random.default_rng(seed)
    y = np.stack([rng.uniform(-0.05 * l, 1.05 * l, size=n) for l in grid.L], axis=1)
    y[0] = [grid.xp[0][5], grid.xu[1][7], grid.xp[2][9]]      # on grid points
    y[1] = [grid.xu[0][4 + 3] + 0.0, grid.xp[1][3 + 3], 0.5 * grid.L[2]]
    y[2] = [-1.0, 0.5, 0.5]                                    # outside along x
    y[3] = [grid.xp[0][1 + 3], grid.xp[1][1 + 3], grid.xp[2][1 + 3]]  # first points
    return y


def _host_call(host, grid, fn, *args):
    xp = (_dp * 3)(*[_p(a) for a in grid.xp])
    xu = (_dp * 3)(*[_p(a) for a in grid.xu])
    return getattr(host, fn)(*grid.N, xp, xu, *args)


@pytest.mark.parametrize("dtype", [1, 2, 3, 4])
def test_delta_kernels_match(host, dtype):
    lb = O.lib()
    reach = 0.0371
    ds = np.concatenate([np.linspace(-1.2 * reach, 1.2 * reach, 997),
                         [0.0, reach, -reach, reach / 2, -reach / 2, np.nextafter(reach, 1.0),
                          np.nextafter(reach / 2, 0.0), 3.0]])
    for d in ds:
        want = lb.orc_ibm_delta(dtype, reach, float(d))
        got = host.host_ibm_delta(dtype, reach, float(d))
        assert got == want or (np.isnan(got) and np.isnan(want)), (dtype, d, got, want)


@pytest.mark.parametrize("dtype,reach_h", [(2, 1.0), (4, 2.0)])
def test_partition_of_unity(host, dtype, reach_h):
    h = 0.01
    x = np.arange(-20, 21) * h
    for y in np.linspace(0.0, h, 13):
        s = sum(host.host_ibm_delta(dtype, reach_h * h, float(y - xi)) for xi in x) * h
        assert abs(s - 1.0) < 1e-12, (dtype, y, s)


def _scan(x, n, y, reach):
    """find_vicinity_coordinates along one axis, as the reference loops (points 1..n, x[i])."""
    for i in range(1, n + 1):
        if abs(y - x[i]) <= reach:
            for j in range(i, n + 1):
                if x[j] - y > reach:
                    return i, j - 1
                if j == n:
                    return i, j
    return -1, -1


def test_vicinity_is_the_linear_scan(host):
    grid = O.Grid(N, L, KINDS)
    rng = np.random.default_rng(5)
    for a in range(3):
        n = N[a] - 1
        for x in (grid.xp[a][3:], grid.xu[a][3:]):
            x = np.ascontiguousarray(x[:n + 1])
            reach = 2.3 * (x[2] - x[1])
            ys = list(rng.uniform(x[1] - 3 * reach, x[n] + 3 * reach, size=200))
            ys += [x[1], x[n], x[5], x[5] + reach, x[5] - reach, x[1] - reach, x[n] + reach, -50.0, 50.0]
            for y in ys:
                lo, hi = C.c_int(), C.c_int()
                host.host_ibm_vicinity(_p(x), n, float(y), reach, C.byref(lo), C.byref(hi))
                assert (lo.value, hi.value) == _scan(x, n, y, reach), (a, y)


@pytest.mark.parametrize("dtype", [1, 2, 3, 4])
def test_interpolate_and_spread_bit_for_bit(host, dtype):
    grid = O.Grid(N, L, KINDS)
    n = 40
    yb = _markers(grid, n, 7 + dtype)
    skip = np.zeros(n, dtype=np.uint8)
    skip[[5, 11]] = 1
    reach = 0.25  # two y spacings, about four x and three z spacings
    vel = grid.random(3, n=3)
    want = grid.ibm_interpolate(yb, vel, dtype, reach, skip)
    flat = np.ascontiguousarray(yb.T)
    ub = np.zeros((3, n))
    wide = _host_call(host, grid, "host_ibm_interpolate", dtype, reach, n, _p(flat),
                      skip.ctypes.data_as(_u8p), _p(vel), _p(ub))
    assert wide == 0
    assert np.array_equal(ub.T, want)
    assert np.all(want[skip == 1] == 0.0) and np.all(want[2] == 0.0)  # skipped; outside
    assert np.count_nonzero(want) > 2 * n  # most markers see the grid
    rng = np.random.default_rng(dtype)
    fb = rng.uniform(-1.0, 1.0, size=(n, 3))
    vol = rng.uniform(0.5, 1.5, size=n) * 1e-3
    fd_want = grid.ibm_spread(yb, fb, vol, dtype, reach, skip)
    fd = grid.zeros(3)
    wide = _host_call(host, grid, "host_ibm_spread", dtype, reach, n, _p(flat), skip.ctypes.data_as(_u8p),
                      _p(np.ascontiguousarray(fb.T)), _p(vol), _p(fd))
    assert wide == 0
    assert np.array_equal(fd, fd_want)
    assert np.count_nonzero(fd_want) > 0


def test_transfers_are_adjoint():
    grid = O.Grid(N, L, KINDS)
    n = 30
    yb = _markers(grid, n, 3)
    reach = 2.0 * L[0] / (N[0] - 1)
    vel = grid.random(11, n=3)
    rng = np.random.default_rng(12)
    fb = rng.uniform(-1.0, 1.0, size=(n, 3))
    vol = rng.uniform(0.5, 1.5, size=n)
    ub = grid.ibm_interpolate(yb, vel, 4, reach)
    fd = grid.ibm_spread(yb, fb, vol, 4, reach)
    lhs = 0.0
    for c in range(3):
        w = []
        for a in range(3):
            i = np.arange(1, N[a]) + 3  # storage index of points 1..N-1
            # cell widths: dxu(i) = xp(i+1) - xp(i) along the component's own axis, else
            # dxp(i) = xu(i) - xu(i-1)
            w.append(grid.xp[a][i + 1] - grid.xp[a][i] if a == c else grid.xu[a][i] - grid.xu[a][i - 1])
        dV = w[2][:, None, None] * w[1][None, :, None] * w[0][None, None, :]
        lhs += np.sum(grid.interior(fd[c]) * grid.interior(vel[c]) * dV)
    rhs = np.sum(fb * vol[:, None] * ub)
    assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(rhs))


def test_support_bound(host):
    grid = O.Grid((33, 33, 33), (1.0, 1.0, 1.0), (0, 0, 0))
    h = 1.0 / 32
    xp, xu = grid.xp[0], grid.xu[0]
    assert host.host_ibm_widest(33, _p(xp), _p(xu), 2.0 * h) == 5
    assert host.host_ibm_widest(33, _p(xp), _p(xu), 7.4 * h) == 15
    assert host.host_ibm_widest(33, _p(xp), _p(xu), 8.0 * h) == 17  # rejected by set_markers (> 16)
