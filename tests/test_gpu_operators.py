"""Parity of every reference launcher (src/*_launcher.cu FFI) against the CPU FP64 oracle.

Each test builds a grid (equidistant or sinh-stretched, sizes divisible by 8 and ragged ones),
fills the fields with seeded U[-1, 1] values, runs the library's launcher on device buffers
through the C ABI, and compares the unique periodic points with the oracle's restatement of the
CPU routine (mod_diff.f90, mod_laplace.f90).  FP64 bar: max |gpu - cpu| / max |cpu| <= 1e-12.
"""
import numpy as np
import pytest

import oracle as O
import impact_b200 as I
from _util import dev, host, ptr, rel_err

TOL = 1e-12
GRIDS = [
    ((17, 17, 33), (1.0, 1.0, 2.0), (0, 0, 0)),   # 16 x 16 x 32, equidistant
    ((33, 25, 17), (1.0, 1.0, 1.0), (1, 1, 0)),   # 32 x 24 x 16, stretched in x and y
    ((22, 15, 13), (1.0, 0.7, 0.9), (1, 0, 1)),   # 21 x 14 x 12, ragged sizes
]


@pytest.fixture(params=range(len(GRIDS)), ids=lambda i: "x".join(str(n - 1) for n in GRIDS[i][0]))
def grids(request):
    N, L, kinds = GRIDS[request.param]
    return O.Grid(N, L, kinds), I.Grid(N, L, kinds)


def _dims(og):
    N1, N2, N3 = og.N
    return N1 + 7, N2 + 7, N3 + 7


def _tab(ig, name, a):
    return dev(ig.tab[name][a])


pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m", [1, 2, 3])
def test_gradient(grids, m):
    og, ig = grids
    nx, ny, nz = _dims(og)
    phi = og.random(10 + m)
    want = og.gradient(m, phi.copy())
    d_phi, d_out, d_c = dev(phi), dev(og.zeros()), _tab(ig, "cG", m - 1)
    I.launchers.call("gradient_launcher_", ("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 6),
                     ("i", og.N[m - 1] + 1), ("p", ptr(d_phi)), ("p", ptr(d_c)), ("p", ptr(d_out)))
    assert rel_err(og.interior(host(d_out)), og.interior(want)) <= TOL


@pytest.mark.parametrize("m", [1, 2, 3])
def test_divergence(grids, m):
    og, ig = grids
    nx, ny, nz = _dims(og)
    phi = og.random(20 + m)
    div0 = og.random(30 + m)  # m = 2, 3 accumulate into the existing values
    want = og.divergence(m, phi.copy(), div0.copy())
    d_phi, d_div, d_c = dev(phi), dev(div0), _tab(ig, "cD", m - 1)
    I.launchers.call("divergence_launcher_", ("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 6),
                     ("i", og.N[m - 1] + 1), ("p", ptr(d_phi)), ("p", ptr(d_div)), ("p", ptr(d_c)))
    assert rel_err(og.interior(host(d_div)), og.interior(want)) <= TOL


def test_divergence2(grids):
    og, ig = grids
    nx, ny, nz = _dims(og)
    vel = og.random(40, n=3)
    want = og.divergence2(vel[0].copy(), vel[1].copy(), vel[2].copy())
    d_vel, d_div = dev(vel), dev(og.zeros())
    c = [_tab(ig, "cD", a) for a in range(3)]
    I.launchers.call("divergence2_launcher_", ("i", nx), ("i", ny), ("i", nz), ("i", 6), ("i", 6), ("i", 6),
                     ("p", ptr(d_vel)), ("p", ptr(d_div)), ("p", ptr(c[0])), ("p", ptr(c[1])), ("p", ptr(c[2])))
    assert rel_err(og.interior(host(d_div)), og.interior(want)) <= TOL


@pytest.mark.parametrize("m", [1, 2, 3])
def test_helmholtz(grids, m):
    og, ig = grids
    nx, ny, nz = _dims(og)
    vel = og.random(50 + m)
    nl = og.random(60 + m)
    multL = 1e-3
    want = og.helmholtz(m, multL, vel.copy(), nl.copy())
    names = [("cuu" if a == m - 1 else "cpp") for a in range(3)]
    c = [_tab(ig, names[a], a) for a in range(3)]
    d_vel, d_nl = dev(vel), dev(nl)
    I.launchers.call("helmholtz_explicit_launcher_", ("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 7), ("i", 7),
                     ("i", 7), ("d", multL), ("p", ptr(d_vel)), ("p", ptr(d_nl)), ("p", ptr(c[0])),
                     ("p", ptr(c[1])), ("p", ptr(c[2])))
    assert rel_err(og.interior(host(d_nl)), og.interior(want)) <= TOL


@pytest.mark.parametrize("m", [1, 2, 3])
def test_interpolate_pre_vel(grids, m):
    og, ig = grids
    nx, ny, nz = _dims(og)
    phi = og.random(70 + m)
    want = og.interpolate_pre_vel(m, phi.copy())
    d_phi, d_out, d_c = dev(phi), dev(og.zeros()), _tab(ig, "cIpu", m - 1)
    I.launchers.call("interpolate2_pre_vel_launcher_", ("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 6),
                     ("i", og.N[m - 1] + 1), ("p", ptr(d_phi)), ("p", ptr(d_c)), ("p", ptr(d_out)))
    assert rel_err(og.interior(host(d_out)), og.interior(want)) <= TOL


@pytest.mark.parametrize("m", [1, 2, 3])
def test_interpolate_vel_pre(grids, m):
    og, ig = grids
    nx, ny, nz = _dims(og)
    phi = og.random(80 + m)
    want = og.interpolate_vel_pre(m, phi.copy())
    d_phi, d_out, d_c = dev(phi), dev(og.zeros()), _tab(ig, "cIup", m - 1)
    I.launchers.call("interpolate2_vel_pre_launcher_", ("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 6),
                     ("i", og.N[m - 1] + 1), ("p", ptr(d_phi)), ("p", ptr(d_c)), ("p", ptr(d_out)))
    assert rel_err(og.interior(host(d_out)), og.interior(want)) <= TOL


@pytest.mark.parametrize("cid", range(1, 10))
def test_nonlinear_upwind(grids, cid):
    og, ig = grids
    nx, ny, nz = _dims(og)
    m, a = (cid - 1) // 3 + 1, (cid - 1) % 3 + 1
    vel = og.random(90 + cid)
    pp = og.random(100 + cid)  # mixed signs exercise both upwind tables
    nl = og.random(110 + cid)
    want = og.nonlinear_upwind(cid, pp.copy(), vel.copy(), nl.copy())
    up, dn = ("cNuU", "cNuD") if a == m else ("cNpU", "cNpD")
    cU, cD = _tab(ig, up, a - 1), _tab(ig, dn, a - 1)
    d_vel, d_pp, d_nl = dev(vel), dev(pp), dev(nl)
    I.launchers.call("nonlinear_upwind_launcher_", ("i", cid), ("i", nx), ("i", ny), ("i", nz), ("i", 7),
                     ("i", og.N[a - 1] + 1), ("p", ptr(d_pp)), ("p", ptr(d_vel)), ("p", ptr(d_nl)),
                     ("p", ptr(cU)), ("p", ptr(cD)))
    assert rel_err(og.interior(host(d_nl)), og.interior(want)) <= TOL


def test_axpby(grids):
    og, _ = grids
    nx, ny, nz = _dims(og)
    x, y = og.random(120), og.random(121)
    want = og.axpby(1.0, -1.0, x, y, og.zeros())
    d_x, d_y, d_z = dev(x), dev(y), dev(og.zeros())
    I.launchers.call("axpby_launcher_", ("i", nx), ("i", ny), ("i", nz), ("d", 1.0), ("d", -1.0),
                     ("p", ptr(d_x)), ("p", ptr(d_y)), ("p", ptr(d_z)))
    assert np.array_equal(og.interior(host(d_z)), og.interior(want))


def test_product_dg_relax(grids):
    og, ig = grids
    nx, ny, nz = _dims(og)
    x = og.random(130)
    want = og.product_dg_relax(x.copy())
    c = [_tab(ig, "cdg", a) for a in range(3)]
    d_x, d_out = dev(x), dev(og.zeros())
    I.launchers.call("product_dg_relax_launcher_", ("i", 1), ("i", nx), ("i", ny), ("i", nz), ("i", og.N[0]),
                     ("i", og.N[1]), ("i", og.N[2]), ("i", 3), ("p", ptr(c[0])), ("p", ptr(c[1])),
                     ("p", ptr(c[2])), ("p", ptr(d_x)), ("p", ptr(d_out)))
    assert rel_err(og.interior(host(d_out)), og.interior(want)) <= TOL


def test_jacobi(grids):
    og, ig = grids
    nx, ny, nz = _dims(og)
    bb, rel = og.random(140), og.random(141)
    want = og.jacobi(bb.copy(), rel.copy(), 2, 0.98, init_yes=False)  # r = 1 is a plain sweep as well
    c = [_tab(ig, "cdg", a) for a in range(3)]
    d_bb, d_rel, d_comp = dev(bb), dev(rel), dev(og.zeros())
    for _ in range(2):
        I.launchers.call("jacobi_launcher_", ("i", 1), ("i", nx), ("i", ny), ("i", nz), ("i", og.N[0]),
                         ("i", og.N[1]), ("i", og.N[2]), ("i", 3), ("d", 0.98), ("p", ptr(c[0])), ("p", ptr(c[1])),
                         ("p", ptr(c[2])), ("p", ptr(d_rel)), ("p", ptr(d_bb)), ("p", ptr(d_comp)))
        d_rel, d_comp = d_comp, d_rel
    assert rel_err(og.interior(host(d_rel)), og.interior(want)) <= TOL


def _faces(og, rel):
    """ghost faces exactly as the host builds them for a periodic single block
    (jacobi_solver_host_v4.f90:257-269 after exchange_relax_GPU)."""
    N1, N2, N3 = og.N
    n1, n2, n3 = N1 - 1, N2 - 1, N3 - 1
    r = og.interior(rel)  # (k, j, i)
    west = np.ascontiguousarray(r[:, :, n1 - 1])     # i = 0 ghost = plane n1, layout (j-1) + n2 (k-1)
    east = np.ascontiguousarray(r[:, :, 0])
    lower = np.ascontiguousarray(r[:, n2 - 1, :])    # (i-1) + n1 (k-1)
    upper = np.ascontiguousarray(r[:, 0, :])
    rear = np.ascontiguousarray(r[n3 - 1, :, :])     # (i-1) + n1 (j-1)
    front = np.ascontiguousarray(r[0, :, :])
    return rear, front, upper, lower, west, east


def test_jor_launcher_and_get_ghost(grids):
    og, ig = grids
    nx, ny, nz = _dims(og)
    bb, rel = og.random(150), og.random(151)
    want = og.jacobi(bb.copy(), rel.copy(), 1, 0.8, init_yes=False)  # one deterministic JOR sweep
    c = [_tab(ig, "cdg", a) for a in range(3)]
    faces = [dev(f) for f in _faces(og, rel)]
    d_bb, d_rel = dev(bb), dev(rel)
    I.launchers.call("jor_launcher_", ("i", 1), ("i", nx), ("i", ny), ("i", nz), ("i", og.N[0]), ("i", og.N[1]),
                     ("i", og.N[2]), ("i", 3), ("d", 0.8), ("p", ptr(c[0])), ("p", ptr(c[1])), ("p", ptr(c[2])),
                     ("p", ptr(d_rel)), ("p", ptr(d_bb)), *[("p", ptr(f)) for f in faces])
    got = host(d_rel)
    assert rel_err(og.interior(got), og.interior(want)) <= TOL
    # get_ghost copies the boundary planes of the new rel into the face arrays
    I.launchers.call("get_ghost_launcher_", ("i", nx), ("i", ny), ("i", nz), ("p", ptr(d_rel)),
                     *[("p", ptr(f)) for f in faces])
    r = og.interior(got)
    rear, front, upper, lower, west, east = [host(f) for f in faces]
    assert np.array_equal(rear, r[0]) and np.array_equal(front, r[-1])
    assert np.array_equal(lower, r[:, 0, :]) and np.array_equal(upper, r[:, -1, :])
    assert np.array_equal(west, r[:, :, 0]) and np.array_equal(east, r[:, :, -1])


def test_pressure_bc(grids):
    og, _ = grids
    nx, ny, nz = _dims(og)
    rng = np.random.default_rng(160)
    lab = np.zeros(og.shape, dtype=np.uint8)
    og.interior(lab)[...] = rng.choice(np.array([0, 1, 5, 9, 11], dtype=np.uint8), size=og.interior(lab).shape)
    rel = og.random(161)
    ks = 4
    want = og.pressure_bc(lab, ks, 1.5, -0.5, 0.25, rel.copy())
    d_lab, d_rel = dev(lab.astype(np.float64)), dev(rel)
    I.launchers.call("pressure_bc_launcher_", ("i", 1), ("i", 1), ("i", 1), ("i", ks), ("i", nx), ("i", ny),
                     ("i", nz), ("d", 1.5), ("d", -0.5), ("d", 0.25), ("p", ptr(d_lab)), ("p", ptr(d_rel)))
    assert np.array_equal(og.interior(host(d_rel)), og.interior(want))


def test_product_scalar(grids):
    og, _ = grids
    a, b = og.random(170), og.random(171)
    want = og.dot(a, b)
    d_a, d_b = dev(a), dev(b)
    got = I.product_scalar(og.N, ptr(d_a), ptr(d_b))
    assert abs(got - want) <= 1e-12 * np.sqrt(og.dot(a, a) * og.dot(b, b))
    # deterministic: identical bits on a second call
    assert I.product_scalar(og.N, ptr(d_a), ptr(d_b)) == got


def test_launcher_rejects_bad_sizes():
    d = dev(np.zeros(8))
    with pytest.raises(I.ImpactError):
        I.launchers.call("gradient_launcher_", ("i", 1), ("i", 10), ("i", 10), ("i", 10), ("i", 6), ("i", 4),
                         ("p", ptr(d)), ("p", ptr(d)), ("p", ptr(d)))
