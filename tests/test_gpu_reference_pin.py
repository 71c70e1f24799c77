"""Pin the oracle to the reference's own implementation.

oracle/build_ref.sh compiles GPU-IMPACT-CT's CUDA operator kernels (src/*_launcher.cu with their
*_kernel.cu, unchanged) into oracle/_ref/libref_kernels.so.  Each reference launcher runs on the
same seeded inputs (ghost layers filled by the periodic exchange, as the Fortran host does before
every call) and its output must equal the oracle's restatement of the CPU routine to 1e-12.
The reference kernels require interior sizes divisible by 8 (jor_kernel_launcher.cu:18-33).
Skipped when the reference library was not built.
"""
import ctypes as C
import os

import numpy as np
import pytest

import oracle as O
import impact_b200 as I
from _util import dev, host, ptr, rel_err

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref", "libref_kernels.so")
TOL = 1e-12


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(REF):
        pytest.skip("oracle/_ref/libref_kernels.so not built (oracle/build_ref.sh)")
    return C.CDLL(REF)


def call(lib, name, *args):
    keep, conv = [], []
    for kind, v in args:
        o = C.c_int(int(v)) if kind == "i" else (C.c_double(float(v)) if kind == "d" else C.c_void_p(int(v)))
        keep.append(o)
        conv.append(C.byref(o))
    getattr(lib, name)(*conv)
    import torch
    torch.cuda.synchronize()


GRIDS = [((17, 17, 33), (1.0, 1.0, 2.0), (0, 0, 0)), ((33, 25, 17), (1.0, 1.0, 1.0), (1, 1, 0))]


@pytest.fixture(params=range(len(GRIDS)), ids=["16x16x32", "32x24x16-stretched"])
def grids(request):
    N, L, kinds = GRIDS[request.param]
    return O.Grid(N, L, kinds), I.Grid(N, L, kinds)


def _dims(og):
    return tuple(n + 7 for n in og.N)


def _ghosted(og, seed, n=None):
    a = og.random(seed, n=n)
    if n is None:
        og.fill_ghosts(a)
    else:
        for q in range(n):
            og.fill_ghosts(a[q])
    return a


@pytest.mark.parametrize("m", [1, 2, 3])
def test_gradient_pin(ref, grids, m):
    og, ig = grids
    nx, ny, nz = _dims(og)
    phi = _ghosted(og, 1 + m)
    want = og.gradient(m, phi.copy())
    d_phi, d_out, d_c = dev(phi), dev(og.zeros()), dev(ig.tab["cG"][m - 1])
    call(ref, "gradient_launcher_", ("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 6), ("i", og.N[m - 1] + 1),
         ("p", ptr(d_phi)), ("p", ptr(d_c)), ("p", ptr(d_out)))
    assert rel_err(og.interior(host(d_out)), og.interior(want)) <= TOL


@pytest.mark.parametrize("m", [1, 2, 3])
def test_divergence_pin(ref, grids, m):
    og, ig = grids
    nx, ny, nz = _dims(og)
    phi, div0 = _ghosted(og, 10 + m), og.random(20 + m)
    want = og.divergence(m, phi.copy(), div0.copy())
    d_phi, d_div, d_c = dev(phi), dev(div0), dev(ig.tab["cD"][m - 1])
    call(ref, "divergence_launcher_", ("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 6), ("i", og.N[m - 1] + 1),
         ("p", ptr(d_phi)), ("p", ptr(d_div)), ("p", ptr(d_c)))
    assert rel_err(og.interior(host(d_div)), og.interior(want)) <= TOL


def test_divergence2_pin(ref, grids):
    og, ig = grids
    nx, ny, nz = _dims(og)
    vel = _ghosted(og, 30, n=3)
    want = og.divergence2(vel[0].copy(), vel[1].copy(), vel[2].copy())
    d_vel, d_div = dev(vel), dev(og.zeros())
    c = [dev(ig.tab["cD"][a]) for a in range(3)]
    call(ref, "divergence2_launcher_", ("i", nx), ("i", ny), ("i", nz), ("i", 6), ("i", 6), ("i", 6),
         ("p", ptr(d_vel)), ("p", ptr(d_div)), ("p", ptr(c[0])), ("p", ptr(c[1])), ("p", ptr(c[2])))
    assert rel_err(og.interior(host(d_div)), og.interior(want)) <= TOL


@pytest.mark.parametrize("m", [1, 2, 3])
def test_helmholtz_pin(ref, grids, m):
    og, ig = grids
    nx, ny, nz = _dims(og)
    vel, nl = _ghosted(og, 40 + m), og.random(50 + m)
    want = og.helmholtz(m, 1e-3, vel.copy(), nl.copy())
    c = [dev(ig.tab["cuu" if a == m - 1 else "cpp"][a]) for a in range(3)]
    d_vel, d_nl = dev(vel), dev(nl)
    call(ref, "helmholtz_explicit_launcher_", ("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 7), ("i", 7), ("i", 7),
         ("d", 1e-3), ("p", ptr(d_vel)), ("p", ptr(d_nl)), ("p", ptr(c[0])), ("p", ptr(c[1])), ("p", ptr(c[2])))
    assert rel_err(og.interior(host(d_nl)), og.interior(want)) <= TOL


@pytest.mark.parametrize("cid", range(1, 10))
def test_nonlinear_upwind_pin(ref, grids, cid):
    og, ig = grids
    nx, ny, nz = _dims(og)
    m, a = (cid - 1) // 3 + 1, (cid - 1) % 3 + 1
    vel, pp, nl = _ghosted(og, 60 + cid), og.random(70 + cid), og.random(80 + cid)
    want = og.nonlinear_upwind(cid, pp.copy(), vel.copy(), nl.copy())
    up, dn = ("cNuU", "cNuD") if a == m else ("cNpU", "cNpD")
    cU, cD = dev(ig.tab[up][a - 1]), dev(ig.tab[dn][a - 1])
    d_vel, d_pp, d_nl = dev(vel), dev(pp), dev(nl)
    call(ref, "nonlinear_upwind_launcher_", ("i", cid), ("i", nx), ("i", ny), ("i", nz), ("i", 7),
         ("i", og.N[a - 1] + 1), ("p", ptr(d_pp)), ("p", ptr(d_vel)), ("p", ptr(d_nl)), ("p", ptr(cU)), ("p", ptr(cD)))
    assert rel_err(og.interior(host(d_nl)), og.interior(want)) <= TOL


@pytest.mark.parametrize("m", [1, 2, 3])
def test_interpolations_pin(ref, grids, m):
    og, ig = grids
    nx, ny, nz = _dims(og)
    phi = _ghosted(og, 90 + m)
    for name, tab, f in (("interpolate2_pre_vel_launcher_", "cIpu", og.interpolate_pre_vel),
                         ("interpolate2_vel_pre_launcher_", "cIup", og.interpolate_vel_pre)):
        want = f(m, phi.copy())
        d_phi, d_out, d_c = dev(phi), dev(og.zeros()), dev(ig.tab[tab][m - 1])
        call(ref, name, ("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 6), ("i", og.N[m - 1] + 1),
             ("p", ptr(d_phi)), ("p", ptr(d_c)), ("p", ptr(d_out)))
        assert rel_err(og.interior(host(d_out)), og.interior(want)) <= TOL, name


def test_jacobi_and_dg_relax_pin(ref, grids):
    og, ig = grids
    nx, ny, nz = _dims(og)
    bb, rel = og.random(100), _ghosted(og, 101)
    c = [dev(ig.tab["cdg"][a]) for a in range(3)]
    want = og.jacobi(bb.copy(), rel.copy(), 1, 0.98, init_yes=False)
    d_bb, d_rel, d_comp = dev(bb), dev(rel), dev(og.zeros())
    call(ref, "jacobi_launcher_", ("i", 1), ("i", nx), ("i", ny), ("i", nz), ("i", og.N[0]), ("i", og.N[1]),
         ("i", og.N[2]), ("i", 3), ("d", 0.98), ("p", ptr(c[0])), ("p", ptr(c[1])), ("p", ptr(c[2])),
         ("p", ptr(d_rel)), ("p", ptr(d_bb)), ("p", ptr(d_comp)))
    assert rel_err(og.interior(host(d_comp)), og.interior(want)) <= TOL
    want = og.product_dg_relax(rel.copy())
    d_out = dev(og.zeros())
    call(ref, "product_dg_relax_launcher_", ("i", 1), ("i", nx), ("i", ny), ("i", nz), ("i", og.N[0]),
         ("i", og.N[1]), ("i", og.N[2]), ("i", 3), ("p", ptr(c[0])), ("p", ptr(c[1])), ("p", ptr(c[2])),
         ("p", ptr(d_rel)), ("p", ptr(d_out)))
    assert rel_err(og.interior(host(d_out)), og.interior(want)) <= TOL


def test_axpby_pin(ref, grids):
    og, _ = grids
    nx, ny, nz = _dims(og)
    x, y = og.random(110), og.random(111)
    want = og.axpby(1.0, -1.0, x, y, og.zeros())
    d_x, d_y, d_z = dev(x), dev(y), dev(og.zeros())
    call(ref, "axpby_launcher_", ("i", nx), ("i", ny), ("i", nz), ("d", 1.0), ("d", -1.0), ("p", ptr(d_x)),
         ("p", ptr(d_y)), ("p", ptr(d_z)))
    assert np.array_equal(og.interior(host(d_z)), og.interior(want))


def test_pressure_bc_pin_plane_offset(ref, grids):
    """set_pressure_BC_kernel.cu tests the C index (k+4) against k_start_index-1 while the CPU
    routine tests the Fortran index; the reference GPU plane therefore sits 3 planes below the
    CPU one.  The oracle (and this library) follow the CPU routine; the pin checks the offset."""
    og, _ = grids
    nx, ny, nz = _dims(og)
    rng = np.random.default_rng(120)
    lab = np.zeros(og.shape, dtype=np.uint8)
    og.interior(lab)[...] = rng.choice(np.array([0, 1, 5, 9], dtype=np.uint8), size=og.interior(lab).shape)
    rel = og.random(121)
    ks = 6
    want = og.pressure_bc(lab, ks, 1.5, -0.5, 0.25, rel.copy())
    d_lab, d_rel = dev(lab.astype(np.float64)), dev(rel)
    call(ref, "pressure_bc_launcher_", ("i", 1), ("i", 1), ("i", 0), ("i", ks + 3), ("i", nx), ("i", ny), ("i", nz),
         ("d", 1.5), ("d", -0.5), ("d", 0.25), ("p", ptr(d_lab)), ("p", ptr(d_rel)))
    assert np.array_equal(og.interior(host(d_rel)), og.interior(want))


def test_pressure_bc_reference_gpu_plane_switch(ref, grids):
    """With impact_b200_set_pressure_bc_plane(1) this library's pressure_bc_launcher_ sets the plane
    the reference GPU kernel sets: both called with the same k_start_index give the same field."""
    og, _ = grids
    nx, ny, nz = _dims(og)
    rng = np.random.default_rng(122)
    lab = np.zeros(og.shape, dtype=np.uint8)
    og.interior(lab)[...] = rng.choice(np.array([0, 1, 5, 9, 11], dtype=np.uint8), size=og.interior(lab).shape)
    rel = og.random(123)
    ks = 9
    d_lab = dev(lab.astype(np.float64))
    d_ref, d_own = dev(rel), dev(rel)
    args = [("i", 1), ("i", 1), ("i", 1), ("i", ks), ("i", nx), ("i", ny), ("i", nz), ("d", 1.5), ("d", -0.5),
            ("d", 0.25), ("p", ptr(d_lab))]
    call(ref, "pressure_bc_launcher_", *args, ("p", ptr(d_ref)))
    I.set_pressure_bc_plane(1)
    try:
        I.launchers.call("pressure_bc_launcher_", *args, ("p", ptr(d_own)))
        I.launchers.sync()
    finally:
        I.set_pressure_bc_plane(0)
    assert np.array_equal(og.interior(host(d_own)), og.interior(host(d_ref)))
    assert not np.array_equal(og.interior(host(d_own)), og.interior(rel))  # the condition set something
