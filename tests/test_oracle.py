"""The CPU FP64 oracle against analytic answers (CPU only, small grids)."""
import numpy as np
import pytest

import oracle as O
from impact_b200 import geometry as G


def _wave(g):
    X, Y, Z = np.meshgrid(g.xp[0][4:g.N[0] + 3], g.xp[1][4:g.N[1] + 3], g.xp[2][4:g.N[2] + 3], indexing="ij")
    f = np.sin(2 * np.pi * X / g.L[0]) * np.cos(2 * np.pi * Y / g.L[1]) * np.sin(2 * np.pi * Z / g.L[2])
    lap = -(2 * np.pi) ** 2 * (1 / g.L[0] ** 2 + 1 / g.L[1] ** 2 + 1 / g.L[2] ** 2) * f
    return f.transpose(2, 1, 0), lap.transpose(2, 1, 0)


def test_high_order_laplacian_converges_at_high_order():
    errs = []
    for n in (16, 32):
        g = O.Grid((n + 1, n + 1, n + 1))
        f, lap = _wave(g)
        phi = g.zeros()
        g.interior(phi)[...] = f
        errs.append(np.abs(g.interior(g.product_div_grad(phi)) - lap).max() / np.abs(lap).max())
    assert errs[1] < errs[0] / 30  # sixth-order stencils: ~64x per halving


def test_compact_laplacian_second_order():
    errs = []
    for n in (16, 32):
        g = O.Grid((n + 1, n + 1, n + 1))
        f, lap = _wave(g)
        phi = g.zeros()
        g.interior(phi)[...] = f
        errs.append(np.abs(g.interior(g.product_dg_relax(phi)) - lap).max() / np.abs(lap).max())
    assert 3.5 < errs[0] / errs[1] < 4.5


def test_divergence_of_gradient_equals_product_div_grad():
    g = O.Grid((17, 21, 13), (1.0, 1.3, 0.8), (1, 0, 1))
    phi = g.random(3)
    lap = g.product_div_grad(phi.copy())
    gr = [g.gradient(m, phi.copy()) for m in (1, 2, 3)]
    div = g.divergence2(gr[0], gr[1], gr[2])
    assert np.abs(g.interior(div) - g.interior(lap)).max() <= 1e-12 * np.abs(g.interior(lap)).max()


@pytest.mark.parametrize("n_sweeps", [0, 4])
def test_bicgstab_solves(n_sweeps):
    g = O.Grid((17, 17, 33), (1.0, 1.0, 2.0))
    b = g.random(4)
    g.interior(b)[...] -= g.interior(b).mean()
    x = g.zeros()
    r = g.bicgstab(b.copy(), x, tol_rel=1e-8, max_it=500, n_sweeps=n_sweeps, init_yes=True)
    assert r.status == 0 and r.res_two <= 1e-8 * r.b_two
    res = g.interior(b) - g.interior(g.product_div_grad(x.copy()))
    assert np.sqrt((res ** 2).sum()) <= 2e-8 * r.b_two


def test_time_step_vessel_runs_and_is_divergence_free():
    g = O.Grid((17, 17, 33), (1.0, 1.0, 2.0))
    lab = G.straight_vessel(g, n_in=4, n_out=4)
    vel, nl, pre = g.zeros(3), g.zeros(3), g.zeros()
    st = O.OrcStepState()
    p = O.step_params(Re=200.0)
    for _ in range(3):
        g.time_step(p, lab, vel, nl, pre, st)
        assert all(s == 0 for s in st.poisson_status)
    assert st.timestep == 3 and st.time > 0
    # the mask forcing holds the inflow buffer at the pulsatile plug velocity
    u_in = G.inflow_velocity(st.time)
    inflow = g.interior(lab) == G.INFLOW
    assert np.allclose(g.interior(vel[2])[inflow], u_in)
    assert np.all(g.interior(vel[0])[g.interior(lab) == G.SOLID] == 0.0)


def test_divergence_metric_restates_the_reference_check():
    """test_divergence (mod_test.f90:300-345): max |div2(u)| and max |div2(u) weight| with the
    weight of mod_coeffs.f90:2242-2262, checked against loops over the tables; a field whose
    components do not vary along their own axis has (discretely) zero divergence."""
    og = O.Grid((13, 11, 17), (1.0, 0.8, 1.3), (1, 1, 0))
    w = og.divergence_weight()
    for (k, j, i) in [(0, 0, 0), (5, 3, 7), (15, 9, 11)]:
        s = 0.0
        for a, q in ((0, i + 1), (1, j + 1), (2, k + 1)):
            c = og.tab["cD"][a]
            s += sum(abs(c[q * 6 + l]) for l in range(6))
        assert abs(w[k, j, i] - 1.0 / s) <= 1e-15 / s
    vel = og.random(5, n=3)
    d = og.interior(og.divergence2(vel[0], vel[1], vel[2]))
    a, b = og.test_divergence(vel)
    assert a == np.abs(d).max() and b == np.abs(d * w).max()
    free = og.zeros(3)
    rng = np.random.default_rng(6)
    N1, N2, N3 = og.N
    og.interior(free[0])[...] = rng.uniform(-1, 1, (N3 - 1, N2 - 1, 1))  # u(y, z)
    og.interior(free[1])[...] = rng.uniform(-1, 1, (N3 - 1, 1, N1 - 1))  # v(x, z)
    og.interior(free[2])[...] = rng.uniform(-1, 1, (1, N2 - 1, N1 - 1))  # w(x, y)
    for m in range(3):
        og.fill_ghosts(free[m])
    a0, b0 = og.test_divergence(free)
    assert a0 <= 1e-11 * a and b0 <= 1e-11 * b
