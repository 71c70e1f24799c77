"""Known-answer pins of the coefficient generators (CPU only).

The reference ships no test-suite; its own known answers for this path are the exact
equidistant finite-difference weights hard-coded in diff_coeffs_exact (src/mod_coeffs.f90:598-751)
and the RK3 stability limits of src/mod_vars.f90:785-795.  tests/golden/make_golden.py extracted
both as fixtures.  The oracle and the library each reproduce the weight table bit for bit, except
two rows that are a typo in the reference (see test_reference_table_typo).
"""
import json
import os

import numpy as np
import pytest

import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
FD = json.load(open(os.path.join(HERE, "golden", "fd_exact_table.json")))["rows"]
STAB = np.array(json.load(open(os.path.join(HERE, "golden", "stability_limit.json")))["values"])

# n = 7, deltaX = -1 / -5, abl = 2: the table has -225 where the Lagrange weight is -255 (its
# weights then do not sum to zero, so the row does not differentiate a constant to zero).
TYPO_ROWS = {(7, -1.0, 2), (7, -5.0, 2)}


def _rows():
    return [r for r in FD if (r["n"], r["deltaX"], r["abl"]) not in TYPO_ROWS]


def test_fixture_complete():
    assert len(FD) == 118
    assert {r["n"] for r in FD} == {2, 3, 4, 5, 6, 7}


@pytest.mark.parametrize("impl", ["oracle", "library"])
def test_fd_exact_table_bit_exact(impl):
    if impl == "oracle":
        f = O.fd_exact
    else:
        import impact_b200 as I
        f = I.fd_exact
    for r in _rows():
        want = np.array(r["num"]) / r["den"]
        got = f(r["abl"], r["n"], r["deltaX"])
        assert np.array_equal(got, want), (r["n"], r["deltaX"], r["abl"], got, want)


def test_reference_table_typo():
    for r in FD:
        if (r["n"], r["deltaX"], r["abl"]) in TYPO_ROWS:
            assert sum(r["num"]) != 0  # reference row: weights do not annihilate constants
            got = O.fd_exact(r["abl"], r["n"], r["deltaX"])
            assert abs(got.sum()) < 1e-12
            # the rows agree everywhere except the one misprinted weight
            want = np.array(r["num"]) / r["den"]
            assert np.sum(got != want) == 1


def test_stability_limits_match_reference():
    g = O.Grid((9, 9, 9))
    assert np.max(np.abs(g.stab - STAB) / STAB) < 1e-8


@pytest.mark.parametrize("kinds", [(0, 0, 0), (1, 1, 0)])
def test_library_coefficients_equal_oracle(kinds):
    import impact_b200 as I
    N, L = (33, 25, 17), (1.0, 1.0, 2.0)
    o, g = O.Grid(N, L, kinds), I.Grid(N, L, kinds)
    for a in range(3):
        assert np.array_equal(g.xp[a], o.xp[a]) and np.array_equal(g.xu[a], o.xu[a])
        for name in list(I.TABLE_WIDTH) + ["cdg"]:
            assert np.array_equal(g.tab[name][a], o.tab[name][a]), (name, a)


@pytest.mark.parametrize("kind", [0, 1])
def test_mapped_derivatives_exact_on_polynomials(kind):
    """equidistant stencils differentiate polynomials of x exactly up to their design order; the
    xi-mapped ones (mod_coeffs.f90:415-520) are exact for the linear function by construction."""
    g = O.Grid((33, 33, 33), (1.0, 1.0, 1.0), (kind, kind, kind))
    M = 33
    xp, xu = g.xp[0], g.xu[0]
    for name, xc, xe, lo, w, deg in [("cG", xp, xu, -2, 6, 5), ("cD", xu, xp, -3, 6, 5), ("cp1", xp, xp, -3, 7, 6)]:
        tab = g.tab[name][0].reshape(M + 1, w)
        for i in range(8, M - 8):  # away from the periodic seam of the stretched grid
            pts = xc[i + lo + 3: i + lo + w + 3]
            for p in range(1, (min(deg, 4) if kind == 0 else 1) + 1):
                got = tab[i] @ (pts ** p)
                want = p * xe[i + 3] ** (p - 1)
                assert abs(got - want) <= 1e-8 * max(1.0, abs(want)), (name, i, p)
