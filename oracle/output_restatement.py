"""Literal CPU restatement of the reference's lambda-2 output field, the checker for
impact_b200.xdmf.lambda2.

TEST INFRASTRUCTURE ONLY: imported by tests/.  Plain Python loops in the order of `lambda`
(mod_inout.f90:2827-3008) over the oracle's velocity interpolation (interpolate_vel_pre) and
its cp1 tables, for small grids.  Parity unpinned: the routine is Fortran and no Fortran
compiler is in this image.
"""
from __future__ import annotations

import math


def lambda2(og, vel):
    """res(i, j, k) of `lambda` for the velocity fields vel (3, padded shape) on oracle grid og;
    returns {(i, j, k): value} over the unique periodic points."""
    N1, N2, N3 = og.N
    nl = [og.interpolate_vel_pre(m, vel[m - 1].copy()) for m in (1, 2, 3)]
    cp = og.tab["cp1"]

    def nlv(c, i, j, k):  # exchange_all_all: periodic wrap of the unique points 1..N-1
        i = (i - 1) % (N1 - 1) + 1
        j = (j - 1) % (N2 - 1) + 1
        k = (k - 1) % (N3 - 1) + 1
        return nl[c][k + 3, j + 3, i + 3]

    pi = 2. * abs(math.acos(0.))
    eps = 10. ** (-5)
    res = {}
    for k in range(1, N3):
        for j in range(1, N2):
            for i in range(1, N1):
                D = [[0.] * 3 for _ in range(3)]
                for ii in range(-3, 4):
                    for m in range(3):
                        D[m][0] = D[m][0] + cp[0][i * 7 + ii + 3] * nlv(m, i + ii, j, k)
                for jj in range(-3, 4):
                    for m in range(3):
                        D[m][1] = D[m][1] + cp[1][j * 7 + jj + 3] * nlv(m, i, j + jj, k)
                for kk in range(-3, 4):
                    for m in range(3):
                        D[m][2] = D[m][2] + cp[2][k * 7 + kk + 3] * nlv(m, i, j, k + kk)
                d = lambda a, b: D[a - 1][b - 1]  # noqa: E731
                T1 = 2. * (d(1, 1) * d(1, 1) + d(1, 2) * d(2, 1) + d(1, 3) * d(3, 1))
                T2 = 2. * (d(2, 1) * d(1, 2) + d(2, 2) * d(2, 2) + d(2, 3) * d(3, 2))
                T3 = 2. * (d(3, 1) * d(1, 3) + d(3, 2) * d(2, 3) + d(3, 3) * d(3, 3))
                T4 = (d(1, 1) + d(2, 2)) * (d(1, 2) + d(2, 1)) + d(1, 3) * d(3, 2) + d(2, 3) * d(3, 1)
                T5 = (d(1, 1) + d(3, 3)) * (d(1, 3) + d(3, 1)) + d(1, 2) * d(2, 3) + d(3, 2) * d(2, 1)
                T6 = (d(2, 2) + d(3, 3)) * (d(2, 3) + d(3, 2)) + d(2, 1) * d(1, 3) + d(3, 1) * d(1, 2)
                PP = T1 + T2 + T3
                QQ = T1 * T2 + T1 * T3 + T2 * T3 - T4 ** 2 - T5 ** 2 - T6 ** 2
                RR = T1 * T2 * T3 + 2. * T4 * T5 * T6 - T1 * T6 ** 2 - T2 * T5 ** 2 - T3 * T4 ** 2
                rho = (PP / 3.) ** 2 - QQ / 3.
                if rho <= eps:
                    res[(i, j, k)] = PP / 3.
                    continue
                rho = math.sqrt(rho)
                QQ = ((PP / 3.) ** 3 - QQ * (PP / 6.) + RR / 2.) / rho ** 3
                if abs(QQ) < 1.:
                    theta = math.acos(QQ) / 3.
                elif QQ > 0.:
                    theta = 0.
                else:
                    theta = pi / 3.
                lam = [math.cos(theta), math.cos(theta + 2. * pi / 3.), math.cos(theta + 4. * pi / 3.)]
                for m in range(3):
                    for n in range(m + 1, 3):
                        if lam[m] > lam[n]:
                            lam[m], lam[n] = lam[n], lam[m]
                res[(i, j, k)] = rho * lam[1] + PP / 6.
    return res
