"""Synthetic vessel geometries as IMPACT voxel-label masks.

The labels follow the CT-forcing convention of apply_CT_forcing (usr_func.f90:909-1049) and the
idealized-aorta labelling of read_vtk_3D (usr_func.f90:454-492):
    0 solid (u = 0), 1 fluid, 5 inflow buffer (u_z = inflow, u_x = u_y = 0),
    7 wall (u = 0), 9 outlet, 11 second outlet.
A label sits at pressure point (i, j, k) and applies to all three velocity components there.
Arrays are uint8 in the padded field layout (N3+7, N2+7, N1+7); only the interior is set.
"""
from __future__ import annotations

import numpy as np

SOLID, FLUID, INFLOW, WALL, OUTLET, OUTLET2 = 0, 1, 5, 7, 9, 11


def _coords(grid):
    N1, N2, N3 = grid.N
    x = grid.xp[0][4:N1 + 3]
    y = grid.xp[1][4:N2 + 3]
    z = grid.xp[2][4:N3 + 3]
    return x, y, z


def _finish(grid, inside, n_in, n_out):
    N1, N2, N3 = grid.N
    lab = np.zeros((N3 + 7, N2 + 7, N1 + 7), dtype=np.uint8)
    core = np.where(inside, FLUID, SOLID).astype(np.uint8)  # (k, j, i)
    nz = core.shape[0]
    if n_in > 0:
        core[:n_in][inside[:n_in]] = INFLOW
    if n_out > 0:
        core[nz - n_out:][inside[nz - n_out:]] = OUTLET
    lab[4:N3 + 3, 4:N2 + 3, 4:N1 + 3] = core
    return lab


def stenosed_radius(z, R, stenoses):
    """r(z) = R (1 - sum_s d_s exp(-(z - z_s)^2 / (2 s_s^2))), d_s = 1 - sqrt(1 - area_reduction_s)."""
    r = np.full_like(z, R, dtype=np.float64)
    for (z0, area_red, sigma) in stenoses:
        d = 1.0 - np.sqrt(1.0 - area_red)
        r = r - R * d * np.exp(-((z - z0) ** 2) / (2.0 * sigma ** 2))
    return r


def straight_vessel(grid, radius_frac=0.25, stenoses=(), n_in=10, n_out=10):
    """Cylinder along z centred in the x-y cross-section, radius = radius_frac * L1; optional
    Gaussian stenoses (z0, area_reduction, sigma).  Inflow buffer: the first n_in planes inside
    the lumen; outlet: the last n_out planes."""
    x, y, z = _coords(grid)
    R = radius_frac * grid.L[0]
    cx, cy = 0.5 * grid.L[0], 0.5 * grid.L[1]
    r = stenosed_radius(z, R, stenoses)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    rr = np.sqrt((X - cx) ** 2 + (Y - cy) ** 2)
    inside = rr <= r[:, None, None]
    return _finish(grid, inside, n_in, n_out)


def curved_tube(grid, rng, radius, stenoses=(), max_curvature=2.0, n_in=10, n_out=10):
    """Tube along a random cubic-spline centreline c(z) = (cx(z), cy(z)) whose curvature stays
    below max_curvature / L3; radius with optional stenoses along z."""
    x, y, z = _coords(grid)
    L1, L2, L3 = grid.L
    # four control offsets, natural cubic interpolation through them
    zk = np.linspace(0.0, L3, 4)
    amp = 0.5 * min(L1, L2) - radius * 1.2
    amp = max(amp, 0.0)
    ox = rng.uniform(-1, 1, 4) * amp * 0.5
    oy = rng.uniform(-1, 1, 4) * amp * 0.5
    cx = 0.5 * L1 + np.interp(z, zk, ox)
    cy = 0.5 * L2 + np.interp(z, zk, oy)
    # smooth the piecewise-linear centreline with a cubic B-spline pass
    for _ in range(3):
        cx[1:-1] = 0.25 * cx[:-2] + 0.5 * cx[1:-1] + 0.25 * cx[2:]
        cy[1:-1] = 0.25 * cy[:-2] + 0.5 * cy[1:-1] + 0.25 * cy[2:]
    # curvature bound: scale offsets down if needed
    dz = z[1] - z[0]
    for c, mid in ((cx, 0.5 * L1), (cy, 0.5 * L2)):
        d2 = np.abs(np.gradient(np.gradient(c, dz), dz))
        kmax = d2.max() if d2.size else 0.0
        lim = max_curvature / L3
        if kmax > lim:
            c[:] = mid + (c - mid) * (lim / kmax)
    r = stenosed_radius(z, radius, stenoses)
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    rr = np.sqrt((X - cx[:, None, None]) ** 2 + (Y - cy[:, None, None]) ** 2)
    inside = rr <= r[:, None, None]
    return _finish(grid, inside, n_in, n_out)


def inflow_velocity(t, U0=1.0, T=1.0):
    """Pulsatile plug inflow u_z = U0 (1 + 0.5 sin(2 pi t / T))."""
    return U0 * (1.0 + 0.5 * np.sin(2.0 * np.pi * t / T))
