"""Literal CPU restatement of the reference's CT-geometry and inflow-waveform preparation, the
checker for impact_b200.ingest.

TEST INFRASTRUCTURE ONLY: imported by tests/.  Plain Python loops in the reference's loop order,
1-based indices, for small grids.  Parity unpinned: read_vtk_3D and convert_waveform are
Fortran (usr_func.f90) and no Fortran compiler is in this image, so this restatement is not
checked against the reference's own output.

    grid_set      read_vtk_3D            usr_func.f90:283-497
    labels        apply_CT_forcing       usr_func.f90:933-945 (the label tests)
    converted     convert_waveform       usr_func.f90:599-651
    inflow        apply_CT_forcing       usr_func.f90:929-945, get_shifted_time_in_pulse :899-906,
                  get_pulse_number_and_length :753-760
    windkessel    get_pressure_waveform_echo_WKM  usr_func.f90:653-750
"""
from __future__ import annotations

import math


def grid_set(values, dims, M, offsets, y1p, y2p, r_inlet):
    """grid_set(1:M1,1:M2,1:M3) as a dict {(i, j, k): value} plus (inlet centre, outlet centre,
    counts), following read_vtk_3D statement by statement."""
    M1, M2, M3 = M
    xo, yo, zo = offsets
    d1, d2, d3 = dims
    g = {}
    for i in range(1, M1 + 1):
        for j in range(1, M2 + 1):
            for k in range(1, M3 + 1):
                g[(i, j, k)] = 2.0
    for i in range(1, d1 + 1):  # usr_func.f90:283-291
        for j in range(1, d2 + 1):
            for k in range(1, d3 + 1):
                g[(j + yo, i + xo, k + zo)] = float(values[(k - 1) * d2 * d1 + (j - 1) * d1 + i - 1])
    half = int(math.floor(M1 / 2.0))
    ks = zo + 1

    def lumen(v):
        return 0.5 <= v < 2.0

    xs = ys = 0.0  # inlet: usr_func.f90:308-346
    inlet = []
    for j in range(1, M2 + 1):
        for i in range(1, half + 1):
            if lumen(g[(i, j, ks)]):
                xs += y1p[i]
                ys += y2p[j]
                inlet.append((i, j))
    cin = (xs / len(inlet), ys / len(inlet)) if inlet else (math.nan, math.nan)
    xs = ys = 0.0  # first outlet: usr_func.f90:353-387
    outlet = []
    for j in range(1, M2 + 1):
        for i in range(half, M1 + 1):
            if lumen(g[(i, j, ks)]):
                xs += y1p[i]
                ys += y2p[j]
                outlet.append((i, j))
    cout = (xs / len(outlet), ys / len(outlet)) if outlet else (math.nan, math.nan)
    ke = zo + d3  # second outlet: usr_func.f90:391-418
    outlet2 = []
    for j in range(1, M2 + 1):
        for i in range(1, M1 + 1):
            if lumen(g[(i, j, ke)]):
                outlet2.append((i, j))
    jet = 0
    for (i, j) in inlet:  # usr_func.f90:446-473
        for k in range(-10, 0):
            g[(i, j, ks + k)] = 7.0
            if math.sqrt((y1p[i] - cin[0]) ** 2 + (y2p[j] - cin[1]) ** 2) <= r_inlet:
                g[(i, j, ks + k)] = 5.0
                if k == -1:
                    jet += 1
    for (i, j) in outlet:  # usr_func.f90:477-485
        for k in range(-10, 0):
            g[(i, j, ks + k)] = 9.0
    for (i, j) in outlet2:  # usr_func.f90:488-497
        for k in range(1, 11):
            g[(i, j, ke + k)] = 11.0
    counts = {"inlet": len(inlet), "outlet": len(outlet), "outlet_2": len(outlet2), "inlet_jet": jet}
    return g, cin, cout, counts


def label(v):
    """The forcing class of a CT value (apply_CT_forcing, usr_func.f90:933-945)."""
    if v < 0.5:
        return 0
    if v == 7.0:
        return 7
    if v == 5.0:
        return 5
    if v == 9.0:
        return 9
    if v == 11.0:
        return 11
    return 1


def converted(table, M1, idealized=False, ct_pixel_width=0.0004, upsampling_factor=1.0, nu=0.0000035):
    """convert_waveform: (times, velocities, reference velocity, length, time, Re)."""
    u_ref = max(v for (_, v) in table) / 1.0
    l_ref = ct_pixel_width / ((1.0 / M1) * upsampling_factor)
    if idealized:
        l_ref, u_ref = 0.2, 2.7
    t_ref = l_ref / u_ref
    times = [t / (1000.0 * t_ref) for (t, _) in table]
    vels = [v / u_ref for (_, v) in table]
    return times, vels, u_ref, l_ref, t_ref, u_ref * l_ref / nu


def inflow(times, vels, t):
    """The imposed inflow velocity at time t, or None (no table interval holds the shifted time)."""
    pulse_length = times[-1]
    pulse_number = math.floor(t / pulse_length) + 1
    ts = t - (pulse_number - 1) * pulse_length
    u = None
    for i in range(len(times) - 1):
        if times[i] <= ts <= times[i + 1]:
            u = vels[i]
    return u


def windkessel(table, times, u_ref, t):
    """(pre_inlet, pre_outlet) of get_pressure_waveform_echo_WKM with its TAVI 000 constants."""
    pulse_length = times[-1]
    pulse_number = math.floor(t / pulse_length) + 1
    ts = t - (pulse_number - 1) * pulse_length
    vel_max = max(v for (_, v) in table)
    res = []
    for R, C, q_max in ((0.78 * 1000000., 2.166 / 1000000., 0.0004 * 1.0),
                        (0.898 * 1000000., 2.066 / 1000000., 0.0004 * 0.85 * 1.0)):
        inlet_area = q_max / vel_max
        pre = 80.
        for i in range(len(table) - 1):
            if times[i] <= ts <= times[i + 1]:
                dt = table[i + 1][0] / 1000. - table[i][0] / 1000.
                q_in = table[i][1] * inlet_area
                pre = pre * (1. - dt / (C * R)) - dt / C * q_in
        res.append(pre / (1060. * u_ref ** 2.) * 133.322)
    return res[0], res[1]
