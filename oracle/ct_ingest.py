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
    windkessel_wkm  get_pressure_and_flow_rate_WKM  usr_func.f90:762-855
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


class windkessel_wkm:
    """get_pressure_and_flow_rate_WKM(branch_number, p, q) with the module's three end-systolic
    pressures (p_end_systole_in / _out / _out_2) as state; the reference's `time`,
    reference_time / _velocity / _length and blood_density = 1060 as inputs."""

    def __init__(self, reference_time, reference_velocity, reference_length):
        self.reference_time = reference_time
        self.reference_velocity = reference_velocity
        self.reference_length = reference_length
        self.p_end_systole_in = 0.
        self.p_end_systole_out = 0.
        self.p_end_systole_out_2 = 0.

    def __call__(self, branch_number, time):
        pi = 4. * math.atan(1.)
        T_beat = 1.
        T_systole = 0.4 * T_beat
        p_diastole = 80.
        if branch_number == 1:
            CWK = 1.5496 / 1000000.
            RWK = 0.9758 * 1000000.
            Q_peak_systole = 0.0004
        elif branch_number == 2:
            CWK = 1.5 / 1000000.
            RWK = 1.12 * 1000000.
            Q_peak_systole = 0.0004 * 0.85
        else:
            CWK = 0.059 / 1000000.
            RWK = 19.68 * 1000000.
            Q_peak_systole = 0.0004 * 0.05
        time_phys = time * self.reference_time
        if time_phys <= T_systole:
            p = (p_diastole + Q_peak_systole * T_systole * RWK * CWK * pi * RWK / (T_systole ** 2. + CWK ** 2. * pi ** 2. * RWK ** 2.)) \
                * math.exp(-1. * time_phys / (RWK * CWK)) \
                - (T_systole * Q_peak_systole * RWK * (CWK * pi * RWK * math.cos(pi * time_phys / T_systole))
                   - T_systole * math.sin(pi * time_phys / T_systole)) / (T_systole ** 2. + CWK ** 2. * pi ** 2. * RWK ** 2.)
            q = Q_peak_systole * math.sin(pi * (time_phys) / T_systole)
            if branch_number == 1:
                self.p_end_systole_in = p
            elif branch_number == 2:
                self.p_end_systole_out = p
            else:
                self.p_end_systole_out_2 = p
        else:
            p_end = {1: self.p_end_systole_in, 2: self.p_end_systole_out}.get(branch_number, self.p_end_systole_out_2)
            p = p_end * math.exp(-1. * (time_phys - T_systole) / (RWK * CWK))
            q = 0.
        p = p / (1060. * self.reference_velocity ** 2.) * 133.322
        q = q / (self.reference_length ** 3. / self.reference_time)
        return p, q
