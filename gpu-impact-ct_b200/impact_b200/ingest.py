"""Geometry and waveform ingest for CT-based cases: the label mask and the measured inflow
waveform, prepared as the reference prepares them before its time loop and handed to a device
case (Case.set_labels, Case.set_inflow_waveform).

    read_vtk_3D            usr_func.f90:187-555   read_vtk_structured_points (or read_nifti) + ct_grid
    read_velocity_waveform usr_func.f90:574-596   read_waveform_csv
    convert_waveform       usr_func.f90:599-651   convert_waveform
    apply_CT_forcing       usr_func.f90:909-1049  labels_from_ct_grid (its label tests),
                                                  inflow_velocity (its inflow lookup)
    get_pressure_waveform_echo_WKM :653-750       windkessel_pressures (inlet / outlet pressure
                                                  for pressure_bc_launcher_)

Reference grid indices are 1-based and the CT grid is M1 x M2 x M3 (grid points per axis, the
library's Grid.N); the library's grids are periodic with n = M - 1 unique points, so the label
mask takes the CT grid's points 1 .. M - 1 of every axis.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# the fringe depth of read_vtk_3D: planes k_start - 10 .. k_start - 1 (inlet, first outlet) and
# k_end + 1 .. k_end + 10 (second outlet)
FRINGE = 10
# physical constants of the reference (mod_vars.f90:235-236)
BLOOD_KINEMATIC_VISCOSITY = 0.0000035
BLOOD_DENSITY = 1060.0
# the jet flow rate that sizes the inflow jet (read_vtk_3D, usr_func.f90:448: Q_max = 0.0004 m^3/s)
Q_MAX = 0.0004


@dataclass
class VtkVolume:
    """A legacy-VTK STRUCTURED_POINTS scalar volume; values[(k-1) d2 d1 + (j-1) d1 + i - 1] is
    point (i, j, k) of the dims d1 x d2 x d3 (i fastest)."""
    dims: tuple
    spacing: tuple
    origin: tuple
    values: np.ndarray
    name: str = ""


def read_vtk_structured_points(path) -> VtkVolume:
    """Read a legacy VTK file holding one STRUCTURED_POINTS scalar field (ASCII, or BINARY
    big-endian), the format read_vtk_3D reads (usr_func.f90:222-268: two header lines, the format,
    DATASET, DIMENSIONS, SPACING, ORIGIN, POINT_DATA, SCALARS, LOOKUP_TABLE, then the values)."""
    with open(path, "rb") as f:
        raw = f.read()
    pos = 0

    def line():
        nonlocal pos
        end = raw.index(b"\n", pos)
        text = raw[pos:end].decode("ascii", errors="replace").strip()
        pos = end + 1
        return text

    line()  # version
    line()  # title
    fmt = line().upper()
    if fmt not in ("ASCII", "BINARY"):
        raise ValueError(f"{path}: data format {fmt!r} is neither ASCII nor BINARY")
    dims = spacing = origin = None
    npts, name, dtype = None, "", "float"
    while True:
        text = line()
        if not text:
            continue
        key, *rest = text.split()
        key = key.upper()
        if key == "DATASET":
            if rest[0].upper() != "STRUCTURED_POINTS":
                raise ValueError(f"{path}: dataset {rest[0]} is not STRUCTURED_POINTS")
        elif key == "DIMENSIONS":
            dims = tuple(int(v) for v in rest[:3])
        elif key in ("SPACING", "ASPECT_RATIO"):
            spacing = tuple(float(v) for v in rest[:3])
        elif key == "ORIGIN":
            origin = tuple(float(v) for v in rest[:3])
        elif key == "POINT_DATA":
            npts = int(rest[0])
        elif key == "SCALARS":
            name = rest[0]
            dtype = rest[1].lower() if len(rest) > 1 else "float"
            if len(rest) > 2 and int(rest[2]) != 1:
                raise ValueError(f"{path}: only one component per point is supported")
        elif key == "LOOKUP_TABLE":
            break
        else:
            raise ValueError(f"{path}: unexpected keyword {key}")
    if dims is None or npts is None:
        raise ValueError(f"{path}: DIMENSIONS or POINT_DATA missing")
    if npts != dims[0] * dims[1] * dims[2]:
        raise ValueError(f"{path}: POINT_DATA {npts} differs from the product of DIMENSIONS {dims}")
    if fmt == "ASCII":
        vals = np.array(raw[pos:].split()[:npts], dtype=np.float64)
    else:
        be = {"float": ">f4", "double": ">f8", "int": ">i4", "unsigned_char": "u1", "char": "i1",
              "short": ">i2", "unsigned_short": ">u2", "unsigned_int": ">u4"}
        if dtype not in be:
            raise ValueError(f"{path}: binary scalar type {dtype} not supported")
        vals = np.frombuffer(raw, dtype=be[dtype], count=npts, offset=pos).astype(np.float64)
    if vals.size != npts:
        raise ValueError(f"{path}: {vals.size} values for POINT_DATA {npts}")
    return VtkVolume(dims, spacing or (1.0, 1.0, 1.0), origin or (0.0, 0.0, 0.0), vals, name)


_NIFTI_TYPES = {2: "u1", 4: "i2", 8: "i4", 16: "f4", 64: "f8", 256: "i1", 512: "u2", 768: "u4"}


def read_nifti(path) -> VtkVolume:
    """A NIfTI-1 single-file volume (.nii, or gzip-compressed .nii.gz; either byte order) as a
    VtkVolume: the first three dimensions with x fastest (the point order of a VTK volume), the
    voxel sizes as spacing, the values scaled by scl_slope / scl_inter when the slope is not 0.
    CT label volumes prepared for read_vtk_3D are often kept in this format before conversion."""
    import gzip
    import struct

    opener = gzip.open if str(path).endswith(".gz") else open
    with opener(path, "rb") as f:
        raw = f.read()
    if len(raw) < 348:
        raise ValueError(f"{path}: shorter than a NIfTI-1 header")
    for end in ("<", ">"):
        if struct.unpack(end + "i", raw[0:4])[0] == 348:
            break
    else:
        raise ValueError(f"{path}: not a NIfTI-1 header (sizeof_hdr is not 348)")
    if raw[344:347] not in (b"n+1", b"ni1"):
        raise ValueError(f"{path}: NIfTI magic missing")
    if raw[344:347] == b"ni1":
        raise ValueError(f"{path}: a two-file NIfTI pair (.hdr/.img) is not supported")
    dim = struct.unpack(end + "8h", raw[40:56])
    if dim[0] < 3 or any(d > 1 for d in dim[4:dim[0] + 1]):
        raise ValueError(f"{path}: not a single 3-D volume (dim = {dim})")
    datatype = struct.unpack(end + "h", raw[70:72])[0]
    if datatype not in _NIFTI_TYPES:
        raise ValueError(f"{path}: NIfTI datatype {datatype} not supported")
    pixdim = struct.unpack(end + "8f", raw[76:108])
    vox_offset = int(struct.unpack(end + "f", raw[108:112])[0])
    slope, inter = struct.unpack(end + "2f", raw[112:120])
    n1, n2, n3 = dim[1], dim[2], dim[3]
    npts = n1 * n2 * n3
    vals = np.frombuffer(raw, dtype=np.dtype(_NIFTI_TYPES[datatype]).newbyteorder(end), count=npts,
                         offset=vox_offset).astype(np.float64)
    if slope != 0.0:
        vals = vals * float(slope) + float(inter)
    return VtkVolume((n1, n2, n3), tuple(float(p) for p in pixdim[1:4]), (0.0, 0.0, 0.0), vals, "nifti")


def write_vtk_structured_points(path, volume: VtkVolume):
    """Write the volume as an ASCII legacy-VTK file (the layout read_vtk_structured_points reads)."""
    d1, d2, d3 = volume.dims
    with open(path, "w") as f:
        f.write("# vtk DataFile Version 3.0\nCT labels\nASCII\nDATASET STRUCTURED_POINTS\n")
        f.write(f"DIMENSIONS {d1} {d2} {d3}\n")
        f.write("SPACING {} {} {}\n".format(*volume.spacing))
        f.write("ORIGIN {} {} {}\n".format(*volume.origin))
        f.write(f"POINT_DATA {d1 * d2 * d3}\nSCALARS {volume.name or 'labels'} float\nLOOKUP_TABLE default\n")
        vals = volume.values
        for s in range(0, vals.size, 9):
            f.write(" ".join(repr(float(v)) for v in vals[s:s + 9]) + "\n")


def pressure_coords(grid):
    """(y1p, y2p) of a Grid as 1-based arrays: y1p[i] is the x coordinate of pressure point i."""
    return grid.xp[0][3:], grid.xp[1][3:]


def inlet_radius(reference_velocity, reference_length):
    """Radius of the incoming jet (read_vtk_3D, usr_func.f90:448): Q_max = 0.0004 m^3/s through a
    circle at the reference velocity, in units of the reference length."""
    return math.sqrt(Q_MAX / (4.0 * math.atan(1.0) * reference_velocity)) / reference_length


@dataclass
class CtGrid:
    """The reference's CT grid grid_set(1:M1, 1:M2, 1:M3) (Fortran order) after read_vtk_3D, with
    the quantities it reports."""
    values: np.ndarray
    inlet_centre: tuple = (0.0, 0.0)
    outlet_centre: tuple = (0.0, 0.0)
    counts: dict = field(default_factory=dict)


def ct_grid(volume: VtkVolume, M, offsets, y1p, y2p, r_inlet) -> CtGrid:
    """grid_set of read_vtk_3D (usr_func.f90:283-497) for a CT grid of M = (M1, M2, M3) points.

    The volume is placed with its axes swapped in x and y -- grid_set(j + y_offset, i + x_offset,
    k + z_offset) = point (i, j, k) -- on a background of 2.0 (outside the CT box).  On plane
    k_start = z_offset + 1 the lumen points (0.5 <= value < 2) with i <= M1 / 2 are the inlet and
    those with i >= M1 / 2 the first outlet; on plane k_end = z_offset + d3 every lumen point
    belongs to the second outlet.  The 10 planes below k_start under an inlet point become 7.0
    (5.0 within r_inlet of the inlet points' mean coordinates), those under a first-outlet point
    9.0, and the 10 planes above k_end over a second-outlet point 11.0, in this order.  y1p[i],
    y2p[j] are the pressure-grid coordinates of points i, j (1-based; index 0 unused)."""
    M1, M2, M3 = (int(m) for m in M)
    xo, yo, zo = (int(o) for o in offsets)
    d1, d2, d3 = volume.dims
    if d2 + yo > M1 or d1 + xo > M2 or d3 + zo > M3 or min(xo, yo, zo) < 0:
        raise ValueError(f"the volume {volume.dims} with offsets {offsets} does not fit the grid {M}")
    if zo + 1 - FRINGE < 1 or zo + d3 + FRINGE > M3:
        raise ValueError(f"the fringe planes of the volume fall outside the grid (z offset {zo}, {M3} planes)")
    g = np.full((M1 + 1, M2 + 1, M3 + 1), 2.0)  # 1-based, index 0 unused
    vol = volume.values.reshape(d3, d2, d1)  # [k, j, i]
    g[1 + yo:1 + yo + d2, 1 + xo:1 + xo + d1, 1 + zo:1 + zo + d3] = vol.transpose(1, 2, 0)
    ks, ke = zo + 1, zo + d3
    half = M1 // 2

    def lumen_points(k, i_lo, i_hi):
        # points (i, j) of plane k in the reference's loop order: j outer, i inner
        sl = g[i_lo:i_hi + 1, 1:M2 + 1, k]
        jj, ii = np.nonzero(((sl >= 0.5) & (sl < 2.0)).T)
        return ii + i_lo, jj + 1

    y1p = np.asarray(y1p, dtype=np.float64)
    y2p = np.asarray(y2p, dtype=np.float64)
    ii_in, jj_in = lumen_points(ks, 1, half)
    ii_out, jj_out = lumen_points(ks, half, M1)
    ii_o2, jj_o2 = lumen_points(ke, 1, M1)

    def centre(ii, jj):
        # running sums in loop order, then the division (x_mean_centre = sum / count)
        sx = sy = 0.0
        for a, b in zip(ii, jj):
            sx += y1p[a]
            sy += y2p[b]
        return (sx / len(ii), sy / len(ii)) if len(ii) else (math.nan, math.nan)

    cin, cout = centre(ii_in, jj_in), centre(ii_out, jj_out)
    jet = np.sqrt((y1p[ii_in] - cin[0]) ** 2 + (y2p[jj_in] - cin[1]) ** 2) <= r_inlet
    for k in range(-FRINGE, 0):
        g[ii_in, jj_in, ks + k] = 7.0
        g[ii_in[jet], jj_in[jet], ks + k] = 5.0
    for k in range(-FRINGE, 0):
        g[ii_out, jj_out, ks + k] = 9.0
    for k in range(1, FRINGE + 1):
        g[ii_o2, jj_o2, ke + k] = 11.0
    counts = {"inlet": int(len(ii_in)), "outlet": int(len(ii_out)), "outlet_2": int(len(ii_o2)),
              "inlet_jet": int(jet.sum())}
    return CtGrid(np.asfortranarray(g[1:, 1:, 1:]), cin, cout, counts)


def labels_from_ct_grid(values: np.ndarray, grid) -> np.ndarray:
    """uint8 labels of the library (padded layout (N3+7, N2+7, N1+7)) from a CT grid of Grid.N
    points per axis, by the tests of apply_CT_forcing (usr_func.f90:933-945): value < 0.5 -> 0
    (no flow), 7 -> 7 (no flow), 5 -> 5 (inflow), 9 -> 9 and 11 -> 11 (outlets), anything else
    (the lumen 1.0, outside the CT box 2.0) -> 1 (free flow).  Points 1 .. N - 1 of every axis
    (the library's grids are periodic)."""
    N1, N2, N3 = grid.N
    if values.shape != (N1, N2, N3):
        raise ValueError(f"CT grid {values.shape} does not match the grid points {grid.N}")
    v = np.asarray(values)[:N1 - 1, :N2 - 1, :N3 - 1]
    lab = np.ones(v.shape, dtype=np.uint8)
    for code in (5, 7, 9, 11):
        lab[v == float(code)] = code
    lab[v < 0.5] = 0
    out = np.zeros((N3 + 7, N2 + 7, N1 + 7), dtype=np.uint8)
    out[4:N3 + 3, 4:N2 + 3, 4:N1 + 3] = lab.transpose(2, 1, 0)
    return out


def read_waveform_csv(path, n=None) -> np.ndarray:
    """(time in pulse [ms], inflow velocity [m/s]) pairs, one per line, separated by a comma or
    blanks (read_velocity_waveform, usr_func.f90:574-596, reads number_of_digitized_points = 74 of
    them); n: read only the first n pairs."""
    rows = []
    with open(path) as f:
        for text in f:
            parts = text.replace(",", " ").split()
            if len(parts) < 2:
                continue
            rows.append((float(parts[0]), float(parts[1])))
            if n is not None and len(rows) == n:
                break
    if len(rows) < 2:
        raise ValueError(f"{path}: fewer than two waveform points")
    return np.array(rows, dtype=np.float64)


@dataclass
class Waveform:
    """The nondimensional inflow table and the reference scales convert_waveform derives."""
    time: np.ndarray
    velocity: np.ndarray
    reference_velocity: float
    reference_length: float
    reference_time: float
    Re: float


def convert_waveform(table: np.ndarray, M1: int, idealized: bool = False, ct_pixel_width: float = 0.0004,
                     upsampling_factor: float = 1.0,
                     kinematic_viscosity: float = BLOOD_KINEMATIC_VISCOSITY) -> Waveform:
    """convert_waveform (usr_func.f90:599-651): reference velocity = the largest inflow velocity
    (its nondimensional maximum is 1), reference length = CT pixel width / (upsampling / M1)
    (the idealized aorta: 0.2 m and 2.7 m/s), Re = U L / nu, reference time = L / U; the table's
    times become t_ms / (1000 reference time), its velocities v / reference velocity."""
    t_ms, vel = table[:, 0], table[:, 1]
    u_ref = float(np.max(vel)) / 1.0
    l_ref = ct_pixel_width / ((1.0 / M1) * upsampling_factor)
    if idealized:
        l_ref, u_ref = 0.2, 2.7
    t_ref = l_ref / u_ref
    return Waveform(t_ms / (1000.0 * t_ref), vel / u_ref, u_ref, l_ref, t_ref, u_ref * l_ref / kinematic_viscosity)


def inflow_velocity(time: np.ndarray, velocity: np.ndarray, t: float):
    """The inflow velocity apply_CT_forcing (usr_func.f90:929-945) imposes at nondimensional time
    t: t shifted into the current pulse (get_shifted_time_in_pulse, :899-906; pulse length = the
    last table time, :753-760), then the value at the start of the last interval [t_i, t_i+1]
    holding it; None when no interval holds it (the velocity is left as it is)."""
    length = float(time[-1])
    ts = t - (math.floor(t / length) + 1.0 - 1.0) * length
    u = None
    for i in range(len(time) - 1):
        if time[i] <= ts <= time[i + 1]:
            u = float(velocity[i])
    return u


# RK3 coefficients of the reference (mod_vars.f90:774-775)
A_RK = (8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0)
B_RK = (0.0, -17.0 / 60.0, -5.0 / 12.0)


def jor_pressures(p_inlet, p_outlet, p_outlet_2, substep, dtime):
    """The boundary values the reference's JOR loop passes to pressure_bc_launcher_: each pressure
    times (aRK + bRK) of RK substep `substep` (1..3) times the time step
    (jacobi_solver_host_v4.f90:302-304); for impact_b200.jacobi_solve(..., pressures=...).  The
    reference applies the condition in substep 3 only (jacobi_solver_host_v4.f90:304-305): pass
    labels and these pressures to jacobi_solve in substep 3, and no labels in substeps 1 and 2."""
    f = A_RK[substep - 1] + B_RK[substep - 1]
    return tuple(p * f * dtime for p in (p_inlet, p_outlet, p_outlet_2))


class AnalyticWindkessel:
    """Pressure and flow rate of the three branches -- 1 inlet, 2 first outlet, 3 second outlet --
    from the analytic two-element Windkessel of get_pressure_and_flow_rate_WKM (usr_func.f90:
    762-855): a half-sine systolic inflow of peak q_peak over the first 0.4 s of a 1 s beat gives
    the closed-form systolic pressure from 80 mmHg; in diastole the pressure decays from the last
    systolic value with time constant R C.  Returns nondimensional (p, q): p / (density U_ref^2)
    in Pa (mmHg x 133.322), q / (L_ref^3 / T_ref).  The last systolic pressure of each branch is
    state (the reference keeps it in p_end_systole_in / _out / _out_2 and its restart files);
    pass end_systole to continue from saved values."""

    # (C [m^3/Pa-ish, as the reference divides], R, peak flow) per branch, in the reference's own
    # arithmetic: C = value / 1e6, R = value * 1e6, peak = 0.0004 x fraction
    BRANCHES = {1: (1.5496 / 1000000.0, 0.9758 * 1000000.0, 0.0004),
                2: (1.5 / 1000000.0, 1.12 * 1000000.0, 0.0004 * 0.85),
                3: (0.059 / 1000000.0, 19.68 * 1000000.0, 0.0004 * 0.05)}

    def __init__(self, reference_time, reference_velocity, reference_length, density=BLOOD_DENSITY,
                 end_systole=(0.0, 0.0, 0.0)):
        self.reference_time = float(reference_time)
        self.reference_velocity = float(reference_velocity)
        self.reference_length = float(reference_length)
        self.density = float(density)
        self.end_systole = {b: float(v) for b, v in zip((1, 2, 3), end_systole)}

    def __call__(self, branch, t):
        c, r, q_peak = self.BRANCHES[branch]
        beat = 1.0
        systole = 0.4 * beat
        p_dia = 80.0
        pi = 4.0 * math.atan(1.0)
        tp = t * self.reference_time
        den = systole ** 2.0 + c ** 2.0 * pi ** 2.0 * r ** 2.0
        if tp <= systole:
            p = ((p_dia + q_peak * systole * r * c * pi * r / den) * math.exp(-1.0 * tp / (r * c))
                 - (systole * q_peak * r * (c * pi * r * math.cos(pi * tp / systole))
                    - systole * math.sin(pi * tp / systole)) / den)
            q = q_peak * math.sin(pi * tp / systole)
            self.end_systole[branch] = p
        else:
            p = self.end_systole[branch] * math.exp(-1.0 * (tp - systole) / (r * c))
            q = 0.0
        p = p / (self.density * self.reference_velocity ** 2.0) * 133.322
        q = q / (self.reference_length ** 3.0 / self.reference_time)
        return p, q


def windkessel_pressures(table: np.ndarray, waveform: Waveform, t: float, r_in=0.78e6, c_in=2.166e-6,
                         r_out=0.898e6, c_out=2.066e-6, q_max=Q_MAX, outlet_fraction=0.85, p0_mmhg=80.0,
                         density=BLOOD_DENSITY):
    """Inlet and outlet pressures at nondimensional time t from the echo waveform and a
    two-element Windkessel model (get_pressure_waveform_echo_WKM, usr_func.f90:653-750; defaults:
    the reference's TAVI 000 resistances and compliances).  For each table interval holding the
    time shifted into the current pulse, starting from p0 = 80 mmHg:
    p = p (1 - dt / (C R)) - dt / C q with dt the interval's length in seconds and q its start
    velocity times the inlet area q_max / (peak velocity) (outlet: q_max x 0.85); the result is made
    nondimensional by density x reference velocity^2 (mmHg -> Pa: 133.322).  These are the values
    the reference's pressure boundary condition (pressure_bc_launcher_) receives."""
    t_ms, vel = table[:, 0], table[:, 1]
    length = float(waveform.time[-1])
    ts = t - (math.floor(t / length) + 1.0 - 1.0) * length
    vmax = float(np.max(vel))
    out = []
    for r, c, q in ((r_in, c_in, q_max), (r_out, c_out, q_max * outlet_fraction)):
        area = q / vmax
        p = p0_mmhg
        for i in range(len(t_ms) - 1):
            if waveform.time[i] <= ts <= waveform.time[i + 1]:
                dt = t_ms[i + 1] / 1000.0 - t_ms[i] / 1000.0
                p = p * (1.0 - dt / (c * r)) - dt / c * (vel[i] * area)
        out.append(p / (density * waveform.reference_velocity ** 2.0) * 133.322)
    return out[0], out[1]
