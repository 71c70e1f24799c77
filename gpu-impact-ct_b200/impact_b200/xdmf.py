"""Field output for visualisation: XDMF 2 light data with raw binary heavy data.

Follows write_fields, filespace_props and write_3D_xdmf (mod_inout.f90:78-500, 2713-2815,
3166-3290): the velocity components are interpolated to the pressure points with the cIup
tables (interpolate2_vel_pre, mod_diff.f90:1740-1825), the pressure is written as it is, and
every field is written on the pressure grid of the unique periodic points 1..N-1, sub-sampled by
a stride per axis that must divide N - 1.  One XDMF file per output and stride names the
3DRectMesh (VXVYVZ coordinates y1p, y2p, y3p at the sampled points), the time and the node
attributes Pressure, Velocity_X, Velocity_Y, Velocity_Z and optionally Lambda_2 (lambda,
:2827-3008), optionally scaled to physical units by Function items (length L_ref, velocity
U_ref, pressure rho U_ref^2, time L_ref / U_ref, lambda-2 U_ref / L_ref as the reference writes).

The reference writes its heavy data with parallel HDF5, which this image does not carry; here
each field is a flat little-endian float64 file read by the XDMF Format="Binary" data item
(ParaView and VisIt read both forms).  File names keep the reference's pattern
<field>_<stride name>_<5-digit count> with the extension .bin; the light data is
<base>_<stride name>_<count>.xmf.

Host-side output code: the snapshot that feeds it is taken on the device
(Case.snapshot / Case.download), the interpolation and the writes run on the host cores.
"""
from __future__ import annotations

import math
import os
import xml.etree.ElementTree as ET
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np

VELOCITY = ("vel1", "vel2", "vel3")
_THREADS = max(1, min(16, os.cpu_count() or 1))
ATTRIBUTES = (("Pressure", "pre"), ("Velocity_X", "velX"), ("Velocity_Y", "velY"), ("Velocity_Z", "velZ"))


def velocity_at_pressure_points(grid, vel, m):
    """Velocity component m (1..3) interpolated to the pressure points 1..N-1 of every axis.

    vel is a field of shape grid.shape whose unique periodic points are its interior; the ghosts
    are not read (the periodic continuation is taken from the interior, as exchange would fill
    them).  Returns the interior-sized array (N3-1, N2-1, N1-1).  The six products are summed in
    the order l = -3..2 of the stencil, so the result matches the reference loop bit for bit.
    """
    if m not in (1, 2, 3):
        raise ValueError("velocity component m must be 1, 2 or 3")
    vel = np.asarray(vel, dtype=np.float64)
    if vel.shape != grid.shape:
        raise ValueError(f"field shape {vel.shape} is not the grid's {grid.shape}")
    N = grid.N[m - 1]
    rows = np.asarray(grid.tab["cIup"][m - 1], dtype=np.float64).reshape(N + 1, 6)[1:N]
    axis = 3 - m                       # (k, j, i) storage: m = 1 is the last axis
    inner = vel[4:grid.N[2] + 3, 4:grid.N[1] + 3, 4:grid.N[0] + 3]
    return _periodic_stencil(inner, rows, axis, -3)


def _periodic_stencil(u, rows, axis, lo):
    """sum over l of rows[:, l - lo] * u(i + l) along `axis` of the interior array u, periodic,
    the terms added in the order of l (the first one not added to zero).  Large arrays are cut
    into slabs across another axis and done by a thread pool (numpy's arithmetic releases the
    interpreter lock); every point gets the same operations in the same order either way."""
    split = 0 if axis != 0 else 1
    slabs = min(_THREADS, u.shape[split]) if u.size >= (1 << 20) else 1
    if slabs > 1:
        edges = np.linspace(0, u.shape[split], slabs + 1).astype(int)
        out = np.empty(u.shape)

        def work(q):
            sl = [slice(None)] * 3
            sl[split] = slice(edges[q], edges[q + 1])
            out[tuple(sl)] = _stencil_block(u[tuple(sl)], rows, axis, lo)

        with ThreadPoolExecutor(slabs) as ex:
            list(ex.map(work, range(slabs)))
        return out
    return _stencil_block(u, rows, axis, lo)


def _stencil_block(u, rows, axis, lo):
    n = u.shape[axis]
    width = rows.shape[1]
    pad = [(0, 0)] * 3
    pad[axis] = (-lo, width - 1 + lo)
    wrapped = np.pad(u, pad, mode="wrap")   # u(i + l) at wrapped[i - 1 - lo + l]
    bshape = [1, 1, 1]
    bshape[axis] = n
    out = None
    for l in range(lo, lo + width):
        sl = [slice(None)] * 3
        sl[axis] = slice(l - lo, l - lo + n)
        term = rows[:, l - lo].reshape(bshape) * wrapped[tuple(sl)]
        out = term if out is None else out + term
    return out


def lambda2(grid, vel1, vel2, vel3):
    """The lambda-2 vortex criterion at the pressure points (lambda, mod_inout.f90:2827-3008):
    the velocity interpolated to the pressure points, its gradient Dvel(m, a) = d u_m / d x_a with
    the 7-point cp tables (periodic), the symmetric tensor TT of the reference, and the middle
    eigenvalue from the trigonometric solution of its characteristic cubic (PP / 3 where the
    discriminant rho <= 1e-5).  Returns the interior-sized array (N3-1, N2-1, N1-1)."""
    w = [velocity_at_pressure_points(grid, v, m) for m, v in ((1, vel1), (2, vel2), (3, vel3))]
    D = [[None] * 3 for _ in range(3)]
    for a in range(3):
        N = grid.N[a]
        rows = np.asarray(grid.tab["cp1"][a], dtype=np.float64).reshape(N + 1, 7)[1:N]
        for m in range(3):
            D[m][a] = _periodic_stencil(w[m], rows, 2 - a, -3)
    d = lambda m, a: D[m - 1][a - 1]  # noqa: E731  (Dvel(m, a) of the reference, 1-based)
    t1 = 2.0 * (d(1, 1) * d(1, 1) + d(1, 2) * d(2, 1) + d(1, 3) * d(3, 1))
    t2 = 2.0 * (d(2, 1) * d(1, 2) + d(2, 2) * d(2, 2) + d(2, 3) * d(3, 2))
    t3 = 2.0 * (d(3, 1) * d(1, 3) + d(3, 2) * d(2, 3) + d(3, 3) * d(3, 3))
    t4 = (d(1, 1) + d(2, 2)) * (d(1, 2) + d(2, 1)) + d(1, 3) * d(3, 2) + d(2, 3) * d(3, 1)
    t5 = (d(1, 1) + d(3, 3)) * (d(1, 3) + d(3, 1)) + d(1, 2) * d(2, 3) + d(3, 2) * d(2, 1)
    t6 = (d(2, 2) + d(3, 3)) * (d(2, 3) + d(3, 2)) + d(2, 1) * d(1, 3) + d(3, 1) * d(1, 2)
    pp = t1 + t2 + t3
    qq = t1 * t2 + t1 * t3 + t2 * t3 - t4 ** 2 - t5 ** 2 - t6 ** 2
    rr = t1 * t2 * t3 + 2.0 * t4 * t5 * t6 - t1 * t6 ** 2 - t2 * t5 ** 2 - t3 * t4 ** 2
    rho = (pp / 3.0) ** 2 - qq / 3.0
    flat = rho <= 1e-5
    sr = np.sqrt(np.where(flat, 1.0, rho))
    q = ((pp / 3.0) ** 3 - qq * (pp / 6.0) + rr / 2.0) / sr ** 3
    pi = 2.0 * abs(math.acos(0.0))
    theta = np.where(np.abs(q) < 1.0, np.arccos(np.clip(q, -1.0, 1.0)) / 3.0, np.where(q > 0.0, 0.0, pi / 3.0))
    lam = np.sort(np.stack([np.cos(theta), np.cos(theta + 2.0 * pi / 3.0), np.cos(theta + 4.0 * pi / 3.0)]), axis=0)
    return np.where(flat, pp / 3.0, sr * lam[1] + pp / 6.0)


def sampled_points(N, stride):
    """Indices (1-based) of the points an output with this stride holds along an axis of N
    points: 1, 1 + stride, ..., (N - 1) / stride of them; the stride must divide N - 1."""
    if stride < 1 or (N - 1) % stride != 0:
        raise ValueError(f"stride {stride} does not divide N - 1 = {N - 1}")
    return np.arange(1, N, stride)


@dataclass
class Scale:
    """Physical units of the output (scale_output_yes): reference length, velocity, density."""
    L_ref: float
    U_ref: float
    rho: float = 1060.0


class XdmfWriter:
    """Writes numbered outputs of one grid into a directory.

    strides: {name: (s1, s2, s3)}, one output per entry (the reference's large / med / small).
    """

    def __init__(self, directory, grid, strides=None, scale: Scale | None = None, base="IMPACT_xdmf3d",
                 with_lambda2=False):
        self.directory, self.grid, self.scale, self.base = str(directory), grid, scale, base
        self.with_lambda2 = bool(with_lambda2)  # write_lambda2_yes: also the Lambda_2 attribute
        self.strides = dict(strides or {"large": (1, 1, 1)})
        self.points = {}
        for name, st in self.strides.items():
            if len(st) != 3:
                raise ValueError("a stride has three components")
            self.points[name] = [sampled_points(grid.N[a], int(st[a])) for a in range(3)]
        self.count = 0
        os.makedirs(self.directory, exist_ok=True)

    def fields_from_case(self, case):
        """The four state fields of a device case, downloaded to host arrays."""
        return {f: case.download(f) for f in VELOCITY + ("pre",)}

    def write(self, fields, time, count=None):
        """Write one output of the fields {"vel1", "vel2", "vel3", "pre"} (grid-shaped host
        arrays) at `time`.  Returns the paths of the XDMF files, one per stride."""
        count = self.count if count is None else int(count)
        g = self.grid
        data = {"pre": np.asarray(fields["pre"], dtype=np.float64)[4:g.N[2] + 3, 4:g.N[1] + 3, 4:g.N[0] + 3]}
        for m, key in enumerate(("velX", "velY", "velZ"), start=1):
            data[key] = velocity_at_pressure_points(g, fields[VELOCITY[m - 1]], m)
        if self.with_lambda2:
            data["lamb"] = lambda2(g, *(fields[v] for v in VELOCITY))
        paths = []
        for name in self.strides:
            p1, p2, p3 = self.points[name]
            tag = f"{name}_{count:05d}"
            files = {}
            for key, arr in data.items():
                sub = arr[np.ix_(p3 - 1, p2 - 1, p1 - 1)]
                files[key] = self._bin(f"{key}_{tag}.bin", sub)
            coords = []
            for a, pts in enumerate((p1, p2, p3)):
                coords.append(self._bin(f"coord{'XYZ'[a]}_{tag}.bin", g.xp[a][pts + 3]))
            paths.append(self._xml(tag, (len(p1), len(p2), len(p3)), coords, files, time))
        self.count = count + 1
        return paths

    def _bin(self, name, arr):
        np.ascontiguousarray(arr, dtype="<f8").tofile(os.path.join(self.directory, name))
        return name

    def _item(self, parent, dims, fname, factor):
        dims_s = " ".join(str(d) for d in dims)
        if factor is not None:
            parent = ET.SubElement(parent, "DataItem", ItemType="Function", Function=f"{factor!r} * $0",
                                   Dimensions=dims_s, NumberType="Float", Precision="8")
        it = ET.SubElement(parent, "DataItem", Format="Binary", Dimensions=dims_s, NumberType="Float",
                           Precision="8", Endian="Little")
        it.text = fname

    def _xml(self, tag, n, coords, files, time):
        sc = self.scale
        root = ET.Element("Xdmf", Version="2.0")
        grid = ET.SubElement(ET.SubElement(root, "Domain"), "Grid", Name="IMPACT mesh", GridType="Uniform")
        ET.SubElement(grid, "Topology", TopologyType="3DRectMesh", Dimensions=f"{n[2]} {n[1]} {n[0]}")
        geo = ET.SubElement(grid, "Geometry", GeometryType="VXVYVZ")
        for a in range(3):
            self._item(geo, (n[a],), coords[a], None if sc is None else sc.L_ref)
        t = time if sc is None else time * sc.L_ref / sc.U_ref
        ET.SubElement(grid, "Time", TimeType="Single", Value=repr(float(t)))
        attrs = ATTRIBUTES + ((("Lambda_2", "lamb"),) if "lamb" in files else ())
        for attr, key in attrs:
            a = ET.SubElement(grid, "Attribute", Name=attr, Center="Node")
            factor = None
            if sc is not None:  # the reference's factors, U_ref / L_ref for lambda-2 included
                factor = {"pre": sc.rho * sc.U_ref ** 2, "lamb": sc.U_ref / sc.L_ref}.get(key, sc.U_ref)
            self._item(a, (n[2], n[1], n[0]), files[key], factor)
        path = os.path.join(self.directory, f"{self.base}_{tag}.xmf")
        ET.indent(root)
        with open(path, "w") as f:
            f.write('<?xml version="1.0" ?>\n<!DOCTYPE Xdmf SYSTEM "Xdmf.dtd" []>\n')
            f.write(ET.tostring(root, encoding="unicode"))
            f.write("\n")
        return path


def read_output(path):
    """Read an XDMF file this module wrote back into {"x", "y", "z", "time", attribute name:
    array (n3, n2, n1)}, with any Function scaling applied."""
    root = ET.parse(path).getroot()
    here = os.path.dirname(os.path.abspath(path))
    grid = root.find("Domain/Grid")

    def load(item):
        if item.get("ItemType") == "Function":
            factor = float(item.get("Function").split("*")[0])
            return factor * load(item.find("DataItem"))
        dims = tuple(int(d) for d in item.get("Dimensions").split())
        return np.fromfile(os.path.join(here, item.text.strip()), dtype="<f8").reshape(dims)

    out = {"time": float(grid.find("Time").get("Value"))}
    for key, item in zip(("x", "y", "z"), grid.find("Geometry").findall("DataItem")):
        out[key] = load(item)
    for a in grid.findall("Attribute"):
        out[a.get("Name")] = load(a.find("DataItem"))
    return out
