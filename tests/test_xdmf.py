"""Field output (impact_b200.xdmf) against write_fields / write_3D_xdmf (mod_inout.f90:78-500,
3166-3290): the velocity interpolated to the pressure points matches the oracle's
interpolate_vel_pre bit for bit on a stretched grid (ghost values are not read), the strided
outputs hold the points 1, 1 + s, ... with their coordinates, the XDMF files parse and read back
to the written data and time, physical scaling multiplies lengths, velocities, pressure and time,
a stride that does not divide N - 1 is an error, and the lambda-2 field (lambda,
mod_inout.f90:2827-3008) matches a literal loop restatement to rounding."""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

import impact_b200 as I
import oracle as O
import output_restatement as R
from impact_b200 import xdmf as X

N = (17, 13, 25)
L = (1.0, 1.5, 2.0)
KINDS = (1, 0, 1)


def _fields(seed=3):
    rng = np.random.default_rng(seed)
    shape = (N[2] + 7, N[1] + 7, N[0] + 7)
    return {f: rng.uniform(-1.0, 1.0, size=shape) for f in ("vel1", "vel2", "vel3", "pre")}


def test_velocity_interpolation_matches_oracle():
    grid, og = I.Grid(N, L, KINDS), O.Grid(N, L, KINDS)
    f = _fields()
    for m in (1, 2, 3):
        got = X.velocity_at_pressure_points(grid, f[f"vel{m}"], m)
        want = og.interior(og.interpolate_vel_pre(m, f[f"vel{m}"].copy()))
        assert got.shape == (N[2] - 1, N[1] - 1, N[0] - 1)
        assert np.array_equal(got, want), m
    with pytest.raises(ValueError):
        X.velocity_at_pressure_points(grid, f["vel1"], 4)


def test_strided_outputs_round_trip(tmp_path):
    grid = I.Grid(N, L, KINDS)
    f = _fields(4)
    w = X.XdmfWriter(tmp_path, grid, strides={"large": (1, 1, 1), "small": (2, 4, 3)})
    paths = w.write(f, 0.125)
    assert len(paths) == 2 and w.count == 1
    vel = [X.velocity_at_pressure_points(grid, f[f"vel{m}"], m) for m in (1, 2, 3)]
    pre = grid.interior(f["pre"])
    for path, st in zip(paths, ((1, 1, 1), (2, 4, 3))):
        root = ET.parse(path).getroot()
        topo = root.find("Domain/Grid/Topology")
        n = [(N[a] - 1) // st[a] for a in range(3)]
        assert topo.get("TopologyType") == "3DRectMesh"
        assert topo.get("Dimensions") == f"{n[2]} {n[1]} {n[0]}"
        back = X.read_output(path)
        assert back["time"] == 0.125
        sl = (slice(None, None, st[2]), slice(None, None, st[1]), slice(None, None, st[0]))
        assert np.array_equal(back["Pressure"], pre[sl])
        for name, v in zip(("Velocity_X", "Velocity_Y", "Velocity_Z"), vel):
            assert np.array_equal(back[name], v[sl]), name
        for a, key in enumerate("xyz"):
            pts = np.arange(1, N[a], st[a])
            assert np.array_equal(back[key], grid.xp[a][pts + 3])
    assert (tmp_path / "IMPACT_xdmf3d_small_00000.xmf").exists()
    assert (tmp_path / "velY_large_00000.bin").stat().st_size == 8 * grid.cells
    w.write(f, 0.25)
    assert (tmp_path / "pre_large_00001.bin").exists() and w.count == 2


def test_physical_scaling(tmp_path):
    grid = I.Grid(N, L, KINDS)
    f = _fields(5)
    sc = X.Scale(L_ref=0.02, U_ref=0.5, rho=1060.0)
    path = X.XdmfWriter(tmp_path, grid, scale=sc).write(f, 2.0, count=7)[0]
    assert path.endswith("IMPACT_xdmf3d_large_00007.xmf")
    back = X.read_output(path)
    assert back["time"] == pytest.approx(2.0 * 0.02 / 0.5)
    assert np.allclose(back["Pressure"], 1060.0 * 0.25 * grid.interior(f["pre"]), rtol=1e-15, atol=0)
    vz = X.velocity_at_pressure_points(grid, f["vel3"], 3)
    assert np.allclose(back["Velocity_Z"], 0.5 * vz, rtol=1e-15, atol=0)
    assert np.allclose(back["x"], 0.02 * grid.xp[0][4:N[0] + 3], rtol=1e-15, atol=0)


def test_stride_must_divide(tmp_path):
    grid = I.Grid(N, L, KINDS)
    with pytest.raises(ValueError):
        X.XdmfWriter(tmp_path / "out", grid, strides={"bad": (3, 1, 1)})  # 16 % 3 != 0


def test_lambda2_matches_restatement(tmp_path):
    n = (13, 9, 11)
    grid, og = I.Grid(n, L, KINDS), O.Grid(n, L, KINDS)
    rng = np.random.default_rng(8)
    vel = og.zeros(3)
    for m in range(3):
        og.interior(vel[m])[...] = rng.uniform(-1.0, 1.0, size=og.interior(vel[m]).shape)
    got = X.lambda2(grid, vel[0], vel[1], vel[2])
    want = R.lambda2(og, vel)
    scale = max(abs(v) for v in want.values())
    for (i, j, k), v in want.items():
        assert abs(got[k - 1, j - 1, i - 1] - v) <= 1e-9 * scale, (i, j, k)
    # the writer's Lambda_2 attribute, scaled by U_ref / L_ref as the reference writes it
    fields = {f"vel{m + 1}": vel[m] for m in range(3)}
    fields["pre"] = og.zeros()
    w = X.XdmfWriter(tmp_path, grid, with_lambda2=True, scale=X.Scale(L_ref=0.5, U_ref=2.0))
    back = X.read_output(w.write(fields, 1.0)[0])
    assert np.allclose(back["Lambda_2"], 4.0 * got, rtol=1e-15, atol=0)  # U_ref / L_ref
