"""Geometry and waveform ingest (impact_b200.ingest) against the literal restatement of
read_vtk_3D, convert_waveform and the inflow lookup of apply_CT_forcing (oracle/ct_ingest.py,
usr_func.f90:283-651, 899-945): the CT grid bit for bit on a synthetic volume whose lumen reaches
both halves of the inlet plane (the column i = M1 / 2 belongs to the inlet and the first outlet,
and the outlet fringe overwrites the inlet's), the label mask, the converted waveform and the
inflow at table times, between them, before the first one and over several pulses; VTK files in
ASCII and big-endian binary, NIfTI-1 volumes in either byte order, gzip-compressed and scaled;
the Windkessel inlet and outlet pressures of get_pressure_waveform_echo_WKM (usr_func.f90:653-750)
and the analytic branches of get_pressure_and_flow_rate_WKM (:762-855);
and the errors for volumes that do not fit.
"""
import math
import struct

import numpy as np
import pytest

import ct_ingest as R
import impact_b200 as I
from impact_b200 import ingest as G

M = (17, 17, 37)
OFFSETS = (3, 2, 10)
DIMS = (10, 12, 14)  # d1 (VTK i), d2 (j), d3 (k)


def _volume(seed=0):
    """A lumen of two discs in every plane (one each side of the grid's x midline once the volume
    is placed), lumen value 1, tissue 0, a few in-between values."""
    d1, d2, d3 = DIMS
    rng = np.random.default_rng(seed)
    v = np.zeros((d3, d2, d1))
    jj, ii = np.meshgrid(np.arange(1, d2 + 1), np.arange(1, d1 + 1), indexing="ij")
    for k in range(d3):
        a = (jj - 4.5) ** 2 + (ii - 4.0 - 0.1 * k) ** 2 <= 6.0   # first index j + 2: up to M1 / 2
        b = (jj - 10.0) ** 2 + (ii - 6.0) ** 2 <= 4.0             # -> above M1 / 2
        v[k][a | b] = 1.0
    v[rng.random(v.shape) < 0.03] = 0.7  # lumen-like values other than 1
    v[rng.random(v.shape) < 0.02] = 0.3
    return G.VtkVolume(DIMS, (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), v.reshape(-1))


def _grid():
    return I.Grid(M, (1.0, 1.0, 2.0))


def test_vtk_ascii_round_trip(tmp_path):
    vol = _volume()
    p = tmp_path / "ct.vtk"
    G.write_vtk_structured_points(p, vol)
    back = G.read_vtk_structured_points(p)
    assert back.dims == vol.dims
    assert np.array_equal(back.values, vol.values)


@pytest.mark.parametrize("scalar,fmt", [("double", ">d"), ("float", ">f")])
def test_vtk_binary_big_endian(tmp_path, scalar, fmt):
    vals = np.arange(24, dtype=np.float64) / 4.0
    head = ("# vtk DataFile Version 3.0\nb\nBINARY\nDATASET STRUCTURED_POINTS\nDIMENSIONS 2 3 4\n"
            "SPACING 1 1 1\nORIGIN 0 0 0\nPOINT_DATA 24\nSCALARS s %s 1\nLOOKUP_TABLE default\n" % scalar)
    p = tmp_path / "b.vtk"
    p.write_bytes(head.encode() + b"".join(struct.pack(fmt, v) for v in vals))
    v = G.read_vtk_structured_points(p)
    assert v.dims == (2, 3, 4)
    assert np.array_equal(v.values, vals)


def test_ct_grid_matches_restatement():
    vol, grid = _volume(1), _grid()
    y1p, y2p = G.pressure_coords(grid)
    r_in = 0.12
    got = G.ct_grid(vol, M, OFFSETS, y1p, y2p, r_in)
    want, cin, cout, counts = R.grid_set(vol.values, DIMS, M, OFFSETS, y1p, y2p, r_in)
    g = got.values
    assert g.shape == M
    for (i, j, k), v in want.items():
        assert g[i - 1, j - 1, k - 1] == v, (i, j, k)
    assert got.inlet_centre == cin and got.outlet_centre == cout
    assert got.counts == counts
    # the volume exercises every label: the jet, the inlet ring, both outlets, the shared column
    assert counts["inlet_jet"] > 0 and counts["inlet"] > counts["inlet_jet"] and counts["outlet_2"] > 0
    assert np.any(g == 5.0) and np.any(g == 7.0) and np.any(g == 9.0) and np.any(g == 11.0)
    half = M[0] // 2
    assert np.any(g[half - 1, :, OFFSETS[2] - 1] == 9.0)  # plane k_start - 1 of the shared column


def test_labels_match_forcing_classes():
    vol, grid = _volume(2), _grid()
    y1p, y2p = G.pressure_coords(grid)
    ct = G.ct_grid(vol, M, OFFSETS, y1p, y2p, 0.12).values
    lab = G.labels_from_ct_grid(ct, grid)
    N1, N2, N3 = M
    assert lab.shape == (N3 + 7, N2 + 7, N1 + 7) and lab.dtype == np.uint8
    for k in range(1, N3):
        for j in range(1, N2):
            for i in range(1, N1):
                assert lab[k + 3, j + 3, i + 3] == R.label(ct[i - 1, j - 1, k - 1])
    inner = np.zeros(lab.shape, dtype=bool)
    inner[4:N3 + 3, 4:N2 + 3, 4:N1 + 3] = True
    assert not lab[~inner].any()


def _table():
    t = np.arange(5.0, 805.0, 10.0)  # ms; the first point at 5 ms leaves [0, 5 ms) uncovered
    v = 0.2 + 0.8 * np.sin(np.pi * (t - 5.0) / 800.0) ** 2
    return np.stack([t, v], axis=1)


@pytest.mark.parametrize("idealized", [False, True])
def test_waveform_conversion_and_lookup(tmp_path, idealized):
    tab = _table()
    p = tmp_path / "waveform.csv"
    p.write_text("".join(f"{a:.6f},{b:.6f}\n" for a, b in tab))
    tab = G.read_waveform_csv(p)
    w = G.convert_waveform(tab, M[0], idealized=idealized)
    times, vels, u_ref, l_ref, t_ref, Re = R.converted([tuple(r) for r in tab], M[0], idealized=idealized)
    assert np.array_equal(w.time, np.array(times)) and np.array_equal(w.velocity, np.array(vels))
    assert (w.reference_velocity, w.reference_length, w.reference_time, w.Re) == (u_ref, l_ref, t_ref, Re)
    length = times[-1]
    probes = [0.0, 0.5 * times[0], times[0], times[3], 0.5 * (times[3] + times[4]), times[-1],
              length + times[10], 3 * length + 0.25 * (times[7] + times[8]) * 2]
    for t in probes:
        assert G.inflow_velocity(w.time, w.velocity, t) == R.inflow(times, vels, t), t
    assert G.inflow_velocity(w.time, w.velocity, 0.5 * times[0]) is None
    # at a table time the later interval wins
    assert G.inflow_velocity(w.time, w.velocity, times[3]) == vels[3]
    # Windkessel pressures for the pressure boundary condition (two updates at a table time)
    for t in probes:
        assert G.windkessel_pressures(tab, w, t) == R.windkessel([tuple(r) for r in tab], times, u_ref, t), t


def test_analytic_windkessel_branches():
    """get_pressure_and_flow_rate_WKM: systolic closed form, then the diastolic decay from the
    branch's last systolic pressure, for the inlet and both outlets, over two beats."""
    t_ref, u_ref, l_ref = 0.05, 1.3, 0.012
    got = G.AnalyticWindkessel(t_ref, u_ref, l_ref)
    want = R.windkessel_wkm(t_ref, u_ref, l_ref)
    times = [0.0, 0.5, 3.0, 7.999, 8.0, 8.1, 12.0, 19.9]  # x t_ref: systole ends at 0.4 s = t 8
    for t in times:
        for b in (1, 2, 3):
            assert got(b, t) == want(b, t), (b, t)
    p_sys, q_sys = got(1, 4.0)
    assert q_sys > 0.0 and p_sys > 0.0
    p_dia, q_dia = got(1, 12.0)
    assert q_dia == 0.0 and 0.0 < p_dia < got(1, 8.0)[0]  # decays from the end-systolic value
    fresh = G.AnalyticWindkessel(t_ref, u_ref, l_ref)
    assert fresh(2, 12.0) == (0.0, 0.0)  # no systole seen yet: the reference's zero initial state
    resumed = G.AnalyticWindkessel(t_ref, u_ref, l_ref, end_systole=tuple(got.end_systole[b] for b in (1, 2, 3)))
    assert resumed(3, 15.0) == got(3, 15.0)


def test_jor_pressures():
    a, b = (8. / 15., 5. / 12., 3. / 4.), (0., -17. / 60., -5. / 12.)
    for sub in (1, 2, 3):
        got = G.jor_pressures(0.3, -0.2, 0.05, sub, 1.7e-3)
        assert got == tuple(p * (a[sub - 1] + b[sub - 1]) * 1.7e-3 for p in (0.3, -0.2, 0.05))
    assert math.isclose(G.jor_pressures(3.0, 0.0, 0.0, 3, 1.0)[0], 1.0)  # aRK + bRK = 1/3


def test_ingest_rejects_volumes_that_do_not_fit():
    vol, grid = _volume(), _grid()
    y1p, y2p = G.pressure_coords(grid)
    with pytest.raises(ValueError):
        G.ct_grid(vol, (13, 17, 37), OFFSETS, y1p, y2p, 0.1)  # d2 + y offset > M1
    with pytest.raises(ValueError):
        G.ct_grid(vol, M, (3, 2, 5), y1p, y2p, 0.1)  # inlet fringe below plane 1
    with pytest.raises(ValueError):
        G.ct_grid(vol, (17, 17, 30), OFFSETS, y1p, y2p, 0.1)  # second-outlet fringe past the top
    with pytest.raises(ValueError):
        G.labels_from_ct_grid(np.zeros((5, 5, 5)), grid)
    assert math.isclose(G.inlet_radius(2.7, 0.2), math.sqrt(0.0004 / (math.pi * 2.7)) / 0.2)


def _nifti_bytes(vals, dims, dtype_code, np_dtype, end, slope=0.0, inter=0.0, pixdim=(0.5, 0.6, 0.7)):
    hdr = bytearray(352)
    struct.pack_into(end + "i", hdr, 0, 348)
    struct.pack_into(end + "8h", hdr, 40, 3, *dims, 1, 1, 1, 1)
    struct.pack_into(end + "h", hdr, 70, dtype_code)
    struct.pack_into(end + "h", hdr, 72, np.dtype(np_dtype).itemsize * 8)
    struct.pack_into(end + "8f", hdr, 76, 1.0, *pixdim, 1.0, 1.0, 1.0, 1.0)
    struct.pack_into(end + "f", hdr, 108, 352.0)
    struct.pack_into(end + "2f", hdr, 112, slope, inter)
    hdr[344:348] = b"n+1\0"
    return bytes(hdr) + np.asarray(vals, dtype=np.dtype(np_dtype).newbyteorder(end)).tobytes()


@pytest.mark.parametrize("end", ["<", ">"])
@pytest.mark.parametrize("code,np_dtype", [(2, "u1"), (16, "f4"), (64, "f8"), (4, "i2")])
def test_nifti_volume(tmp_path, end, code, np_dtype):
    dims = (4, 3, 5)
    vals = (np.arange(60) % 7).astype(np.float64)
    p = tmp_path / "ct.nii"
    p.write_bytes(_nifti_bytes(vals, dims, code, np_dtype, end))
    v = G.read_nifti(p)
    assert v.dims == dims and np.array_equal(v.values, vals)
    assert v.spacing == pytest.approx((0.5, 0.6, 0.7))


def test_nifti_gzip_and_scaling(tmp_path):
    import gzip

    vals = np.arange(24, dtype=np.float64)
    p = tmp_path / "ct.nii.gz"
    with gzip.open(p, "wb") as f:
        f.write(_nifti_bytes(vals, (2, 3, 4), 4, "i2", "<", slope=0.5, inter=1.0))
    v = G.read_nifti(p)
    assert np.array_equal(v.values, vals * 0.5 + 1.0)
    bad = tmp_path / "bad.nii"
    bad.write_bytes(b"\0" * 400)
    with pytest.raises(ValueError):
        G.read_nifti(bad)
