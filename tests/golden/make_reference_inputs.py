"""Fixtures from the input files the reference ships for its CT cases.

    python tests/golden/make_reference_inputs.py path/to/GPU-IMPACT-CT   (or IMPACT_REFERENCE_ROOT)

Reads, through the oracle's loop restatement of the reference's preparation (oracle/ct_ingest.py:
read_vtk_3D's grid_set, apply_CT_forcing's label tests, convert_waveform):
  * preprocessing/TAVI2/Segmentation_1.nii -- the TAVI2 lumen segmentation (NIfTI-1, 0 / 1 voxels),
    placed on a CT grid of CT_GRID points with CT_OFFSETS as read_vtk_3D places its volume
    (inlet, first and second outlet planes, fringe labels 5 / 7 / 9 / 11);
  * preprocessing/*/Echo waveform/waveform.csv and preprocessing/Idealized Case/waveform/waveform.csv
    -- the measured inflow waveforms, converted to the nondimensional table.
Writes tests/golden/reference_inputs.json (file checksums, volume facts, CT-grid counts and
centres, converted waveforms) and tests/golden/tavi2_labels.npz (the CT grid's uint8 labels in the
library's padded field layout), so that the tests and the device tests need no reference tree.
The NIfTI header is decoded here with the struct module (the reader under test is not used).
"""
import hashlib
import json
import math
import os
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle")]

import ct_ingest as R  # noqa: E402

CT_GRID = (161, 81, 161)      # points per axis (160 x 80 x 160 cells, periodic box)
CT_BOX = (1.0, 0.5, 1.0)      # equal spacing 1/160 on every axis
CT_OFFSETS = (4, 4, 16)       # x, y, z offsets of the volume in the grid (read_vtk_3D)
R_INLET = 0.04                # radius of the incoming jet, in box units
WAVEFORMS = {"TAVI0": "preprocessing/TAVI0/Echo waveform/waveform.csv",
             "TAVI1": "preprocessing/TAVI1/Echo waveform/waveform.csv",
             "TAVI2": "preprocessing/TAVI2/Echo waveform/waveform.csv",
             "idealized": "preprocessing/Idealized Case/waveform/waveform.csv"}
NIFTI = "preprocessing/TAVI2/Segmentation_1.nii"


def sha256(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def nifti_values(path):
    """dims, voxel sizes and values (x fastest) of a little- or big-endian NIfTI-1 float/int volume."""
    raw = open(path, "rb").read()
    end = "<" if struct.unpack("<i", raw[:4])[0] == 348 else ">"
    dim = struct.unpack(end + "8h", raw[40:56])
    dtype = {2: "u1", 4: "i2", 8: "i4", 16: "f4", 64: "f8", 256: "i1", 512: "u2", 768: "u4"}[
        struct.unpack(end + "h", raw[70:72])[0]]
    pixdim = struct.unpack(end + "8f", raw[76:108])
    off = int(struct.unpack(end + "f", raw[108:112])[0])
    slope, inter = struct.unpack(end + "2f", raw[112:120])
    n = dim[1] * dim[2] * dim[3]
    v = np.frombuffer(raw, dtype=np.dtype(dtype).newbyteorder(end), count=n, offset=off).astype(np.float64)
    if slope != 0.0:
        v = v * float(slope) + float(inter)
    return (dim[1], dim[2], dim[3]), tuple(float(p) for p in pixdim[1:4]), v


def waveform_table(path):
    rows = []
    for text in open(path):
        parts = text.replace(",", " ").split()
        if len(parts) >= 2:
            rows.append((float(parts[0]), float(parts[1])))
    return rows


def pressure_coords(M, L):
    """1-based pressure coordinates of an equidistant periodic axis: x_i = (i - 1) L / (M - 1)."""
    return [math.nan] + [(i - 1) * L / (M - 1) for i in range(1, M + 1)]


def main(ref):
    out = {"source": "GPU-IMPACT-CT preprocessing/ inputs, through oracle/ct_ingest.py", "waveforms": {}}
    dims, spacing, vals = nifti_values(os.path.join(ref, NIFTI))
    u, c = np.unique(vals, return_counts=True)
    out["nifti"] = {"path": NIFTI, "sha256": sha256(os.path.join(ref, NIFTI)), "dims": list(dims),
                    "spacing": list(spacing), "values": {repr(float(a)): int(b) for a, b in zip(u, c)}}
    y1p, y2p = pressure_coords(CT_GRID[0], CT_BOX[0]), pressure_coords(CT_GRID[1], CT_BOX[1])
    g, cin, cout, counts = R.grid_set(list(vals), dims, CT_GRID, CT_OFFSETS, y1p, y2p, R_INLET)
    M1, M2, M3 = CT_GRID
    lab = np.zeros((M3 + 7, M2 + 7, M1 + 7), dtype=np.uint8)  # padded layout, unique points 1..M-1
    hist = {}
    for k in range(1, M3):
        for j in range(1, M2):
            for i in range(1, M1):
                v = R.label(g[(i, j, k)])
                lab[k + 3, j + 3, i + 3] = v
                hist[v] = hist.get(v, 0) + 1
    np.savez_compressed(os.path.join(HERE, "tavi2_labels.npz"), labels=lab)
    out["ct_grid"] = {"points": list(CT_GRID), "box": list(CT_BOX), "offsets": list(CT_OFFSETS), "r_inlet": R_INLET,
                      "counts": counts, "inlet_centre": list(cin), "outlet_centre": list(cout),
                      "label_counts": {str(k): v for k, v in sorted(hist.items())}}
    for name, rel in WAVEFORMS.items():
        path = os.path.join(ref, rel)
        table = waveform_table(path)
        t, v, u_ref, l_ref, t_ref, Re = R.converted(table, CT_GRID[0], idealized=(name == "idealized"))
        out["waveforms"][name] = {"path": rel, "sha256": sha256(path), "points": len(table), "time": t,
                                  "velocity": v, "reference_velocity": u_ref, "reference_length": l_ref,
                                  "reference_time": t_ref, "Re": Re}
    with open(os.path.join(HERE, "reference_inputs.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote reference_inputs.json and tavi2_labels.npz:", counts, hist)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("IMPACT_REFERENCE_ROOT")
    if not root:
        sys.exit("usage: make_reference_inputs.py path/to/GPU-IMPACT-CT (or set IMPACT_REFERENCE_ROOT)")
    main(root)
