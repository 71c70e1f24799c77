"""The reference's own CT inputs: the TAVI2 lumen segmentation (preprocessing/TAVI2/Segmentation_1.nii)
and the measured inflow waveforms (preprocessing/*/waveform.csv) read through impact_b200.ingest
must give, bit for bit, the CT grid labels and converted tables that the loop restatement of
read_vtk_3D / apply_CT_forcing / convert_waveform (oracle/ct_ingest.py, usr_func.f90:187-651)
gives on the same files -- the fixtures tests/golden/reference_inputs.json and tavi2_labels.npz,
written by tests/golden/make_reference_inputs.py.  The comparison with the files themselves runs
where the reference tree is present (IMPACT_REFERENCE_ROOT, or a directory "reference" beside
this repository); the fixtures' own consistency is checked everywhere.
"""
import json
import os

import numpy as np
import pytest

import impact_b200 as I
from impact_b200 import ingest as G

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
FIX = json.load(open(os.path.join(HERE, "golden", "reference_inputs.json")))
LABELS = np.load(os.path.join(HERE, "golden", "tavi2_labels.npz"))["labels"]


def _ref_root():
    r = os.environ.get("IMPACT_REFERENCE_ROOT") or os.path.join(os.path.dirname(ROOT), "reference")
    return r if os.path.isdir(os.path.join(r, "preprocessing")) else None


def test_fixture_labels_are_consistent_with_the_plane_counts():
    """10 fringe planes per inlet / outlet point: label 5 = 10 x jet points, 7 = 10 x the other
    inlet points, 9 = 10 x first-outlet points, 11 = 10 x second-outlet points."""
    ct = FIX["ct_grid"]
    c = ct["counts"]
    hist = {int(k): v for k, v in ct["label_counts"].items()}
    got = dict(zip(*np.unique(LABELS[4:-4, 4:-4, 4:-4], return_counts=True)))
    assert {int(k): int(v) for k, v in got.items()} == hist
    assert hist[5] == 10 * c["inlet_jet"]
    assert hist[7] == 10 * (c["inlet"] - c["inlet_jet"])
    assert hist[9] == 10 * c["outlet"]
    assert hist[11] == 10 * c["outlet_2"]
    assert LABELS.shape == tuple(n + 7 for n in reversed(ct["points"]))


def test_fixture_waveforms_are_normalised():
    for name, w in FIX["waveforms"].items():
        t, v = np.array(w["time"]), np.array(w["velocity"])
        assert len(t) == w["points"] and np.all(np.diff(t) >= 0.0), name
        if name != "idealized":
            assert v.max() == 1.0, name  # the reference velocity is the peak


@pytest.mark.skipif(_ref_root() is None, reason="the reference tree is not on this machine")
def test_ingest_of_the_reference_files_matches_the_restatement():
    import hashlib

    ref = _ref_root()
    nif = os.path.join(ref, FIX["nifti"]["path"])
    assert hashlib.sha256(open(nif, "rb").read()).hexdigest() == FIX["nifti"]["sha256"]
    vol = G.read_nifti(nif)
    assert list(vol.dims) == FIX["nifti"]["dims"]
    assert list(vol.spacing) == FIX["nifti"]["spacing"]
    ct = FIX["ct_grid"]
    grid = I.Grid(tuple(ct["points"]), tuple(ct["box"]))
    y1p, y2p = G.pressure_coords(grid)
    g = G.ct_grid(vol, ct["points"], ct["offsets"], y1p, y2p, ct["r_inlet"])
    assert g.counts == ct["counts"]
    assert list(g.inlet_centre) == ct["inlet_centre"] and list(g.outlet_centre) == ct["outlet_centre"]
    assert np.array_equal(G.labels_from_ct_grid(g.values, grid), LABELS)
    for name, w in FIX["waveforms"].items():
        path = os.path.join(ref, w["path"])
        assert hashlib.sha256(open(path, "rb").read()).hexdigest() == w["sha256"], name
        cw = G.convert_waveform(G.read_waveform_csv(path), ct["points"][0], idealized=(name == "idealized"))
        assert cw.time.tolist() == w["time"] and cw.velocity.tolist() == w["velocity"], name
        assert (cw.reference_velocity, cw.reference_length, cw.reference_time, cw.Re) == \
               (w["reference_velocity"], w["reference_length"], w["reference_time"], w["Re"]), name
