"""A CT-based case on the device: labels from a synthetic CT volume through read_vtk_3D's
preparation (impact_b200.ingest), and the measured inflow waveform (Case.set_inflow_waveform) that
the end of every time step imposes on the inflow voxels: after each step they hold the table value
the oracle's lookup gives for the step's time (apply_CT_forcing, usr_func.f90:929-945), the
no-flow voxels hold zero, and clearing the waveform restores the sinusoidal inflow.
"""
import math

import numpy as np
import pytest

import ct_ingest as R
import impact_b200 as I
from impact_b200 import ingest as G

pytestmark = pytest.mark.gpu

N = (33, 33, 65)
OFFSETS = (4, 4, 10)
DIMS = (24, 24, 40)


def _case():
    d1, d2, d3 = DIMS
    v = np.zeros((d3, d2, d1))
    jj, ii = np.meshgrid(np.arange(1, d2 + 1), np.arange(1, d1 + 1), indexing="ij")
    for k in range(d3):
        v[k][(jj - 7.0) ** 2 + (ii - 12.0) ** 2 <= 16.0] = 1.0   # ascending: first index j + 4 < 16
        v[k][(jj - 19.0) ** 2 + (ii - 12.0) ** 2 <= 9.0] = 1.0   # descending
    vol = G.VtkVolume(DIMS, (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), v.reshape(-1))
    grid = I.Grid(N, (1.0, 1.0, 2.0))
    y1p, y2p = G.pressure_coords(grid)
    ct = G.ct_grid(vol, N, OFFSETS, y1p, y2p, 0.06)
    assert ct.counts["inlet_jet"] > 0
    lab = G.labels_from_ct_grid(ct.values, grid)
    case = I.Case(grid, precision=0)
    case.set_labels(lab)
    return case, lab


def test_measured_inflow_waveform_on_the_device():
    case, lab = _case()
    p = I.step_params(Re=200.0, tol_rel=1e-8, n_sweeps=4, omega=0.8, precond=1, dtime_max=2e-3)
    times = np.linspace(0.0, 0.02, 9)
    vels = 0.3 + np.arange(9) * 0.1
    case.set_inflow_waveform(times, vels)
    inflow, noflow = lab == 5, (lab == 0) | (lab == 7)
    assert inflow.any() and noflow.any()
    for _ in range(4):
        st = case.step(p)
        want = R.inflow(list(times), list(vels), st.time)
        w = case.download("vel3")
        assert want is not None
        assert np.all(w[inflow] == want)
        assert np.all(case.download("vel1")[inflow] == 0.0)
        for f in ("vel1", "vel2", "vel3"):
            assert np.all(case.download(f)[noflow] == 0.0)
    case.set_inflow_waveform(None)
    st = case.step(p)
    sinus = p.U0 * (1.0 + 0.5 * math.sin(2.0 * math.pi * st.time / p.T_pulse))
    assert np.allclose(case.download("vel3")[inflow], sinus, rtol=0, atol=1e-15)
    with pytest.raises(I.ImpactError):
        case.set_inflow_waveform([0.0, 1.0, 0.5], [1.0, 1.0, 1.0])  # times must not decrease
    case.close()


def test_reference_tavi2_case_steps_like_the_oracle():
    """The TAVI2 case built from the reference's own lumen segmentation (the CT grid labels of
    tests/golden/tavi2_labels.npz, 160 x 80 x 160 cells): three FP64 steps on the device with the
    multigrid-preconditioned solve equal the oracle's to 1e-6 of max|u|; then the case takes its
    measured TAVI2 inflow waveform (converted table of the fixture) and the inflow voxels hold the
    oracle lookup's value after every step."""
    import json
    import os

    import oracle as O

    here = os.path.dirname(os.path.abspath(__file__))
    fix = json.load(open(os.path.join(here, "golden", "reference_inputs.json")))
    lab = np.load(os.path.join(here, "golden", "tavi2_labels.npz"))["labels"]
    Np, L = tuple(fix["ct_grid"]["points"]), tuple(fix["ct_grid"]["box"])
    og, ig = O.Grid(Np, L), I.Grid(Np, L)
    mg = og.multigrid()
    vel, nl, pre = og.zeros(3), og.zeros(3), og.zeros()
    ost = O.OrcStepState()
    op = O.step_params(Re=200.0, tol_rel=1e-8, omega=0.8, mg=mg, mg_down=3, mg_up=3, mg_bottom=3)
    case = I.Case(ig, precision=0)
    case.set_labels(lab)
    sp = I.step_params(Re=200.0, tol_rel=1e-8, omega=0.8, precond=1, max_it=200, mg_down=3, mg_up=3, mg_bottom=3)
    for _ in range(3):
        og.time_step(op, lab, vel, nl, pre, ost)
        st = case.step(sp)
        assert all(s == 0 for s in st.poisson_status)
    umax = max(np.abs(og.interior(vel[m])).max() for m in range(3))
    for m, f in enumerate(("vel1", "vel2", "vel3")):
        assert np.abs(og.interior(case.download(f)) - og.interior(vel[m])).max() <= 1e-6 * umax
    w = fix["waveforms"]["TAVI2"]
    case.set_inflow_waveform(np.array(w["time"]), np.array(w["velocity"]))
    inflow = lab == 5
    assert inflow.sum() == 10 * fix["ct_grid"]["counts"]["inlet_jet"]
    for _ in range(2):
        st = case.step(sp)
        want = R.inflow(w["time"], w["velocity"], st.time)
        assert want is not None
        assert np.all(case.download("vel3")[inflow] == want)
    case.close()
