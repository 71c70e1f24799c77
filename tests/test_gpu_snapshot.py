"""Snapshots and restart files (impact_b200_case_snapshot, impact_b200.restart): a snapshot read
back on a separate stream holds the fields as they were when it was taken, while the case steps
on; a case loaded from a restart file takes the next steps bit for bit like the case that wrote
it (velocity, pressure, time and step count are the whole state of the time loop)."""
import numpy as np
import pytest
import torch

import impact_b200 as I
from impact_b200 import geometry as G
from impact_b200 import restart

pytestmark = pytest.mark.gpu

N, L = (33, 33, 65), (1.0, 1.0, 2.0)
FIELDS = ("vel1", "vel2", "vel3", "pre")


def _case():
    g = I.Grid(N, L)
    c = I.Case(g, precision=1)
    c.set_labels(G.straight_vessel(g, stenoses=[(1.0, 0.5, 0.125)]))
    return c


def _params():
    return I.step_params(Re=300.0, tol_rel=1e-8, omega=0.8, precond=1, max_it=30, inner_tol_rel=3e-3)


def test_snapshot_holds_the_fields_of_its_moment():
    p = _params()
    a, ref = _case(), _case()
    a.step(p, 2)
    ref.step(p, 2)
    out = [torch.empty(a.grid.shape, dtype=torch.float64, pin_memory=True).numpy() for _ in FIELDS]
    copy = torch.cuda.Stream()
    a.snapshot(FIELDS, out, copy.cuda_stream)
    a.step(p, 1)  # overwrites the fields while the read-back may still run
    copy.synchronize()
    for f, o in zip(FIELDS, out):
        assert np.array_equal(o, ref.download(f)), f
    a.snapshot(("pre",), out[:1])  # a second snapshot reuses the buffer after the first read-back
    a.synchronize()
    assert np.array_equal(out[0], a.download("pre"))
    with pytest.raises(ValueError):
        a.snapshot(("pre", "vel1"), out[:1])
    with pytest.raises(I.ImpactError):
        a.snapshot(("pre", "pre"), out[:2])
    a.close()
    ref.close()


def test_restart_continues_bit_for_bit(tmp_path):
    p = _params()
    a = _case()
    a.step(p, 3)
    path = tmp_path / "restart.npz"
    restart.save(a, path)
    a.step(p, 2)
    b = _case()
    restart.load(b, path)
    assert b.state.timestep == 3
    b.step(p, 2)
    assert b.state.timestep == a.state.timestep and b.state.time == a.state.time
    for f in FIELDS:
        assert np.array_equal(b.download(f), a.download(f)), f
    a.close()
    b.close()
