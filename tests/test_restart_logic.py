"""Restart files (impact_b200.restart) with the device case replaced by a stand-in: save writes
velocity, pressure, time, step count and the grid through Case.snapshot, load uploads the same
arrays and restores the time and step count, a file of another grid is refused, and the
analytic Windkessel end-systolic state goes along when asked."""
import numpy as np
import pytest

from impact_b200 import restart


class FakeGrid:
    def __init__(self, N):
        self.N, self.L, self.kinds = N, (1.0, 1.0, 2.0), (0, 0, 0)
        self.shape = (N[2] + 7, N[1] + 7, N[0] + 7)


class FakeState:
    time, timestep = 0.0, 0


class FakeCase:
    def __init__(self, N, seed=0):
        self.grid, self.state = FakeGrid(N), FakeState()
        rng = np.random.default_rng(seed)
        self.fields = {f: rng.random(self.grid.shape) for f in restart.STATE}
        self.synced = False

    def snapshot(self, fields, out, stream=0):
        for f, o in zip(fields, out):
            o[...] = self.fields[f]

    def synchronize(self):
        self.synced = True

    def upload(self, f, a):
        assert a.flags["C_CONTIGUOUS"]
        self.fields[f] = a.copy()


def test_save_and_load(tmp_path):
    a = FakeCase((9, 10, 11), seed=1)
    a.state.time, a.state.timestep = 0.125, 7
    path = tmp_path / "r.npz"
    restart.save(a, path)
    assert a.synced
    b = FakeCase((9, 10, 11), seed=2)
    restart.load(b, path)
    assert b.state.time == 0.125 and b.state.timestep == 7
    for f in restart.STATE:
        assert np.array_equal(b.fields[f], a.fields[f])
    with pytest.raises(ValueError):
        restart.load(FakeCase((9, 10, 13)), path)


def test_windkessel_state_round_trip(tmp_path):
    from impact_b200 import ingest

    wk = ingest.AnalyticWindkessel(0.05, 1.3, 0.012)
    for b in (1, 2, 3):
        wk(b, 6.0)  # systole: each branch remembers its pressure
    a = FakeCase((9, 10, 11), seed=3)
    path = tmp_path / "wk.npz"
    restart.save(a, path, windkessel=wk)
    back = ingest.AnalyticWindkessel(0.05, 1.3, 0.012)
    restart.load(FakeCase((9, 10, 11)), path, windkessel=back)
    assert back.end_systole == wk.end_systole
    assert back(2, 14.0) == wk(2, 14.0)  # the same diastolic decay
    plain = tmp_path / "plain.npz"
    restart.save(a, plain)
    with pytest.raises(ValueError):
        restart.load(FakeCase((9, 10, 11)), plain, windkessel=back)
