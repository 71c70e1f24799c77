"""The serving loop's host logic (impact_b200.serve.Server) with the device case and batch replaced
by recording stand-ins and a virtual clock: admission in arrival order within the HBM budget,
backfill of a later request that fits past one that does not, the batch rebuilt whenever its
membership changes, completions after each request's number of steps, latency = completion -
arrival, the peak budget use (request 1 alone after requests 0 and 2 together), and the error for a
request larger than the whole budget."""
import pytest

from impact_b200 import serve as S


class Clock:
    """Virtual time: a batched step costs 1 s per case in the batch; sleeping jumps ahead."""

    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(0.0, dt)


class FakeState:
    poisson_status = (0, 0, 0)


class FakeCase:
    live = []

    def __init__(self, grid, precision=1, device=0):
        self.grid, self.closed, self.labels = grid, False, None
        self.state = FakeState()
        FakeCase.live.append(self)

    def set_labels(self, lab):
        self.labels = lab

    def set_inflow_waveform(self, time=None, velocity=None):
        self.waveform = (time, velocity)

    def download(self, f):
        return f

    def close(self):
        self.closed = True


class FakeGrid:
    def __init__(self, N, L, kinds):
        self.N = N


def _install(monkeypatch, clock, sizes):
    log = []

    class FakeBatch:
        def __init__(self, cases):
            self.cases = list(cases)
            log.append(("build", tuple(c.grid.N for c in self.cases)))

        def step(self, params, n):
            assert len(params) == len(self.cases) and n == 1
            log.append(("step", tuple(c.grid.N for c in self.cases)))
            clock.t += 1.0 * len(self.cases)

        def close(self):
            pass

    monkeypatch.setattr(S, "Case", FakeCase)
    monkeypatch.setattr(S, "Grid", FakeGrid)
    monkeypatch.setattr(S, "Batch", FakeBatch)
    monkeypatch.setattr(S, "case_bytes", lambda N, precision: sizes[N])
    return log


def _req(rid, n, arrival, steps):
    return S.Request(rid, (n, n, n), (1.0, 1.0, 1.0), "labels", None, steps, arrival)


def test_admission_backfill_and_completions(monkeypatch):
    clock = Clock()
    sizes = {(10, 10, 10): 40, (20, 20, 20): 80, (30, 30, 30): 30}
    log = _install(monkeypatch, clock, sizes)
    FakeCase.live = []
    reqs = [_req(0, 10, 0.0, 3), _req(1, 20, 0.5, 2), _req(2, 30, 0.5, 1)]
    srv = S.Server(100, precision=1, keep=("vel1",), backfill=True)
    done = srv.run(reqs, clock=clock, sleep=clock.sleep)
    # request 1 (80) does not fit beside request 0 (40); request 2 (30) backfills past it
    order = [d.rid for d in done]
    assert order == [2, 0, 1]
    byid = {d.rid: d for d in done}
    assert byid[0].admitted == 0.0 and byid[2].admitted == 1.0  # admitted after the first round
    assert byid[1].admitted >= byid[0].finished  # waits for request 0's memory
    assert all(d.latency == d.finished - d.arrival for d in done)
    assert srv.peak_bytes == 80 and srv.peak_cases == 2  # request 1 alone; requests 0 and 2 together
    assert all(c.closed for c in FakeCase.live) and all(c.labels == "labels" for c in FakeCase.live)
    # a build before every round whose membership changed
    builds = [e for e in log if e[0] == "build"]
    assert builds[0][1] == ((10, 10, 10),) and ((10, 10, 10), (30, 30, 30)) in [b[1] for b in builds]
    assert srv.batch_rebuilds == len(builds)
    steps = {}
    for kind, members in log:
        if kind == "step":
            for m in members:
                steps[m] = steps.get(m, 0) + 1
    assert steps == {(10, 10, 10): 3, (20, 20, 20): 2, (30, 30, 30): 1}
    assert done[0].fields == {"vel1": "vel1"}
    stats = S.summarize(done, clock.t)
    assert stats["requests"] == 3 and stats["latency_max_s"] == max(d.latency for d in done)


def test_without_backfill_requests_wait_in_order(monkeypatch):
    clock = Clock()
    sizes = {(10, 10, 10): 40, (20, 20, 20): 80, (30, 30, 30): 30}
    _install(monkeypatch, clock, sizes)
    FakeCase.live = []
    reqs = [_req(0, 10, 0.0, 3), _req(1, 20, 0.5, 2), _req(2, 30, 0.5, 1)]
    done = S.Server(100, precision=1, keep=(), backfill=False).run(reqs, clock=clock, sleep=clock.sleep)
    byid = {d.rid: d for d in done}
    assert byid[2].admitted >= byid[1].admitted  # no passing
    assert byid[0].fields is None


def test_request_beyond_the_budget_is_an_error(monkeypatch):
    clock = Clock()
    _install(monkeypatch, clock, {(10, 10, 10): 500})
    with pytest.raises(ValueError):
        S.Server(100).run([_req(0, 10, 0.0, 1)], clock=clock, sleep=clock.sleep)


def test_idle_loop_sleeps_until_the_next_arrival(monkeypatch):
    clock = Clock()
    _install(monkeypatch, clock, {(10, 10, 10): 10})
    done = S.Server(100).run([_req(0, 10, 5.0, 1)], clock=clock, sleep=clock.sleep)
    assert done[0].admitted == 5.0 and done[0].finished == 6.0 and done[0].latency == 1.0


def test_ct_request_carries_its_inflow_waveform(monkeypatch):
    clock = Clock()
    _install(monkeypatch, clock, {(10, 10, 10): 10, (20, 20, 20): 10})
    FakeCase.live = []
    wf = ([0.0, 0.5, 1.0], [0.2, 0.9, 0.2])
    reqs = [S.Request(0, (10, 10, 10), (1.0, 1.0, 1.0), "labels", None, 1, 0.0, waveform=wf),
            _req(1, 20, 0.0, 1)]
    S.Server(100).run(reqs, clock=clock, sleep=clock.sleep)
    byN = {c.grid.N: c for c in FakeCase.live}
    assert byN[(10, 10, 10)].waveform == wf
    assert not hasattr(byN[(20, 20, 20)], "waveform")  # the default sinusoidal inflow
