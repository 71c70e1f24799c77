"""Continuous-batching request loop for vessel simulation cases on one GPU.

Requests (a grid, a label mask, step parameters and a number of time steps) arrive over time.
The loop admits waiting requests in arrival order as soon as their device memory fits inside
the HBM budget, keeps every admitted case's fields resident across its time steps, and advances
all admitted cases together, one time step per round, through a Batch (one launch per operator
of the pressure solve over all cases).  A case that has done its steps is downloaded and freed
between rounds, which opens room for the next requests; the batch is rebuilt whenever its
membership changes.  Each case's result is the same as when it runs alone: the batch keeps
every case's tiles, reductions and convergence decisions separate.

Latency of a request = completion time - arrival time (host wall clock, the loop's own clock).
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from . import Batch, Case, Grid, StepParams


@dataclass
class Request:
    rid: int
    N: tuple                   # grid points per axis (N1, N2, N3), cells = (N - 1) per axis
    L: tuple                   # box lengths
    labels: object             # uint8 label mask in the padded layout, or a callable grid -> mask
    params: StepParams
    nsteps: int
    arrival: float = 0.0       # seconds after the start of the stream
    kinds: tuple = (0, 0, 0)   # coordinate kind per axis
    waveform: object = None    # measured inflow (time, velocity) of a CT case, or None: sinusoid


@dataclass
class Completion:
    rid: int
    arrival: float
    admitted: float
    finished: float
    cells: int
    nsteps: int
    status: list = field(default_factory=list)
    fields: dict | None = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def case_bytes(N, precision: int) -> int:
    """Device memory of one case (fields, Krylov and multigrid work, tables)."""
    return Case.bytes_needed(N, precision)


class Server:
    """Admission by HBM budget, resident fields, one batched time step per round."""

    def __init__(self, hbm_budget: int, precision: int = 1, device: int = 0, max_cases: int = 256,
                 keep=("vel1", "vel2", "vel3", "pre"), backfill: bool = True):
        self.budget = int(hbm_budget)
        self.precision = precision
        self.device = device
        self.max_cases = max_cases
        self.keep = keep
        self.backfill = backfill
        self.rounds = 0
        self.batch_rebuilds = 0
        self.peak_bytes = 0
        self.peak_cases = 0
        # host seconds spent per activity of the loop (admission: case allocation + labels;
        # build: batch construction; step: batched time steps; finish: download + free)
        self.seconds = {"admit": 0.0, "build": 0.0, "step": 0.0, "finish": 0.0}

    def run(self, requests, clock=time.perf_counter, sleep=time.sleep):
        pending = sorted(requests, key=lambda r: r.arrival)
        waiting: list[Request] = []
        active: list[dict] = []
        done: list[Completion] = []
        used = 0
        batch = None
        changed = False
        t0 = clock()
        while pending or waiting or active:
            now = clock() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.pop(0))
            # admission: arrival order; with backfill a later request that fits may pass one that
            # does not fit yet
            q = 0
            while q < len(waiting) and len(active) < self.max_cases:
                r = waiting[q]
                need = case_bytes(r.N, self.precision)
                if used + need <= self.budget:
                    ta = clock()
                    g = Grid(r.N, r.L, r.kinds)
                    c = Case(g, precision=self.precision, device=self.device)
                    lab = r.labels(g) if callable(r.labels) else r.labels
                    c.set_labels(lab)
                    if r.waveform is not None:
                        c.set_inflow_waveform(*r.waveform)
                    active.append({"req": r, "case": c, "bytes": need, "steps": 0, "admitted": clock() - t0})
                    self.seconds["admit"] += clock() - ta
                    used += need
                    waiting.pop(q)
                    changed = True
                    continue
                if need > self.budget:
                    raise ValueError(f"request {r.rid} needs {need} bytes, more than the HBM budget")
                if not self.backfill:
                    break
                q += 1
            self.peak_bytes = max(self.peak_bytes, used)
            self.peak_cases = max(self.peak_cases, len(active))
            if not active:
                if pending:
                    sleep(max(0.0, pending[0].arrival - (clock() - t0)))
                continue
            if changed or batch is None:
                tb = clock()
                if batch is not None:
                    batch.close()
                batch = Batch([a["case"] for a in active])
                self.batch_rebuilds += 1
                changed = False
                self.seconds["build"] += clock() - tb
            ts = clock()
            batch.step([a["req"].params for a in active], 1)
            self.rounds += 1
            tf = clock()
            self.seconds["step"] += tf - ts
            keep_active = []
            for a in active:
                a["steps"] += 1
                if a["steps"] < a["req"].nsteps:
                    keep_active.append(a)
                    continue
                c, r = a["case"], a["req"]
                fields = {f: c.download(f) for f in self.keep} if self.keep else None
                st = list(c.state.poisson_status)
                cells = int(np.prod([n - 1 for n in r.N]))
                done.append(Completion(r.rid, r.arrival, a["admitted"], clock() - t0, cells, r.nsteps, st, fields))
                used -= a["bytes"]
                changed = True
            if changed:
                if batch is not None:
                    batch.close()
                    batch = None
                for a in active:
                    if a not in keep_active:
                        a["case"].close()
            active = keep_active
            self.seconds["finish"] += clock() - tf
        if batch is not None:
            batch.close()
        return done


def summarize(done, wall_s: float):
    """throughput (Mcell-steps/s over the whole stream) and p50 / p99 completion latency (s)"""
    lat = np.array([d.latency for d in done], dtype=np.float64)
    work = sum(d.cells * d.nsteps for d in done)
    return {"requests": len(done), "wall_s": wall_s, "throughput_mcell_steps_s": work / wall_s / 1e6 if wall_s > 0 else None,
            "latency_p50_s": float(np.percentile(lat, 50)) if lat.size else None,
            "latency_p99_s": float(np.percentile(lat, 99)) if lat.size else None,
            "latency_max_s": float(lat.max()) if lat.size else None}


def poisson_arrivals(n: int, rate_per_s: float, rng) -> np.ndarray:
    """arrival times of n requests of a Poisson process with the given mean rate"""
    return np.cumsum(rng.exponential(1.0 / rate_per_s, n))
