#!/usr/bin/env python
"""bench.py -- IMPACT fractional-step throughput on B200: Mcell-steps/s at a 1e-8 relative
pressure residual, mixed precision (headline) vs plain FP64.

Workload (default, the mixed-precision single case of the benchmark suite): stenosed vessel on a
384 x 384 x 768 periodic box (L = 1 x 1 x 2, uniform spacing); cylinder of radius 0.25 L1 with a
Gaussian constriction at mid-length (60 % area reduction, sigma = 0.5 R); pulsatile plug inflow
u_z = U0 (1 + 0.5 sin(2 pi t / T)), U0 = 1, T = 1, on the label-5 buffer; Re = 500; dt = 0.2 x the
RK3 stability limit (get_dtime with CFL = 0.2); every Poisson solve is BiCGstab with the
multigrid V-cycle preconditioner (damped Jacobi, omega = 0.8; sweeps and tile depth chosen by the
autotuner during warm-up) to ||b - A x||_2 <= 1e-8 ||b||_2: FP32 inner solve with FP64 refinement
(the line), plain FP64 beside it.  Starts from rest.  One "step" is one RK3 time step (3
substeps, 3 Poisson solves).  Fields are ~0.95 GB each, far larger than L2, so no flush is
needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--size n]

With N > 1 (launched by torchrun, one rank per GPU) every rank advances an independent replica
of the case (the path does not shard: replicas only) and `value` is the whole-job aggregate.
`--impl reference` times IMPACT's CPU algorithm (the FP64 oracle restatement, all host cores)
on bounded samples of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-impact-ct_b200"))

METRIC = "Mcell-steps/s at 1e-8 pressure residual, mixed vs FP64; serve p50/p99 latency"
UNIT = "Mcell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=384, help="cells per x/y axis (z has twice as many)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the plain FP64 comparison run")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--n-sweeps", type=int, default=4)
    ap.add_argument("--inner-tol", type=float, default=3e-3,
                    help="relative tolerance of each FP32 inner solve (batch and serve cases, and --no-tune)")
    ap.add_argument("--precond", type=int, default=1, help="0: JOR sweeps, 1: multigrid V-cycle (default)")
    ap.add_argument("--check-every", type=int, default=2)
    ap.add_argument("--workload", default="single", choices=["single", "batch", "serve", "kernels"],
                    help="single: the 384 mixed case (default line, with short batch and serve samples); "
                         "batch / serve: the full batched or serving workload as the line; kernels: per-kernel "
                         "micro-benchmark on resident random fields (the small case for profilers)")
    ap.add_argument("--kernels", default="all", help="kernels: comma-separated names to run (default all)")
    ap.add_argument("--iters", type=int, default=20, help="kernels: timed launches per kernel")
    ap.add_argument("--no-extra", action="store_true", help="skip the batch and serve samples of the default line")
    ap.add_argument("--no-tune", action="store_true", help="keep --tile-kc and --sweeps (no autotuning)")
    ap.add_argument("--sweeps", type=int, default=3,
                    help="V-cycle sweeps down / up / bottom of the batch and serve cases, and of the single case "
                         "with --no-tune (default: the autotuner's choice on the 384 case)")
    ap.add_argument("--tile-kc", type=int, default=64, help="tile depth of the solver kernels, as --sweeps")
    ap.add_argument("--copy-chunks", type=int, default=8,
                    help="element ranges per field of the end-to-end copies (download and next upload pipeline)")
    ap.add_argument("--no-profile", action="store_true", help="no per-kernel events in the timed steps (no roofline)")
    ap.add_argument("--cases", type=int, default=48, help="batch: number of cases")
    ap.add_argument("--requests", type=int, default=16, help="serve: number of requests")
    ap.add_argument("--case-steps", type=int, default=0, help="batch / serve: time steps per case (0: the spec's)")
    return ap.parse_args()


def workload(n):
    return {"workload": f"stenosed-vessel-{n}x{n}x{2 * n}", "cells": n * n * 2 * n, "box": [1.0, 1.0, 2.0],
            "radius": 0.25, "stenosis": {"z": 1.0, "area_reduction": 0.6, "sigma": 0.125}, "Re": 500.0,
            "inflow": "U0 (1 + 0.5 sin(2 pi t / T)), U0 = 1, T = 1", "dt": "0.2 x CFL limit",
            "poisson": "BiCGstab + multigrid V-cycle (damped Jacobi, omega 0.8, sweeps and tile depth autotuned) to 1e-8 "
                       "relative", "start": "rest",
            "l2_flush": "not needed: every field (0.95 GB at 384) exceeds the 126 MB L2"}


def build_case(n, precision, device):
    import impact_b200 as I
    from impact_b200 import geometry as G
    N = (n + 1, n + 1, 2 * n + 1)
    grid = I.Grid(N, (1.0, 1.0, 2.0))
    lab = G.straight_vessel(grid, radius_frac=0.25, stenoses=[(1.0, 0.6, 0.125)])
    case = I.Case(grid, precision=precision, device=device)
    case.set_labels(lab)
    return grid, lab, case


def step_params(args, precision):
    import impact_b200 as I
    return I.step_params(Re=500.0, CFL=0.2, dtime_max=1.0, dtime0=1e9, U0=1.0, T_pulse=1.0, level_pressure=1,
                         tol_rel=1e-8, max_it=(5000 if args.precond == 0 else 200) if precision == 0 else 40,
                         n_sweeps=args.n_sweeps, omega=0.8, init_yes=0, check_every=args.check_every,
                         inner_tol_rel=args.inner_tol, inner_max_it=4000 if args.precond == 0 else 400,
                         precond=args.precond, mg_down=args.sweeps, mg_up=args.sweeps, mg_bottom=args.sweeps,
                         tile_kc=args.tile_kc)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons, sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(gpu_index)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(dist, values, device=None):
    """Element-wise maximum of per-rank values over all ranks (the job's time is its slowest
    replica's); every rank gets the result."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def whole_job_rate(world, cells, steps, ms_max):
    """Whole-job Mcell-steps/s of `world` replicas that each advance `cells` cells `steps` steps,
    timed by the slowest replica."""
    return world * cells * steps / (ms_max / 1e3) / 1e6


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "of measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "of fallback"


def traffic_ratio():
    """{kernel kind: measured DRAM bytes / algorithmic bytes} of one launch, from the committed ncu
    summaries (profiles/traffic_per_cell.txt)."""
    out = {}
    p = os.path.join(ROOT, "profiles", "traffic_per_cell.txt")
    if os.path.exists(p):
        for line in open(p):
            if line.startswith("#") or not line.strip():
                continue
            k, dram, alg = line.split()[:3]
            out[k] = float(dram) / float(alg)
    return out


def run_arm(args, precision, device, rank, world, dist, profile_on, e2e_on):
    """W warm-up and K timed steps of one case; returns timings and solver statistics."""
    import numpy as np
    import torch

    import impact_b200 as I

    grid, lab, case = build_case(args.size, precision, device)
    sp = step_params(args, precision)
    tuning = None
    for w in range(args.warmup):
        case.step(sp)
        # from rest the first step's Poisson right-hand side is zero: tune on the second one's
        if w == min(1, args.warmup - 1) and not args.no_tune:
            # tile depth and V-cycle sweeps by timing whole Poisson solves of this case (untimed)
            from impact_b200 import autotune
            best, report = autotune.tune(case, sp.poisson, tile_kc=(32, 64), sweeps=((2, 2, 2), (3, 3, 3), (4, 4, 4)))
            sp.poisson = best
            tuning = {"chosen": {"tile_kc": best.tile_kc, "sweeps": [best.mg_down, best.mg_up, best.mg_bottom],
                                 "inner_tol": best.inner_tol_rel if precision == 1 else None},
                      "candidates": report}
    stream = torch.cuda.ExternalStream(case.stream, device=device)
    # pinned host copies of the state the Fortran host owns between time steps -- velocity and
    # pressure (the initial guess of the next Poisson solve); the nonlinear term is not state:
    # the first substep does not read the previous one (mod_rhs.f90, bRK(1) = 0) -- uploaded
    # before and downloaded after every step, as a drop-in call would
    host = {f: torch.empty(grid.shape, dtype=torch.float64, pin_memory=True).numpy()
            for f in ("vel1", "vel2", "vel3", "pre")} if e2e_on else {}
    bytes_in = bytes_out = sum(a.nbytes for a in host.values())
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize(device)
    launches0 = I.launch_count()
    sampler = ClockSampler(device) if rank == 0 and e2e_on else None
    t_dev, t_e2e, its, inner, stats = 0.0, 0.0, [], [], []
    # device-resident timed steps: K steps on the fields in HBM, CUDA events on the case stream
    for _ in range(args.steps):
        e1, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e1.record(stream)
        st = case.step(sp)
        e2.record(stream)
        e2.synchronize()
        t_dev += e1.elapsed_time(e2)
        its.append(list(st.poisson_iterations))
        inner.append(list(st.inner_iterations))
        stats.append(list(st.poisson_status))
    torch.cuda.synchronize(device)
    launches = I.launch_count() - launches0
    for f, a in host.items():  # the host holds the state the device-resident steps reached
        case.download(f, a)
    if dist is not None:
        dist.barrier()
    # end-to-end timed steps: K further steps (both arms advance W + 2K steps), each fed from and
    # drained to pinned host memory.  Inputs go up on a copy-in stream, results come back on a
    # copy-out stream, each field in --copy-chunks element ranges; the upload of a range for the
    # next step waits only for the download of the same range, so the two copy directions run side
    # by side, one range apart.  The step starts once the velocity has landed; the pressure, whose
    # first use follows the explicit part of the first substep, is waited for there
    # (impact_b200_case_defer_pressure), so its upload overlaps that part of the step
    up_s, dn_s = torch.cuda.Stream(device), torch.cuda.Stream(device)
    ranges = [(f, a, j * a.size // args.copy_chunks,
               (j + 1) * a.size // args.copy_chunks - j * a.size // args.copy_chunks)
              for f, a in host.items() for j in range(args.copy_chunks)]
    done = [None] * len(ranges)  # download of each host range enqueued last
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_start.record(up_s)
    for _ in range(args.steps):
        vel_landed = pre_landed = None
        for i, (f, a, first, count) in enumerate(ranges):
            if f == "pre" and vel_landed is None:
                vel_landed = torch.cuda.Event()
                vel_landed.record(up_s)
            if done[i] is not None:
                up_s.wait_event(done[i])
            case.upload_async(f, a, up_s.cuda_stream, first, count)
        if host:
            pre_landed = torch.cuda.Event()
            pre_landed.record(up_s)
            stream.wait_event(vel_landed)
            case.defer_pressure(pre_landed.cuda_event)
        e2 = torch.cuda.Event()
        st = case.step(sp)
        e2.record(stream)
        dn_s.wait_event(e2)
        for i, (f, a, first, count) in enumerate(ranges):
            case.download_async(f, a, dn_s.cuda_stream, first, count)
            done[i] = torch.cuda.Event()
            done[i].record(dn_s)
        e2.synchronize()
    t_end.record(dn_s)
    t_end.synchronize()
    t_e2e = t_start.elapsed_time(t_end)
    torch.cuda.synchronize(device)
    clocks = sampler.stop() if sampler else None
    if dist is not None:
        t_dev, t_e2e = max_over_ranks(dist, [t_dev, t_e2e], f"cuda:{device}")
    out = {"ms_dev": t_dev, "ms_e2e": t_e2e, "iterations": its, "inner_iterations": inner, "status": stats,
           "tuning": tuning,
           "launches": launches, "clocks": clocks, "prof": None, "bytes_in": bytes_in, "bytes_out": bytes_out,
           "dt": st.dtime, "time": st.time}
    fields = None
    if rank == 0:
        fields = {f: case.download(f) for f in ("vel1", "vel2", "vel3", "pre", "nl1", "nl2", "nl3")}
        case.apply("vel1", "res", op=1)  # discrete divergence of the final velocity
        fields["div"] = case.download("res")
    if profile_on:
        # per-kernel device times over K further steps of the same case: the events around every
        # launch (event nodes inside the replayed graphs) slow a step down by about a sixth, so
        # the timed steps above run without them
        torch.cuda.synchronize(device)
        I.profile(True)
        t_prof = 0.0
        for _ in range(args.steps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            case.step(sp)
            b.record(stream)
            b.synchronize()
            t_prof += a.elapsed_time(b)
        torch.cuda.synchronize(device)
        out["prof"] = I.profile_read()
        out["ms_prof"] = t_prof
        I.profile(False)
    case.close()
    del case
    torch.cuda.empty_cache()
    return out, fields, grid, lab


def cpu_baseline(args, fields, lab, fp64_iters):
    """The FP64 CPU oracle on the host cores, on a bounded sample of the same workload: one time
    step with every Poisson solve capped at 2 BiCGstab iterations, plus 2 extra iterations on the
    resident Poisson problem to price one iteration; scaled to a full step with the iteration count
    the FP64 device run needed (same algorithm, same preconditioner)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import oracle as O

    n = args.size
    N = (n + 1, n + 1, 2 * n + 1)
    g = O.Grid(N, (1.0, 1.0, 2.0))
    vel = np.stack([fields["vel1"], fields["vel2"], fields["vel3"]])
    nl = np.stack([fields["nl1"], fields["nl2"], fields["nl3"]])
    pre = fields["pre"].copy()
    st = O.OrcStepState()
    st.timestep = 10
    mg = g.multigrid() if args.precond == 1 else None
    p = O.step_params(Re=500.0, CFL=0.2, dtime_max=1.0, tol_rel=1e-8, max_it=1, n_sweeps=args.n_sweeps, omega=0.8,
                      mg=mg)
    t0 = time.perf_counter()
    g.time_step(p, lab, vel, nl, pre, st)
    t_capped = time.perf_counter() - t0
    used = sum(st.poisson_iterations)
    # price of two more BiCGstab iterations on the current Poisson problem
    b = g.divergence2(vel[0].copy(), vel[1].copy(), vel[2].copy())
    t0 = time.perf_counter()
    if mg is not None:
        r = mg.bicgstab(b, pre.copy(), tol_rel=0.0, max_it=2, omega=0.8, init_yes=False)
    else:
        r = g.bicgstab(b, pre.copy(), tol_rel=0.0, max_it=2, n_sweeps=args.n_sweeps, omega=0.8, init_yes=False)
    t_two = time.perf_counter() - t0
    t_it = t_two / max(1, r.iterations)
    full = t_capped + max(0.0, sum(fp64_iters) - used) * t_it
    cells = n * n * 2 * n
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    return {"value": cells / full / 1e6, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": (f"FP64 oracle, {n}x{n}x{2*n}, same preconditioner: one step with Poisson solves capped at 1 BiCGstab "
                       f"iterations ({t_capped:.1f} s) + 2 iterations ({t_two:.1f} s); scaled to "
                       f"{sum(fp64_iters)} iterations per step (FP64 device run)"),
            "seconds_per_step": full}


def reference_arm(args, rank, world):
    """IMPACT's CPU algorithm (FP64 oracle, all host cores) on bounded samples of the workload."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import oracle as O
    from impact_b200 import geometry as G

    n = args.size
    N = (n + 1, n + 1, 2 * n + 1)
    g = O.Grid(N, (1.0, 1.0, 2.0))
    lab = G.straight_vessel(g, radius_frac=0.25, stenoses=[(1.0, 0.6, 0.125)])
    vel, nl, pre = g.zeros(3), g.zeros(3), g.zeros()
    st = O.OrcStepState()
    # warm-up: develop the flow with capped solves (bounded work), then time capped steps and
    # price BiCGstab iterations; extrapolate to the iteration count a full 1e-8 solve needs
    cap = 1
    mg = g.multigrid() if args.precond == 1 else None
    p = O.step_params(Re=500.0, CFL=0.2, dtime_max=1.0, tol_rel=1e-8, max_it=cap, n_sweeps=args.n_sweeps, omega=0.8,
                      mg=mg)
    for _ in range(min(args.warmup, 2)):
        g.time_step(p, lab, vel, nl, pre, st)
    ref_iters = 3 * _iters_estimate(n, args.precond)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        g.time_step(p, lab, vel, nl, pre, st)
        t_capped = time.perf_counter() - t0
        used = sum(st.poisson_iterations)
        b = g.divergence2(vel[0].copy(), vel[1].copy(), vel[2].copy())
        t0 = time.perf_counter()
        if mg is not None:
            r = mg.bicgstab(b, pre.copy(), tol_rel=0.0, max_it=2, omega=0.8)
        else:
            r = g.bicgstab(b, pre.copy(), tol_rel=0.0, max_it=2, n_sweeps=args.n_sweeps, omega=0.8)
        t_it = (time.perf_counter() - t0) / max(1, r.iterations)
        times.append(t_capped + max(0, ref_iters - used) * t_it)
    cells = n * n * 2 * n
    val = cells * len(times) / sum(times) / 1e6
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload(n),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": (f"each step: one FP64 oracle step with Poisson solves capped at {cap} "
                                        f"BiCGstab iterations + 2 priced iterations, extrapolated to {ref_iters} "
                                        "iterations per step")},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _iters_estimate(n, precond=1):
    """BiCGstab iterations per 1e-8 solve measured on the device for this workload family:
    JOR-4 preconditioner ~1.6 n (64: 110, 128: 210, 256: 405); multigrid V-cycle ~8, independent
    of n."""
    return 8 if precond == 1 else int(round(1.6 * n))


# ---------------------------------------------------------------------------------------------
# batched uneven cases and the serving stream
# ---------------------------------------------------------------------------------------------
def batch_specs(n_cases, seed=7):
    """Uneven vessel cases: n log-uniform in [32, 160] (n x n x 2n cells, rounded to a multiple of 8
    so that the multigrid hierarchy coarsens at least three times), straight cylinder of radius
    U[0.15, 0.3], 0-2 Gaussian stenoses of 30-70 % area reduction at random z (sigma = 0.5 R),
    U0 in U[0.5, 1.5], Re in U[100, 800]."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_cases):
        n = int(max(32, min(160, round(float(np.exp(rng.uniform(np.log(32), np.log(160)))) / 8) * 8)))
        radius = float(rng.uniform(0.15, 0.3))
        sten = [(float(rng.uniform(0.3, 1.7)), float(rng.uniform(0.3, 0.7)), 0.5 * radius)
                for _ in range(int(rng.integers(0, 3)))]
        out.append({"n": n, "radius": radius, "stenoses": sten, "U0": float(rng.uniform(0.5, 1.5)),
                    "Re": float(rng.uniform(100, 800))})
    return out


def _case_params(spec, precision, args):
    import impact_b200 as I
    return I.step_params(Re=spec["Re"], CFL=0.2, dtime_max=1.0, dtime0=1e9, U0=spec["U0"], T_pulse=1.0,
                         level_pressure=1, tol_rel=1e-8, max_it=200 if precision == 0 else 40, omega=0.8,
                         init_yes=0, check_every=args.check_every, inner_tol_rel=args.inner_tol, inner_max_it=400,
                         precond=1, mg_down=args.sweeps, mg_up=args.sweeps, mg_bottom=args.sweeps,
                         tile_kc=args.tile_kc)


def _make_case(spec, precision, device, labels=None):
    import impact_b200 as I
    from impact_b200 import geometry as G
    n = spec["n"]
    g = I.Grid((n + 1, n + 1, 2 * n + 1), (1.0, 1.0, 2.0))
    c = I.Case(g, precision=precision, device=device)
    c.set_labels(labels(g) if labels else G.straight_vessel(g, radius_frac=spec["radius"] / g.L[0],
                                                            stenoses=spec["stenoses"]))
    return c


def batch_bench(args, device, n_cases, steps):
    """48 uneven cases x `steps` mixed-precision steps advanced as one batch, against the same
    cases run one after another in plain FP64 (each case alone, the drop-in's way).  Device time
    from CUDA events on the batch stream / on each case's stream; one untimed warm-up step."""
    import torch

    import impact_b200 as I
    specs = batch_specs(n_cases)
    cells = [s["n"] * s["n"] * 2 * s["n"] for s in specs]
    out = {"workload": f"batched-vessels-{n_cases}", "cases": n_cases, "steps_per_case": steps,
           "cells_total": sum(cells), "n_range": [min(s["n"] for s in specs), max(s["n"] for s in specs)]}
    # mixed, batched
    cases = [_make_case(s, 1, device) for s in specs]
    params = [_case_params(s, 1, args) for s in specs]
    batch = I.Batch(cases)
    batch.step(params, 1)
    stream = torch.cuda.ExternalStream(batch.stream, device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    I.profile(True)
    launches0 = I.launch_count()
    e0.record(stream)
    for _ in range(steps):
        st = batch.step(params, 1)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    prof = I.profile_read()
    I.profile(False)
    out["mixed_batched"] = {"value": round(sum(cells) * steps / (ms / 1e3) / 1e6, 3), "unit": UNIT,
                            "ms_per_step": ms / steps, "launches_per_step": (I.launch_count() - launches0) / steps,
                            "inner_iterations_per_substep_max": max(max(s.inner_iterations) for s in st),
                            "status_ok": all(all(x == 0 for x in s.poisson_status) for s in st),
                            "kernels_ms_per_step": {k: round(v[1] / steps, 2) for k, v in prof.items() if v[0] > 0}}
    batch.close()
    for c in cases:
        c.close()
    del cases
    torch.cuda.empty_cache()
    # plain FP64, one case after another
    total = 0.0
    for s in specs:
        c = _make_case(s, 0, device)
        p = _case_params(s, 0, args)
        c.step(p, 1)
        cs = torch.cuda.ExternalStream(c.stream, device=device)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(cs)
        c.step(p, steps)
        b.record(cs)
        b.synchronize()
        total += a.elapsed_time(b)
        c.close()
    out["fp64_sequential"] = {"value": round(sum(cells) * steps / (total / 1e3) / 1e6, 3), "unit": UNIT,
                              "ms_per_step": total / steps}
    out["batched_mixed_over_sequential_fp64"] = round(out["mixed_batched"]["value"] / out["fp64_sequential"]["value"], 3)
    torch.cuda.empty_cache()
    return out


def serve_bench(args, device, n_req, steps, budget_gb=160.0, rate=20.0):
    """Poisson arrivals (mean `rate` / s) of curved-tube vessel cases, n log-uniform in [64, 256]
    (n x n x 2n, multiple of 8), radius U[0.15, 0.3], 0-2 stenoses; admission by an HBM budget,
    mixed precision at 1e-8, `steps` steps per case; throughput and p50 / p99 completion latency
    on the loop's host clock."""
    import numpy as np
    import torch

    import impact_b200 as I
    from impact_b200 import geometry as G
    from impact_b200 import serve as S
    rng = np.random.default_rng(11)
    arrivals = S.poisson_arrivals(n_req, rate, rng)
    reqs = []
    cells = 0
    for r in range(n_req):
        n = int(max(64, min(256, round(float(np.exp(rng.uniform(np.log(64), np.log(256)))) / 8) * 8)))
        radius = float(rng.uniform(0.15, 0.3))
        sten = [(float(rng.uniform(0.3, 1.7)), float(rng.uniform(0.3, 0.7)), 0.5 * radius)
                for _ in range(int(rng.integers(0, 3)))]
        seed = int(rng.integers(1 << 30))
        spec = {"n": n, "radius": radius, "stenoses": sten, "U0": float(rng.uniform(0.5, 1.5)),
                "Re": float(rng.uniform(100, 800))}

        # the client submits its label mask with the request: built here, before the stream starts
        N = (n + 1, n + 1, 2 * n + 1)
        labels = G.curved_tube(I.Grid(N, (1.0, 1.0, 2.0)), np.random.default_rng(seed), radius, stenoses=sten)
        reqs.append(S.Request(r, N, (1.0, 1.0, 2.0), labels, _case_params(spec, 1, args), steps, float(arrivals[r])))
        cells += n * n * 2 * n
    srv = S.Server(int(budget_gb * 1e9), precision=1, device=device, keep=())
    t0 = time.perf_counter()
    done = srv.run(reqs)
    wall = time.perf_counter() - t0
    torch.cuda.synchronize(device)
    stats = S.summarize(done, wall)
    stats.update({"workload": f"serving-{n_req}-requests", "arrival_rate_per_s": rate, "steps_per_case": steps,
                  "hbm_budget_gb": budget_gb, "peak_cases": srv.peak_cases, "peak_gb": round(srv.peak_bytes / 1e9, 2),
                  "batch_rebuilds": srv.batch_rebuilds, "rounds": srv.rounds,
                  "host_seconds": {k: round(v, 3) for k, v in srv.seconds.items()},
                  "status_ok": all(all(x == 0 for x in d.status) for d in done),
                  "clock": "host wall clock of the request loop (latency = completion - arrival)"})
    return stats


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        reference_arm(args, rank, world)
        return
    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    device = local if world > 1 else 0
    if args.workload == "kernels":
        if rank == 0:
            kernels_main(args, device)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return
    if args.workload != "single":
        extra_main(args, device, rank, world, dist)
        return
    mixed, fields, grid, lab = run_arm(args, 1, device, rank, world, dist, profile_on=not args.no_profile,
                                       e2e_on=True)
    fp64 = None
    if not args.no_fp64:
        fp64, fields64, _, _ = run_arm(args, 0, device, rank, world, dist, profile_on=False, e2e_on=False)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    cells = args.size * args.size * 2 * args.size
    K = args.steps
    value = whole_job_rate(world, cells, K, mixed["ms_dev"])
    e2e = whole_job_rate(world, cells, K, mixed["ms_e2e"])
    peaks, peak_note = measured_peaks()
    prof = mixed["prof"] or {}
    dom = max(prof.items(), key=lambda kv: kv[1][1]) if prof else None
    roof = None
    if dom and dom[1][0] > 0:
        name, (launches, ms, byts) = dom
        per_launch_bytes = byts / launches
        achieved = per_launch_bytes / (ms / launches / 1e3) / 1e9
        ratio = traffic_ratio().get(name)
        roof = {"bound": "hbm", "kernel": name, "achieved": round(achieved, 1), "peak": peaks["hbm_gbs"],
                "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 4), "peak_source": peak_note,
                "traffic": round(ratio * per_launch_bytes) if ratio else None,
                "traffic_source": "ncu dram bytes / algorithmic bytes of one finest-level launch (profiles/), "
                                  "times the algorithmic bytes per launch" if ratio else None,
                "algorithmic_bytes_per_launch": per_launch_bytes,
                "launches": launches, "avg_launch_ms": ms / launches,
                "share_of_step": round(ms / mixed["ms_prof"], 3),
                "measured_over": (f"{K} further steps of the same case after the timed ones, CUDA events around every "
                                  f"launch on the case stream ({mixed['ms_prof'] / K:.1f} ms per step with the events, "
                                  f"{mixed['ms_dev'] / K:.1f} ms without)"),
                "all_kernels": {k: {"launches": v[0], "ms": round(v[1], 2),
                                    "GB/s": round(v[2] / (v[1] / 1e3) / 1e9, 1) if v[1] > 0 else None}
                                for k, v in prof.items() if v[0] > 0}}
    line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": mixed["ms_dev"] / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 inner solve / f64 residual+RHS", "data": "synthetic",
            "config": dict(workload(args.size), parallelism=f"replicas x{world}" if world > 1 else "single GPU",
                           precision="mixed"),
            "e2e": {"value": round(e2e, 3), "unit": UNIT, "h2d_bytes_per_step": mixed["bytes_in"],
                    "d2h_bytes_per_step": mixed["bytes_out"], "ms_per_step": mixed["ms_e2e"] / K,
                    "copies": f"pinned host, vel1-3 + pre, {args.copy_chunks} ranges per field each way on "
                              "copy-in / copy-out streams"},
            "gpu_launches": mixed["launches"], "clocks": mixed["clocks"], "roofline": roof,
            "solver": {"mixed_outer_per_substep": mixed["iterations"], "mixed_inner_per_substep": mixed["inner_iterations"],
                       "status": mixed["status"], "dt": mixed["dt"], "autotune": mixed["tuning"]}}
    if fp64 is not None:
        import numpy as np
        v64 = world * cells * K / (fp64["ms_dev"] / 1e3) / 1e6
        line["fp64"] = {"value": round(v64, 3), "unit": UNIT, "ms_per_step": fp64["ms_dev"] / K,
                        "iterations_per_substep": fp64["iterations"], "status": fp64["status"],
                        "autotune": (fp64["tuning"] or {}).get("chosen")}
        line["mixed_over_fp64"] = round(value / v64, 3)
        if fields is not None and fields64 is not None:
            sl = (slice(4, -4), slice(4, -4), slice(4, -4))  # interior points
            umax = max(float(np.abs(fields64[f][sl]).max()) for f in ("vel1", "vel2", "vel3"))
            du = max(float(np.abs(fields[f][sl] - fields64[f][sl]).max()) for f in ("vel1", "vel2", "vel3"))
            pmax = float(np.abs(fields64["pre"][sl]).max())
            dp = float(np.abs(fields["pre"][sl] - fields64["pre"][sl]).max())
            line["mixed_vs_fp64"] = {
                "after_steps": args.warmup + 2 * K, "velocity_max_abs_err_rel": du / umax if umax else None,
                "pressure_max_abs_err_rel": dp / pmax if pmax else None,
                "divergence_max_abs": {"mixed": float(np.abs(fields["div"][sl]).max()),
                                       "fp64": float(np.abs(fields64["div"][sl]).max())},
                "note": "same workload from rest, same steps; interior points; relative to max|.| of the FP64 run"}
    if not args.no_extra and world == 1:
        line["batch"] = batch_bench(args, device, min(args.cases, 48), args.case_steps or 5)
        line["serve"] = serve_bench(args, device, args.requests, args.case_steps or 10)
    if world == 1 and not args.no_cpu:
        its = fp64["iterations"][-1] if fp64 is not None else [_iters_estimate(args.size, args.precond)] * 3
        try:
            line["cpu_baseline"] = cpu_baseline(args, fields, lab, its)
        except Exception as ex:  # the CPU sample must never hide the device number
            line["cpu_baseline"] = {"value": None, "error": str(ex)[:200]}
    print(json.dumps(line), flush=True)


# kernel micro-benchmark: (name, precision, entry, id, algorithmic bytes per cell at that precision)
# entry "step": impact_b200_case_kernel_bench (FP64 passes of the time step); "engine":
# impact_b200_case_engine_bench on the finest level (FP64, or FP32 = the inner solve of a mixed case)
KERNELS = [("rhs_vel_1", 0, "step", 10, 56), ("rhs_vel_2", 0, "step", 11, 56), ("rhs_vel_3", 0, "step", 12, 56),
           ("interpolate_vel", 0, "step", 13, 48), ("project", 0, "step", 14, 56), ("divergence2", 0, "step", 15, 32)]
ENGINE = [("mg_sweep", 0), ("mg_init", 1), ("mg_residual", 2), ("mg_prolong", 3), ("mg_restrict", 4), ("ax_dot", 5),
          ("ax_dot2", 6), ("x_update", 7), ("p_update", 8), ("r_update", 9), ("vcycle", 10), ("bicgstab_iteration", 11),
          ("mg_pre_smooth", 12), ("mg_post_smooth", 13)]
for _nm, _k in ENGINE:
    KERNELS += [(_nm + "_f64", 0, "engine", _k, None), (_nm + "_f32", 1, "engine", _k, None)]


def kernels_main(args, device):
    """Average device time of every hot kernel (or of the --kernels subset), --iters launches each
    on resident seeded U[-1, 1] fields of the --size grid, CUDA events on the case stream."""
    import numpy as np

    import impact_b200 as I
    want = None if args.kernels == "all" else set(args.kernels.split(","))
    sel = [k for k in KERNELS if want is None or k[0] in want]
    n = args.size
    cells = n * n * 2 * n
    out = {}
    for prec in (0, 1):
        todo = [k for k in sel if k[1] == prec]
        if not todo:
            continue
        grid = I.Grid((n + 1, n + 1, 2 * n + 1), (1.0, 1.0, 2.0))
        case = I.Case(grid, precision=prec, device=device)
        rng = np.random.default_rng(5)
        for f in ("vel1", "vel2", "vel3", "pre", "nl1", "nl2", "nl3", "res"):
            case.upload(f, rng.uniform(-1.0, 1.0, grid.shape))
        if any(k[2] == "step" for k in todo):
            case.kernel_bench(13, 1)  # interpolated velocities for the rhs_vel passes
        sp = I.solver_params(precond=1, omega=0.8, tile_kc=32, mg_down=3, mg_up=3, mg_bottom=3)
        for name, _, entry, kid, bpc in todo:
            if entry == "step":
                ms = case.kernel_bench(kid, args.iters)
                byts = bpc * cells
            else:
                ms, byts = case.engine_bench(kid, args.iters, sp)
            out[name] = {"ms": round(ms, 4), "GB/s": round(byts / (ms / 1e3) / 1e9, 1) if byts else None}
        case.close()
    print(json.dumps({"workload": f"kernels-{n}x{n}x{2 * n}", "cells": cells, "iters": args.iters,
                      "fields": "seeded U[-1, 1]", "kernels": out}), flush=True)


def extra_main(args, device, rank, world, dist):
    """--workload batch | serve: the batched or serving workload as the benchmark line (every rank
    runs its own replica; value = whole-job aggregate)."""
    import torch
    if args.workload == "batch":
        r = batch_bench(args, device, args.cases, args.case_steps or 50)
        v = r["mixed_batched"]["value"]
        ms = r["mixed_batched"]["ms_per_step"]
    else:
        r = serve_bench(args, device, args.requests, args.case_steps or 200)
        v = r["throughput_mcell_steps_s"]
        ms = 1e3 * r["wall_s"]
    if dist is not None:
        t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{device}")
        dist.all_reduce(t, op=dist.ReduceOp.MIN)
        v = float(t[0]) * world
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": METRIC, "value": round(v, 3), "unit": UNIT, "n_gpus": world, "steps": args.case_steps or 0,
            "warmup": 1, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 inner solve / f64 residual+RHS", "data": "synthetic", "config": r}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
