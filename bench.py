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
    ap.add_argument("--workload", default="single", choices=["single", "batch", "serve", "kernels", "plain",
                                                               "operators"],
                    help="single: the 384 mixed case (default line, with short batch and serve samples); "
                         "batch / serve: the full batched or serving workload as the line; kernels: per-kernel "
                         "micro-benchmark on resident random fields (the small case for profilers); plain: the "
                         "64x64x128 FP64 plain step (10 steps) against the oracle on one and all host cores; "
                         "operators: the 256x256x512 stretched operator microbench, FP64 / FP32 / the reference's "
                         "own kernels, against the oracle")
    ap.add_argument("--kernels", default="all", help="kernels: comma-separated names to run (default all)")
    ap.add_argument("--iters", type=int, default=20, help="kernels: timed launches per kernel")
    ap.add_argument("--no-extra", action="store_true", help="skip the batch and serve samples of the default line")
    ap.add_argument("--no-tune", action="store_true", help="keep --tile-kc and --sweeps (no autotuning)")
    ap.add_argument("--sweeps", type=int, default=3,
                    help="V-cycle sweeps down / up / bottom of the batch and serve cases, and of the single case "
                         "with --no-tune (default: the autotuner's choice on the 384 case)")
    ap.add_argument("--tile-kc", type=int, default=64, help="tile depth of the solver kernels, as --sweeps")
    ap.add_argument("--explicit-fp32", type=int, default=0,
                    help="mixed precision: 1 = rhs_vel as the FP32 pass (FP32 work fields and nonlinear term)")
    ap.add_argument("--copy-chunks", type=int, default=8,
                    help="element ranges per field of the end-to-end copies (download and next upload pipeline)")
    ap.add_argument("--no-profile", action="store_true", help="no per-kernel events in the timed steps (no roofline)")
    ap.add_argument("--bottom-cheb", type=int, default=32,
                    help="batch / serve: Chebyshev steps on the coarsest multigrid level (0: Jacobi "
                         "sweeps, the reference's relax_bottom; the sequential FP64 arm always uses those)")
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
                         tile_kc=args.tile_kc, explicit_fp32=args.explicit_fp32 if precision == 1 else 0)


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
           "tuning": tuning, "sp": sp, "state": (case.state.time, case.state.timestep),
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


def _div_metric(grid, div):
    """[max |div|, max |div weight|] over the unique points of a device-computed divergence field,
    weight = 1 / (sum |cDu1(:,i)| + sum |cDv2(:,j)| + sum |cDw3(:,k)|) (mod_coeffs.f90:2242-2262)."""
    import numpy as np
    s = []
    for a in range(3):
        c = np.asarray(grid.tab["cD"][a]).reshape(grid.N[a] + 1, 6)
        s.append(np.abs(c[1:grid.N[a]]).sum(axis=1))
    w = 1.0 / (s[2][:, None, None] + s[1][None, :, None] + s[0][None, None, :])
    d = np.abs(div[4:-4, 4:-4, 4:-4])
    return [float(d.max()), float((d * w).max())]


def step_from_state(args, precision, device, fields, state, sp):
    """One untimed device step of a fresh case of the workload started from `fields` (velocity,
    pressure) at `state` (time, step count) with the solver parameters `sp`; returns the new
    velocity and pressure (host arrays) and the step's solver statistics."""
    import torch
    _, _, case = build_case(args.size, precision, device)
    for f in ("vel1", "vel2", "vel3", "pre"):
        case.upload(f, fields[f])
    case.state.time, case.state.timestep = state
    st = case.step(sp)
    out = {f: case.download(f) for f in ("vel1", "vel2", "vel3", "pre")}
    stats = {"iterations": list(st.poisson_iterations), "inner_iterations": list(st.inner_iterations),
             "status": list(st.poisson_status), "dt": st.dtime}
    case.close()
    del case
    torch.cuda.empty_cache()
    return out, stats


def _fluid_inner(og, lab):
    """Interior points labelled fluid whose divergence stencil (3 points each way) sees only fluid."""
    import numpy as np
    from impact_b200 import geometry as G
    fl = og.interior(lab) == G.FLUID
    inner = fl.copy()
    for ax in range(3):
        for sh in (-3, -2, -1, 1, 2, 3):
            inner &= np.roll(fl, sh, axis=ax)
    return inner


def oracle_step_leg(args, fields, lab, state, sweeps, dev_next):
    """The FP64 CPU oracle on the host cores: ONE full time step of the workload (every Poisson
    solve to the 1e-8 relative residual, no cap), started from the FP64 device run's state after
    its timed steps.  Its wall time is the CPU baseline (measured, not extrapolated); its result
    is the reference for the device's step from the same state (FP64 and mixed precision):
    velocity and pressure errors and the divergence metric of test_divergence (mod_test.f90:300-345)
    on all points and on the fluid points away from the mask."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np

    import oracle as O

    n = args.size
    N = (n + 1, n + 1, 2 * n + 1)
    og = O.Grid(N, (1.0, 1.0, 2.0))
    vel = np.stack([fields["vel1"], fields["vel2"], fields["vel3"]])
    nl = np.stack([fields["nl1"], fields["nl2"], fields["nl3"]])
    pre = fields["pre"].copy()
    st = O.OrcStepState()
    st.time, st.timestep = state
    mg = og.multigrid() if args.precond == 1 else None
    p = O.step_params(Re=500.0, CFL=0.2, dtime_max=1.0, tol_rel=1e-8, max_it=2000, n_sweeps=args.n_sweeps, omega=0.8,
                      mg=mg, mg_down=sweeps[0], mg_up=sweeps[1], mg_bottom=sweeps[2])
    t0 = time.perf_counter()
    og.time_step(p, lab, vel, nl, pre, st)
    secs = time.perf_counter() - t0
    cells = n * n * 2 * n
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    iters = list(st.poisson_iterations)
    cpu = {"value": cells / secs / 1e6, "unit": UNIT, "cores": cores, "kind": "port",
           "sample": (f"one full FP64 oracle time step of {n}x{n}x{2*n} (same multigrid-preconditioned BiCGstab, "
                      f"sweeps {list(sweeps)}, every Poisson solve to 1e-8, no cap; {iters} iterations) from the FP64 "
                      f"device run's state at step {state[1]}, timed on the host: {secs:.1f} s"),
           "seconds_per_step": secs}
    inner = _fluid_inner(og, lab)
    umax = max(float(np.abs(og.interior(vel[m])).max()) for m in range(3))
    pmax = float(np.abs(og.interior(pre)).max())
    div_all, div_in = og.test_divergence(vel), og.test_divergence(vel, inner)
    par = {"start_step": state[1], "oracle": {"iterations": iters, "dt": st.dtime, "div_max": div_all[0],
                                              "div_weighted_max": div_all[1], "div_fluid_inner_max": div_in[0]}}
    for name, (d, stats) in dev_next.items():
        if d is None:
            continue
        dv = np.stack([d["vel1"], d["vel2"], d["vel3"]])
        g_all, g_in = og.test_divergence(dv), og.test_divergence(dv, inner)
        du = max(float(np.abs(og.interior(dv[m]) - og.interior(vel[m])).max()) for m in range(3))
        dp = float(np.abs(og.interior(d["pre"]) - og.interior(pre)).max())
        par[name] = {"velocity_max_abs_err_rel": du / umax, "pressure_max_abs_err_rel": dp / pmax,
                     "div_max": g_all[0], "div_weighted_max": g_all[1], "div_fluid_inner_max": g_in[0],
                     "div_max_err_rel": abs(g_all[0] - div_all[0]) / div_all[0],
                     "div_weighted_max_err_rel": abs(g_all[1] - div_all[1]) / div_all[1],
                     "iterations": stats["iterations"], "inner_iterations": stats["inner_iterations"],
                     "status": stats["status"], "dt_err_rel": abs(stats["dt"] - st.dtime) / st.dtime}
    par["note"] = ("one step from the same state on the device and in the FP64 oracle; errors relative to max|u| and "
                   "max|p| of the oracle's step; div_* = test_divergence's max |div2(u)| and max |div2(u) weight| over "
                   "all points, and max |div2(u)| over fluid points whose stencil sees only fluid")
    return cpu, par


def reference_arm(args, rank, world):
    """IMPACT's CPU algorithm (the FP64 oracle restatement, all host cores) on the workload.

    A full step of the 384 case takes about a minute on the host, so the timed steps are bounded
    samples priced by one measured full step:
      warm-up: step 1 from rest (its Poisson right-hand sides are zero); step 2 in full (every
               solve to 1e-8, no cap) -- its wall time T_full and iteration count n_full are
               measured; step 3 with every solve capped at one BiCGstab iteration (T_cap), so one
               iteration costs t_it = (T_full - T_cap) / (n_full - 3); further warm-up steps capped.
      timed:   K capped steps, each priced as its own wall time plus (n_full - 3) t_it.
    ms_per_step is that full-step price; sample_ms_per_step the capped steps' own wall time."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from impact_b200 import geometry as G

    n = args.size
    N = (n + 1, n + 1, 2 * n + 1)
    g = O.Grid(N, (1.0, 1.0, 2.0))
    lab = G.straight_vessel(g, radius_frac=0.25, stenoses=[(1.0, 0.6, 0.125)])
    vel, nl, pre = g.zeros(3), g.zeros(3), g.zeros()
    st = O.OrcStepState()
    mg = g.multigrid() if args.precond == 1 else None
    sw = args.sweeps

    def params(cap):
        return O.step_params(Re=500.0, CFL=0.2, dtime_max=1.0, tol_rel=1e-8, max_it=cap, n_sweeps=args.n_sweeps,
                             omega=0.8, mg=mg, mg_down=sw, mg_up=sw, mg_bottom=sw)

    def timed(p):
        t0 = time.perf_counter()
        g.time_step(p, lab, vel, nl, pre, st)
        return time.perf_counter() - t0, list(st.poisson_iterations)

    full_p, cap_p = params(2000), params(1)
    timed(full_p)                      # from rest: zero right-hand sides
    t_full, it_full = timed(full_p)    # one full step, measured
    t_cap, it_cap = timed(cap_p)
    n_full = sum(it_full)
    t_it = max(0.0, (t_full - t_cap) / max(1, n_full - sum(it_cap)))
    for _ in range(max(0, args.warmup - 3)):
        timed(cap_p)
    samples, priced = [], []
    for _ in range(args.steps):
        t, its = timed(cap_p)
        samples.append(t)
        priced.append(t + max(0, n_full - sum(its)) * t_it)
    cells = n * n * 2 * n
    val = cells * len(priced) / sum(priced) / 1e6
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    sample = (f"FP64 oracle, {n}x{n}x{2*n}, multigrid-preconditioned BiCGstab (sweeps {sw}/{sw}/{sw}) to 1e-8: one "
              f"full step measured in warm-up ({t_full:.1f} s, {it_full} iterations, {cells / t_full / 1e6:.3f} "
              f"Mcell-steps/s); each timed step runs the full explicit part with every Poisson solve capped at one "
              f"BiCGstab iteration ({1e3 * sum(samples) / len(samples):.0f} ms on average) and is priced with the "
              f"remaining {n_full} - 3 iterations at the full step's {t_it:.2f} s per iteration")
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * sum(priced) / len(priced),
            "sample_ms_per_step": 1e3 * sum(samples) / len(samples), "full_step_measured_ms": 1e3 * t_full,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload(n),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


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


def _case_params(spec, precision, args, bottom_cheb=None):
    import impact_b200 as I
    return I.step_params(Re=spec["Re"], CFL=0.2, dtime_max=1.0, dtime0=1e9, U0=spec["U0"], T_pulse=1.0,
                         level_pressure=1, tol_rel=1e-8, max_it=200 if precision == 0 else 40, omega=0.8,
                         init_yes=0, check_every=args.check_every, inner_tol_rel=args.inner_tol, inner_max_it=400,
                         precond=1, mg_down=args.sweeps, mg_up=args.sweeps, mg_bottom=args.sweeps,
                         tile_kc=args.tile_kc,
                         bottom_cheb=args.bottom_cheb if bottom_cheb is None else bottom_cheb)


def _make_case(spec, precision, device, labels=None):
    import impact_b200 as I
    from impact_b200 import geometry as G
    n = spec["n"]
    g = I.Grid((n + 1, n + 1, 2 * n + 1), (1.0, 1.0, 2.0))
    c = I.Case(g, precision=precision, device=device)
    c.set_labels(labels(g) if labels else G.straight_vessel(g, radius_frac=spec["radius"] / g.L[0],
                                                            stenoses=spec["stenoses"]))
    return c


def _batch_run(specs, cells, precision, steps, args, device, profile_steps=2):
    """The cases of `specs` advanced `steps` steps as one batch at `precision` after one untimed
    warm-up step: device time from CUDA events on the batch stream, no per-kernel events in the
    timed steps; the per-kernel times come from `profile_steps` further steps."""
    import torch

    import impact_b200 as I
    cases = [_make_case(s, precision, device) for s in specs]
    params = [_case_params(s, precision, args) for s in specs]
    batch = I.Batch(cases)
    batch.step(params, 1)
    stream = torch.cuda.ExternalStream(batch.stream, device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = I.launch_count()
    e0.record(stream)
    for _ in range(steps):
        st = batch.step(params, 1)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    launches = (I.launch_count() - launches0) / steps
    I.profile(True)
    for _ in range(profile_steps):
        batch.step(params, 1)
    prof = I.profile_read()
    I.profile(False)
    out = {"value": round(sum(cells) * steps / (ms / 1e3) / 1e6, 3), "unit": UNIT, "ms_per_step": ms / steps,
           "launches_per_step": launches,
           "iterations_per_substep_max": max(max(s.inner_iterations if precision else s.poisson_iterations) for s in st),
           "status_ok": all(all(x == 0 for x in s.poisson_status) for s in st),
           "kernels_ms_per_step": {k: round(v[1] / profile_steps, 2) for k, v in prof.items() if v[0] > 0},
           "kernels_measured_over": f"{profile_steps} further steps with CUDA events around every launch"}
    batch.close()
    for c in cases:
        c.close()
    del cases
    torch.cuda.empty_cache()
    return out


def batch_bench(args, device, n_cases, steps):
    """48 uneven cases x `steps` steps advanced as one batch in mixed precision and in plain FP64,
    against the same cases run one after another in plain FP64 (each case alone, the drop-in's
    way).  Device time from CUDA events on the batch stream / on each case's stream."""
    import torch

    import impact_b200 as I
    specs = batch_specs(n_cases)
    cells = [s["n"] * s["n"] * 2 * s["n"] for s in specs]
    out = {"workload": f"batched-vessels-{n_cases}", "cases": n_cases, "steps_per_case": steps,
           "cells_total": sum(cells), "n_range": [min(s["n"] for s in specs), max(s["n"] for s in specs)],
           "bottom": (f"{args.bottom_cheb} Chebyshev steps on the coarsest level (batched arms)"
                      if args.bottom_cheb > 0 else f"{args.sweeps} + {args.sweeps} Jacobi sweeps")}
    out["mixed_batched"] = _batch_run(specs, cells, 1, steps, args, device)
    out["fp64_batched"] = _batch_run(specs, cells, 0, steps, args, device)
    # plain FP64, one case after another
    total = 0.0
    for s in specs:
        c = _make_case(s, 0, device)
        p = _case_params(s, 0, args, bottom_cheb=0)
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
    out["batched_mixed_over_batched_fp64"] = round(out["mixed_batched"]["value"] / out["fp64_batched"]["value"], 3)
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
                  "bottom": (f"{args.bottom_cheb} Chebyshev steps on the coarsest level" if args.bottom_cheb > 0
                             else f"{args.sweeps} + {args.sweeps} Jacobi sweeps"),
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
    if args.workload in ("plain", "operators"):
        if rank == 0:
            (plain_main if args.workload == "plain" else operators_main)(args, device)
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
                                for k, v in prof.items() if v[0] > 0},
                "all_kernels_note": ("launches include those whose work a device-side flag skips (BiCGstab "
                                     "iterations queued past convergence in a graph chunk; the first p update of "
                                     "every inner solve, whose pp the outer residual writes), and GB/s counts the "
                                     "algorithmic bytes of every launch, so it overstates the Krylov updates "
                                     "(p_update most)")}
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
                "test_divergence": {"mixed": _div_metric(grid, fields["div"]), "fp64": _div_metric(grid, fields64["div"])},
                "note": "same workload from rest, same steps; interior points; relative to max|.| of the FP64 run; "
                        "test_divergence = [max |div2(u)|, max |div2(u) weight|] over all points (mod_test.f90:300-345), "
                        "after the mask forcing, as the reference prints it at the start of a step"}
    if not args.no_extra and world == 1:
        line["batch"] = batch_bench(args, device, min(args.cases, 48), args.case_steps or 5)
        line["serve"] = serve_bench(args, device, args.requests, args.case_steps or 10)
    if world == 1 and not args.no_cpu and fp64 is not None:
        try:
            sw = [fp64["sp"].poisson.mg_down, fp64["sp"].poisson.mg_up, fp64["sp"].poisson.mg_bottom]
            nxt = {"fp64": step_from_state(args, 0, device, fields64, fp64["state"], fp64["sp"]),
                   "mixed": step_from_state(args, 1, device, fields64, fp64["state"], mixed["sp"])}
            line["cpu_baseline"], line["parity_vs_oracle"] = oracle_step_leg(args, fields64, lab, fp64["state"], sw,
                                                                             nxt)
        except Exception as ex:  # the CPU leg must never hide the device number
            line["cpu_baseline"] = {"value": None, "error": str(ex)[:300]}
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
        sp = I.solver_params(precond=1, omega=0.8, tile_kc=args.tile_kc, mg_down=3, mg_up=3, mg_bottom=3)
        for name, _, entry, kid, bpc in todo:
            if entry == "step":
                ms = case.kernel_bench(kid, args.iters)
                byts = bpc * cells
            else:
                ms, byts = case.engine_bench(kid, args.iters, sp)
            out[name] = {"ms": round(ms, 4), "GB/s": round(byts / (ms / 1e3) / 1e9, 1) if byts else None}
        case.close()
    if want is None or "ibm" in want:
        out["ibm"] = ibm_timing(args, device, n)
    print(json.dumps({"workload": f"kernels-{n}x{n}x{2 * n}", "cells": cells, "iters": args.iters,
                      "fields": "seeded U[-1, 1]", "kernels": out}), flush=True)


def ibm_timing(args, device, n):
    """The diffuse-interface immersed-boundary transfers (interpolate_vel_to_ib and
    spread_force_dens_to_vel_grid, mod_ibm.f90:428-737) on the resident fields of the n x n x 2n
    case: markers on a sphere of radius 0.2 (10^4 and 10^5 of them), hat kernel of reach 2 cells;
    wall time per call over --iters calls after a warm-up, including the markers' host <-> device
    transfers of each call (interpolate: the marker velocities come back; spread: the marker
    forces go up)."""
    import numpy as np
    import torch

    import impact_b200 as I
    grid = I.Grid((n + 1, n + 1, 2 * n + 1), (1.0, 1.0, 2.0))
    case = I.Case(grid, precision=0, device=device)
    rng = np.random.default_rng(9)
    for f in ("vel1", "vel2", "vel3"):
        case.upload(f, rng.uniform(-1.0, 1.0, grid.shape))
    res = {}
    for m in (10_000, 100_000):
        v = rng.normal(size=(m, 3))
        yb = np.array([0.5, 0.5, 1.0]) + 0.2 * v / np.linalg.norm(v, axis=1)[:, None]
        case.set_markers(yb, reach=2.0 / n, delta_type=2)
        fb, vol = rng.uniform(-1.0, 1.0, (m, 3)), np.full(m, 1e-4)
        case.ibm_interpolate()
        case.ibm_spread(fb, vol, into="rhs")
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        for _ in range(args.iters):
            case.ibm_interpolate()
        torch.cuda.synchronize(device)
        t1 = time.perf_counter()
        for _ in range(args.iters):
            case.ibm_spread(fb, vol, into="rhs")
        torch.cuda.synchronize(device)
        t2 = time.perf_counter()
        res[f"markers_{m}"] = {"interpolate_ms": round(1e3 * (t1 - t0) / args.iters, 4),
                               "spread_ms": round(1e3 * (t2 - t1) / args.iters, 4)}
    case.close()
    return res


def plain_main(args, device):
    """The plain IMPACT step: 64 x 64 x 128 cells (periodic box 1 x 1 x 2), straight vessel of radius
    0.25 L1 (label-5 inflow buffer on the first 10 planes, label-9 outlet on the last 10), pulsatile
    plug inflow, Re = 200, dt = 0.2 x the CFL limit, 10 FP64 steps from rest, every Poisson solve
    BiCGstab with the JOR preconditioner (omega = 0.8, 4 sweeps) to a 1e-8 relative residual.
    Device: W warm-up and K timed runs of the 10 steps, each on a fresh case (CUDA events on the
    case stream around the 10 steps).  CPU: the FP64 oracle's 10 steps on all host cores, and a
    bounded single-core sample (steps 2-3: step 1 from rest has no Poisson work).  Parity of the
    device's 10 steps against the all-core oracle run."""
    import numpy as np
    import torch

    import impact_b200 as I
    from impact_b200 import geometry as G
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    N, L, nsteps = (65, 65, 129), (1.0, 1.0, 2.0), 10
    cells = 64 * 64 * 128
    ig, og = I.Grid(N, L), O.Grid(N, L)
    lab = G.straight_vessel(ig, radius_frac=0.25, n_in=10, n_out=10)
    sp = I.step_params(Re=200.0, CFL=0.2, tol_rel=1e-8, n_sweeps=4, omega=0.8, max_it=2000, precond=0)

    def device_run():
        case = I.Case(ig, precision=0, device=device)
        case.set_labels(lab)
        stream = torch.cuda.ExternalStream(case.stream, device=device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        e0.record(stream)
        its = []
        for _ in range(nsteps):
            st = case.step(sp)
            its.append(list(st.poisson_iterations))
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
        out = (ms, its, np.stack([case.download(f) for f in ("vel1", "vel2", "vel3")]), case.download("pre"))
        case.close()
        return out

    for _ in range(args.warmup):
        device_run()
    sampler = ClockSampler(device)
    runs = [device_run() for _ in range(args.steps)]
    clocks = sampler.stop()
    ms = sum(r[0] for r in runs) / len(runs)
    _, dev_its, dvel, dpre = runs[-1]
    # CPU: all cores, the full 10 steps
    cores = O.set_threads(0)
    vel, nl, pre = og.zeros(3), og.zeros(3), og.zeros()
    st = O.OrcStepState()
    op = O.step_params(Re=200.0, CFL=0.2, tol_rel=1e-8, n_sweeps=4, omega=0.8)
    t_all, orc_its = [], []
    for _ in range(nsteps):
        t0 = time.perf_counter()
        og.time_step(op, lab, vel, nl, pre, st)
        t_all.append(time.perf_counter() - t0)
        orc_its.append(list(st.poisson_iterations))
    # CPU: one core, steps 1-3 of the same run (bounded sample)
    O.set_threads(1)
    v1, n1, p1 = og.zeros(3), og.zeros(3), og.zeros()
    s1 = O.OrcStepState()
    t_one = []
    for _ in range(3):
        t0 = time.perf_counter()
        og.time_step(op, lab, v1, n1, p1, s1)
        t_one.append(time.perf_counter() - t0)
    O.set_threads(cores)
    umax = max(float(np.abs(og.interior(vel[m])).max()) for m in range(3))
    du = max(float(np.abs(og.interior(dvel[m]) - og.interior(vel[m])).max()) for m in range(3))
    dp = float(np.abs(og.interior(dpre) - og.interior(pre)).max()) / float(np.abs(og.interior(pre)).max())
    inner = _fluid_inner(og, lab)
    w_all, g_all = og.test_divergence(vel), og.test_divergence(dvel)
    w_in, g_in = og.test_divergence(vel, inner), og.test_divergence(dvel, inner)
    one_ps = sum(t_one[1:]) / 2  # steps 2-3
    all_ps_sampled = sum(t_all[1:3]) / 2
    line = {"metric": METRIC, "value": round(cells * nsteps / (ms / 1e3) / 1e6, 3), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / nsteps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "plain-step-64x64x128", "cells": cells, "box": [1.0, 1.0, 2.0], "radius": 0.25,
                       "Re": 200.0, "steps_per_run": nsteps, "poisson": "BiCGstab + JOR (omega 0.8, 4 sweeps) to 1e-8",
                       "start": "rest", "timed": f"{args.steps} runs of the 10 steps, each on a fresh case",
                       "l2_flush": "none: the whole case (about 0.3 GB) is L2-sized; each run starts from a fresh case"},
            "clocks": clocks,
            "iterations": {"device": dev_its, "oracle": orc_its},
            "cpu_all_cores": {"value": cells * nsteps / sum(t_all) / 1e6, "unit": UNIT, "cores": cores,
                              "kind": "port", "seconds_per_step": [round(t, 3) for t in t_all],
                              "sample": "the FP64 oracle's 10 steps from rest"},
            "cpu_single_core": {"value": cells / one_ps / 1e6, "unit": UNIT, "cores": 1, "kind": "port",
                                "seconds_per_step": [round(t, 3) for t in t_one],
                                "all_cores_same_steps_s": all_ps_sampled,
                                "sample": "steps 2-3 of the 10 on one thread (step 1 from rest has no Poisson work); "
                                          "value = cells / their mean time"},
            "parity_vs_oracle": {"velocity_max_abs_err_rel": du / umax, "pressure_max_abs_err_rel": dp,
                                 "test_divergence": {"oracle": list(w_all), "device": list(g_all)},
                                 "div_fluid_inner_max": {"oracle": w_in[0], "device": g_in[0]},
                                 "after_steps": nsteps}}
    print(json.dumps(line), flush=True)


# Operator microbench: name, FP64 launcher, arguments builder key, algorithmic FP64 bytes per cell
def operators_main(args, device):
    """The operator microbench: 256 x 256 x 512 cells, x and y stretched by x_i = sinh(2 (i/N - 1/2)) /
    sinh 1 (box 2 x 2 x 4), z uniform, i.i.d. U[-1, 1] fields from seeds.  Every operator of the
    reference's launcher FFI in FP64, its _sp FP32 counterpart, and the reference's own CUDA kernel
    (src/*_launcher.cu compiled from the reference tree for sm_100a, FP64) on the same device
    fields: --iters launches each after 3 warm-ups, CUDA events on the launch stream; every field
    exceeds the 126 MB L2 (FP64 270 MB, FP32 135 MB).  The FP64 oracle on all host cores gives
    ns/cell and the values each result is compared with."""
    import ctypes as C

    import numpy as np
    import torch

    import impact_b200 as I
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    N, L, kinds = (257, 257, 513), (2.0, 2.0, 4.0), (1, 1, 0)
    ig, og = I.Grid(N, L, kinds), O.Grid(N, L, kinds)
    cells = 256 * 256 * 512
    nx, ny, nz = (n + 7 for n in N)
    refp = os.path.join(ROOT, "oracle", "_ref", "libref_kernels.so")
    ref = C.CDLL(refp) if os.path.exists(refp) else None

    def dv(a, f32=False):
        return torch.from_numpy(np.ascontiguousarray(a.astype(np.float32) if f32 else a)).cuda(device)

    def tab(name, a, f32):
        return dv(ig.tab[name][a], f32)

    def call(lib, name, spec):
        keep, conv = [], []
        for kind, v in spec:
            if kind == "p":  # a device array: the launchers take double** / float** (by reference)
                o = C.cast(C.c_void_p(int(v)), C.POINTER(C.c_double))
            else:
                o = {"i": C.c_int, "d": C.c_double, "f": C.c_float}[kind](v)
            keep.append(o)
            conv.append(C.byref(o))
        getattr(lib, name)(*conv)

    def timed(lib, name, spec, iters):
        for _ in range(3):
            call(lib, name, spec)
        torch.cuda.synchronize(device)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(iters):
            call(lib, name, spec)
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / iters

    def err(d_out, want):
        got = d_out.cpu().numpy().astype(np.float64)
        return float(np.abs(og.interior(got) - og.interior(want)).max() / np.abs(og.interior(want)).max())

    L64 = I.lib()
    rows = {}
    rng_seed = [2000]

    def field(n=None):
        rng_seed[0] += 1
        a = og.random(rng_seed[0], n=n)
        if n is None:
            og.fill_ghosts(a)
        else:
            for m in range(n):
                og.fill_ghosts(a[m])
        return a

    def run(key, name, build, cpu, bpc, out_init):
        """build(f32, target) -> (spec, d_out); cpu() -> (oracle result, seconds)."""
        want, secs = cpu()
        r = {"bytes_per_cell_fp64": bpc, "cpu_ns_per_cell": round(1e9 * secs / cells, 3)}
        for tag, lib, nm, f32 in (("fp64", L64, name + "_", False), ("fp32", L64, name + "_sp_", True),
                                  ("reference", ref, name + "_", False)):
            if lib is None:
                continue
            spec, d_out = build(f32)
            ms = timed(lib, nm, spec, args.iters)
            b = bpc * cells / (2 if f32 else 1)
            spec, d_out = build(f32)  # fresh output (accumulating operators) for the values
            call(lib, nm, spec)
            torch.cuda.synchronize(device)
            r[tag] = {"ms": round(ms, 4), "GB/s": round(b / (ms / 1e3) / 1e9, 1), "err_vs_oracle": err(d_out, want)}
        if "reference" in r:
            r["fp64_speedup_vs_reference"] = round(r["reference"]["ms"] / r["fp64"]["ms"], 2)
        rows[key] = r

    def cpu_timed(fn):
        t0 = time.perf_counter()
        w = fn()
        return w, time.perf_counter() - t0

    S = lambda f32: "f" if f32 else "d"  # noqa: E731
    phi = field()
    for m in (1, 2, 3):
        def b_grad(f32, m=m):
            d_in, d_out, t = dv(phi, f32), dv(og.zeros(), f32), tab("cG", m - 1, f32)
            return ([("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 6), ("i", N[m - 1] + 1), ("p", d_in.data_ptr()),
                     ("p", t.data_ptr()), ("p", d_out.data_ptr())], _Keep(d_out, d_in, t))
        run(f"gradient_{m}", "gradient_launcher", b_grad, lambda m=m: cpu_timed(lambda: og.gradient(m, phi)), 16, None)
    vel3 = field(3)

    def b_div2(f32):
        d_in, d_out = dv(vel3, f32), dv(og.zeros(), f32)
        c = [tab("cD", a, f32) for a in range(3)]
        return ([("i", nx), ("i", ny), ("i", nz), ("i", 6), ("i", 6), ("i", 6), ("p", d_in.data_ptr()),
                 ("p", d_out.data_ptr())] + [("p", t.data_ptr()) for t in c], _Keep(d_out, d_in, *c))
    run("divergence2", "divergence2_launcher", b_div2,
        lambda: cpu_timed(lambda: og.divergence2(vel3[0], vel3[1], vel3[2])), 32, None)
    u, nl0, pp = field(), field(), field()
    for m in (1, 2, 3):
        names = [("cuu" if a == m - 1 else "cpp") for a in range(3)]

        def b_helm(f32, m=m, names=names):
            d_in, d_out = dv(u, f32), dv(nl0, f32)
            c = [tab(names[a], a, f32) for a in range(3)]
            return ([("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 7), ("i", 7), ("i", 7), (S(f32), 1e-3),
                     ("p", d_in.data_ptr()), ("p", d_out.data_ptr())] + [("p", t.data_ptr()) for t in c],
                    _Keep(d_out, d_in, *c))
        run(f"helmholtz_{m}", "helmholtz_explicit_launcher", b_helm,
            lambda m=m: cpu_timed(lambda: og.helmholtz(m, 1e-3, u, nl0.copy())), 24, None)
    for cid in range(1, 10):
        m, a = (cid - 1) // 3 + 1, (cid - 1) % 3 + 1
        up, dn = ("cNuU", "cNuD") if a == m else ("cNpU", "cNpD")

        def b_up(f32, cid=cid, a=a, up=up, dn=dn):
            d_pp, d_u, d_nl = dv(pp, f32), dv(u, f32), dv(nl0, f32)
            t1, t2 = tab(up, a - 1, f32), tab(dn, a - 1, f32)
            return ([("i", cid), ("i", nx), ("i", ny), ("i", nz), ("i", 7), ("i", N[a - 1] + 1),
                     ("p", d_pp.data_ptr()), ("p", d_u.data_ptr()), ("p", d_nl.data_ptr()), ("p", t1.data_ptr()),
                     ("p", t2.data_ptr())], _Keep(d_nl, d_pp, d_u, t1, t2))
        run(f"upwind_{cid}", "nonlinear_upwind_launcher", b_up,
            lambda cid=cid: cpu_timed(lambda: og.nonlinear_upwind(cid, pp, u, nl0.copy())), 24 if a == 1 else 32, None)
    for m in (1, 2, 3):
        for nm, tb, fn in (("interpolate2_pre_vel", "cIpu", og.interpolate_pre_vel),
                           ("interpolate2_vel_pre", "cIup", og.interpolate_vel_pre)):
            def b_int(f32, m=m, tb=tb):
                d_in, d_out = dv(u, f32), dv(og.zeros(), f32)
                t = tab(tb, m - 1, f32)
                return ([("i", m), ("i", nx), ("i", ny), ("i", nz), ("i", 6), ("i", N[m - 1] + 1),
                         ("p", d_in.data_ptr()), ("p", t.data_ptr()), ("p", d_out.data_ptr())], _Keep(d_out, d_in, t))
            run(f"{nm}_{m}", nm + "_launcher", b_int, lambda m=m, fn=fn: cpu_timed(lambda: fn(m, u)), 16, None)
    bb, rel = field(), field()

    def b_jor(f32):
        d_bb, d_rel, d_out = dv(bb, f32), dv(rel, f32), dv(og.zeros(), f32)
        c = [tab("cdg", a, f32) for a in range(3)]
        return ([("i", 1), ("i", nx), ("i", ny), ("i", nz), ("i", N[0]), ("i", N[1]), ("i", N[2]), ("i", 3),
                 (S(f32), 0.8)] + [("p", t.data_ptr()) for t in c] +
                [("p", d_rel.data_ptr()), ("p", d_bb.data_ptr()), ("p", d_out.data_ptr())], _Keep(d_out, d_bb, d_rel, *c))
    run("jor_sweep", "jacobi_launcher", b_jor, lambda: cpu_timed(lambda: og.jacobi(bb.copy(), rel.copy(), 1, 0.8)), 24,
        None)
    peaks, note = measured_peaks()
    tot = {t: sum(r[t]["ms"] for r in rows.values() if t in r) for t in ("fp64", "fp32", "reference")}
    line = {"workload": "operators-256x256x512-stretched", "cells": cells, "iters": args.iters,
            "grid": "x, y: x_i = sinh(2 (i/N - 1/2)) / sinh 1 (box 2 x 2 x 4), z uniform",
            "fields": "seeded U[-1, 1], ghost layers filled periodically (the reference kernels read them)",
            "cpu_cores": O.set_threads(0), "peak_hbm_gbs": peaks["hbm_gbs"], "peak_source": note,
            "jor_50_sweeps_ms": {t: round(50 * rows["jor_sweep"][t]["ms"], 3) for t in ("fp64", "fp32", "reference")
                                 if t in rows["jor_sweep"]},
            "all_operators_ms": {t: round(v, 3) for t, v in tot.items()},
            "reference_kernels": "oracle/_ref/libref_kernels.so" if ref is not None else "not built",
            "operators": rows}
    print(json.dumps(line), flush=True)


class _Keep:
    """Holds the device tensors of one launch alive; `first` is the output."""

    def __init__(self, first, *rest):
        self.first, self.rest = first, rest

    def cpu(self):
        return self.first.cpu()


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
