"""Restart files of a case: the state the time loop carries from step to step -- velocity,
pressure (the next Poisson solve's initial guess), time and step count -- taken with
Case.snapshot and written as a numpy .npz file, and loaded back into a case of the same grid.
The reference writes velX/Y/Z_restart### and pre_restart### as HDF5 (write_restart /
read_restart, mod_inout.f90:326-371); no HDF5 library is in this image, so the file is .npz with
the fields in the reference's padded layout.  The nonlinear term is not state: the first RK
substep does not read the previous one (bRK(1) = 0, mod_rhs.f90), so a case continued from a
restart file takes the same steps bit for bit.  A CT case driven by the analytic Windkessel
branches (ingest.AnalyticWindkessel) also stores their end-systolic pressures, as the reference's
restart files carry p_end_systole_in / _out / _out_2 (mod_inout.f90:468-470, 622-624).
"""
from __future__ import annotations

import numpy as np

STATE = ("vel1", "vel2", "vel3", "pre")


def save(case, path, windkessel=None):
    """Snapshot the case's state at this point of its work and write it to `path`; windkessel:
    an ingest.AnalyticWindkessel whose end-systolic pressures are stored too."""
    out = [np.empty(case.grid.shape, dtype=np.float64) for _ in STATE]
    case.snapshot(STATE, out)
    case.synchronize()
    extra = {}
    if windkessel is not None:
        extra["end_systole"] = np.array([windkessel.end_systole[b] for b in (1, 2, 3)])
    np.savez(path, **{f: a for f, a in zip(STATE, out)}, time=case.state.time, timestep=case.state.timestep,
             N=np.array(case.grid.N), L=np.array(case.grid.L), kinds=np.array(case.grid.kinds), **extra)


def load(case, path, windkessel=None):
    """Upload the state stored in `path` into the case (same grid) and set its time and step
    count; windkessel: an ingest.AnalyticWindkessel that takes back the stored end-systolic
    pressures (an error if the file holds none)."""
    d = np.load(path)
    if tuple(int(n) for n in d["N"]) != tuple(case.grid.N):
        raise ValueError(f"{path}: grid {tuple(d['N'])} differs from the case's {case.grid.N}")
    if windkessel is not None and "end_systole" not in d:
        raise ValueError(f"{path}: no Windkessel state stored")
    for f in STATE:
        case.upload(f, np.ascontiguousarray(d[f]))
    case.state.time = float(d["time"])
    case.state.timestep = int(d["timestep"])
    if windkessel is not None:
        windkessel.end_systole = {b: float(v) for b, v in zip((1, 2, 3), d["end_systole"])}
