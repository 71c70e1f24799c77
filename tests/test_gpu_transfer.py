"""Asynchronous field transfers (impact_b200_case_upload_async / _download_async): copies of whole
fields or element ranges enqueued on caller streams, ordered against the case stream by events,
give the same bytes as the synchronous upload / download, and a time step fed and drained that
way (in ranges, the pressure waited for only where the step first reads it, as the benchmark's
end-to-end loop does) equals one fed synchronously."""
import numpy as np
import pytest
import torch

import impact_b200 as I
from impact_b200 import geometry as G

pytestmark = pytest.mark.gpu


def _pinned(shape):
    return torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()


def test_async_copies_equal_synchronous():
    g = I.Grid((33, 25, 17), (1.0, 1.0, 1.0))
    c = I.Case(g)
    rng = np.random.default_rng(3)
    src = _pinned(g.shape)
    src[...] = rng.uniform(-1.0, 1.0, g.shape)
    up = torch.cuda.Stream()
    c.upload_async("pre", src, up.cuda_stream)
    up.synchronize()
    assert np.array_equal(c.download("pre"), src)
    dst = _pinned(g.shape)
    dst[...] = 0.0
    dn = torch.cuda.Stream()
    c.download_async("pre", dst, dn.cuda_stream)
    dn.synchronize()
    assert np.array_equal(dst, src)
    # element ranges: the halves of the field moved separately, last range ragged
    n = src.size
    part = _pinned(g.shape)
    part[...] = 0.0
    for first, count in ((0, n // 3), (n // 3, n - n // 3)):
        c.download_async("pre", part, dn.cuda_stream, first, count)
    dn.synchronize()
    assert np.array_equal(part, src)
    half = _pinned(g.shape)
    half[...] = 7.0
    c.upload_async("pre", half, up.cuda_stream, 5, 11)
    up.synchronize()
    want = src.copy().reshape(-1)
    want[5:16] = 7.0
    assert np.array_equal(c.download("pre").reshape(-1), want)
    with pytest.raises(ValueError):
        c.upload_async("pre", np.zeros((3, 3, 3)), up.cuda_stream)
    with pytest.raises(ValueError):
        c.download_async("pre", dst, dn.cuda_stream, n - 4, 5)
    c.close()


def test_step_with_async_transfers_equals_synchronous():
    g = I.Grid((33, 33, 65), (1.0, 1.0, 2.0))
    lab = G.straight_vessel(g)
    p = I.step_params(Re=300.0, tol_rel=1e-8, omega=0.8, precond=1, max_it=200)
    ref, c = I.Case(g), I.Case(g)
    for k in (ref, c):
        k.set_labels(lab)
        k.step(p, 2)
    fields = ("vel1", "vel2", "vel3", "pre")
    host = {f: _pinned(g.shape) for f in fields}
    for f in fields:
        c.download(f, host[f])
    up, dn = torch.cuda.Stream(), torch.cuda.Stream()
    comp = torch.cuda.ExternalStream(c.stream)
    n = host["pre"].size
    cuts = [0, n // 4, n // 2, n]
    for f in fields:
        if f == "pre":  # the step starts once the velocity has landed and waits for the pressure
            ev = torch.cuda.Event()  # only where it first reads it (impact_b200_case_defer_pressure)
            ev.record(up)
            comp.wait_event(ev)
        for a, b in zip(cuts, cuts[1:]):
            c.upload_async(f, host[f], up.cuda_stream, a, b - a)
    ev_pre = torch.cuda.Event()
    ev_pre.record(up)
    c.defer_pressure(ev_pre.cuda_event)
    c.step(p, 1)
    ev2 = torch.cuda.Event()
    ev2.record(comp)
    dn.wait_event(ev2)
    for f in fields:
        for a, b in zip(cuts, cuts[1:]):
            c.download_async(f, host[f], dn.cuda_stream, a, b - a)
    dn.synchronize()
    ref.step(p, 1)
    for f in fields:
        assert np.array_equal(host[f], ref.download(f)), f
    ref.close()
    c.close()
