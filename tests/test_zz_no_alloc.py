"""The allocation-free inner product (impact_b200_product_scalar_noalloc).

Some callers cannot let the library allocate device memory -- a host code whose GPU memory is
all claimed by its own allocator, or a loop that cannot afford cudaMalloc/cudaFree and the device
synchronisation they can cause.  The no-allocation entry point keeps its scratch in a fixed device
array instead.  Its result must match the FP64 oracle's inner product and the allocating entry
point's (impact_b200_product_scalar) on two calls in a row, through the C ABI, whether this file
runs alone or after the others; it must leave the device's free memory unchanged, and it must
run on the library's current stream, after the launchers queued there.
"""
import numpy as np
import pytest

import oracle as O
import impact_b200 as I
from _util import dev, ptr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [(17, 17, 33), (22, 15, 13)])
def test_noalloc_matches_oracle_and_allocating_entry_point(N):
    og = O.Grid(N)
    a, b = og.random(1), og.random(2)
    d_a, d_b = dev(a), dev(b)
    want = og.dot(a, b)
    tol = 1e-12 * np.sqrt(og.dot(a, a) * og.dot(b, b))
    first = I.product_scalar_noalloc(N, ptr(d_a), ptr(d_b))
    second = I.product_scalar_noalloc(N, ptr(d_a), ptr(d_b))
    assert abs(first - want) <= tol
    assert abs(second - want) <= tol
    assert first == second  # the shared scratch keeps no state from the first call
    assert abs(first - I.product_scalar(N, ptr(d_a), ptr(d_b))) <= tol


def test_noalloc_leaves_device_memory_unchanged():
    """After a warm-up call (which loads the kernels and resolves the array's address), calls on a
    grid size not seen before change the device's free memory by nothing."""
    import torch

    og0 = O.Grid((17, 17, 17))
    w = dev(og0.random(3))
    I.product_scalar_noalloc(og0.N, ptr(w), ptr(w))
    N = (41, 23, 57)
    og = O.Grid(N)
    a, b = og.random(4), og.random(5)
    d_a, d_b = dev(a), dev(b)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    vals = [I.product_scalar_noalloc(N, ptr(d_a), ptr(d_b)) for _ in range(3)]
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert vals[0] == vals[1] == vals[2]
    assert abs(vals[0] - og.dot(a, b)) <= 1e-12 * np.sqrt(og.dot(a, a) * og.dot(b, b))


def test_noalloc_is_ordered_after_launchers_on_a_non_blocking_stream():
    """A caller sets a non-blocking stream, queues axpby_launcher_ on it and calls the inner product
    at once: the inner product sees the launcher's output."""
    import torch

    N = (129, 129, 129)
    og = O.Grid(N)
    x, y = og.random(6), og.random(7)
    d_x, d_y, d_z = dev(x), dev(y), dev(og.zeros())
    torch.cuda.synchronize()
    s = torch.cuda.Stream()  # created non-blocking by torch
    nx, ny, nz = (n + 7 for n in N)
    I.lib().impact_b200_set_stream(s.cuda_stream)
    try:
        I.launchers.call("axpby_launcher_", ("i", nx), ("i", ny), ("i", nz), ("d", 2.0), ("d", -1.0),
                         ("p", ptr(d_x)), ("p", ptr(d_y)), ("p", ptr(d_z)))
        got = I.product_scalar_noalloc(N, ptr(d_z), ptr(d_z))
    finally:
        I.lib().impact_b200_set_stream(None)
    z = og.axpby(2.0, -1.0, x, y, og.zeros())
    want = og.dot(z, z)
    assert abs(got - want) <= 1e-12 * want


def test_noalloc_rejects_grids_beyond_its_scratch():
    d = dev(np.zeros(8))
    with pytest.raises(I.ImpactError, match="16384"):
        I.product_scalar_noalloc((17, 17, 16387), ptr(d), ptr(d))
