"""The allocation-free inner product (impact_b200_product_scalar_noalloc).

Some callers cannot let the library allocate device memory -- a host code whose GPU memory is
all claimed by its own allocator, or a loop that cannot afford cudaMalloc/cudaFree and the device
synchronisation they can cause.  The no-allocation entry point keeps its scratch in a fixed device
array instead.  Its result must match the allocating entry point's (impact_b200_product_scalar)
on two calls in a row, through the C ABI, whether this file runs alone or after the others.
"""
import numpy as np
import pytest

import oracle as O
import impact_b200 as I
from _util import dev, ptr

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N", [(17, 17, 33), (22, 15, 13)])
def test_noalloc_matches_allocating_entry_point(N):
    og = O.Grid(N)
    a, b = og.random(1), og.random(2)
    d_a, d_b = dev(a), dev(b)
    want = I.product_scalar(N, ptr(d_a), ptr(d_b))
    tol = 1e-12 * np.sqrt(og.dot(a, a) * og.dot(b, b))
    first = I.product_scalar_noalloc(N, ptr(d_a), ptr(d_b))
    second = I.product_scalar_noalloc(N, ptr(d_a), ptr(d_b))
    assert abs(first - want) <= tol
    assert abs(second - want) <= tol
    assert first == second  # the shared scratch keeps no state from the first call


def test_noalloc_rejects_grids_beyond_its_scratch():
    d = dev(np.zeros(8))
    with pytest.raises(I.ImpactError, match="16384"):
        I.product_scalar_noalloc((17, 17, 16387), ptr(d), ptr(d))
