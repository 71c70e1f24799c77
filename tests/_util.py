"""Shared helpers of the test-suite: device buffers through torch, comparison metrics."""
import numpy as np


def dev(a):
    """numpy float64 / uint8 array -> CUDA tensor with the same bytes (contiguous)."""
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    import torch
    torch.cuda.synchronize()
    return t.cpu().numpy()


def ptr(t):
    return t.data_ptr()


def rel_err(got, want):
    """max |got - want| / max |want| over the arrays (interior views expected)."""
    d = np.abs(np.asarray(got, dtype=np.float64) - np.asarray(want, dtype=np.float64)).max()
    s = np.abs(want).max()
    return d / s if s > 0 else d
