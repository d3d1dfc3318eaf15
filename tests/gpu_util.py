"""Shared helpers of the GPU parity tests (arrays move between numpy
Fortran-ordered arrays and 1-D CUDA tensors in the same element order)."""
import numpy as np


def to_dev(a, dtype=None):
    import torch
    t = torch.from_numpy(np.asarray(a, dtype=np.float64).ravel(order="F").copy())
    if dtype is not None:
        t = t.to(dtype)
    return t.cuda()


def from_dev(t, shape):
    return t.double().cpu().numpy().reshape(shape, order="F")


def nan_dev(shape, dtype=None):
    """Output buffers poisoned with NaN, so unwritten elements show up."""
    import torch
    return torch.full((int(np.prod(shape)),), float("nan"), dtype=dtype or torch.float64, device="cuda")


def rel_err(got, ref):
    """max |got - ref| / max |ref| over the array; NaN must match NaN."""
    got = np.asarray(got)
    ref = np.asarray(ref)
    gn, rn = np.isnan(got), np.isnan(ref)
    if not np.array_equal(gn, rn):
        return float("inf")
    m = ~rn
    if not m.any():
        return 0.0
    den = np.max(np.abs(ref[m]))
    return float(np.max(np.abs(got[m] - ref[m])) / (den if den > 0 else 1.0))
