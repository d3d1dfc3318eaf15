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


# A TENO cutoff decision (omega_q < CT) can differ between two correct
# implementations only on a face whose omega_q lies within rounding of CT.
TENO_BAND = 1e-10


def teno_check(got, ref, margin, tol, what=""):
    """TENO outputs against the oracle: NaN exactly where the oracle has NaN,
    and every entry off by more than tol (relative to max |ref|) on a face
    whose cutoff margin min_q |omega_q - CT| / CT (oracle.teno_margin) is at
    most TENO_BAND.  Returns the number of such cutoff flips."""
    got = np.asarray(got)
    ref = np.asarray(ref)
    assert np.array_equal(np.isnan(got), np.isnan(ref)), f"NaN pattern differs {what}"
    ok = ~np.isnan(ref)
    if not ok.any():
        return 0
    den = max(float(np.max(np.abs(ref[ok]))), 1e-300)
    bad = np.zeros(ref.shape, dtype=bool)
    bad[ok] = np.abs(got[ok] - ref[ok]) / den > tol
    nbad = int(bad.sum())
    if nbad:
        assert margin is not None, f"{nbad} entries past {tol} and no cutoff margin to excuse them {what}"
        far = bad & ~(np.asarray(margin) <= TENO_BAND)
        assert not far.any(), (f"{int(far.sum())} of {nbad} mismatches are not cutoff flips {what}; "
                               f"worst error {float(np.max(np.abs(got[far] - ref[far])) / den):.3e}")
    return nbad
