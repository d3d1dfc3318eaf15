"""Input generators: the device (torch) versions evaluate the same formulas
as the numpy ones (checked here on the CPU device)."""
import numpy as np


def test_sinusoid_shock_dev_matches_numpy():
    from wenostandalone_b200 import fields as F
    for shock in (False, True):
        a = F.sinusoid_shock_field(7, 5, 6, 3, 6, seed=3, shock=shock).ravel(order="F")
        b = F.sinusoid_shock_field_dev(7, 5, 6, 3, 6, seed=3, shock=shock, device="cpu").numpy()
        assert np.abs(a - b).max() <= 1e-13


def test_smooth_jump_dev_matches_numpy_up_to_noise():
    from wenostandalone_b200 import fields as F
    a = F.smooth_jump_field(7, 5, 6, 3, 6, seed=3, noise=1e-3).ravel(order="F")
    b = F.smooth_jump_field_dev(7, 5, 6, 3, 6, seed=3, noise=1e-3, device="cpu").numpy()
    assert np.abs(a - b).max() <= 2e-3 + 1e-13
    c = F.smooth_jump_field_dev(7, 5, 6, 3, 6, seed=3, noise=0.0, device="cpu").numpy()
    d = F.smooth_jump_field(7, 5, 6, 3, 6, seed=3, noise=0.0).ravel(order="F")
    assert np.abs(c - d).max() <= 1e-13
