"""Pin the CPU oracle to the reference's own published checksums, and check
it on known-answer cases.  CPU only."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


def reference_checksums():
    out = {}
    with open(os.path.join(HERE, "golden", "reference_checksums.txt")) as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            case, label, val = line.split()
            out.setdefault(case, {})[label] = float(val)
    return out


def rel(a, e):
    return abs(a - e) / max(abs(e), 1e-300)


def test_oracle_reproduces_weno5_golden(oracle_mod):
    """tests/golden/weno5.txt of the reference: 200^3 x 8, WENO5-JS, scope=full."""
    exp = reference_checksums()["weno5_full"]
    X, Y, Z, T = oracle_mod.harness_run(199, 199, 199, 8, 6)
    for lab, val in zip("XYZT", (X, Y, Z, T)):
        assert rel(val, exp[lab]) <= 1e-10, (lab, val, exp[lab])
        # the survey's restatement matched every printed digit
        assert f"{val:.10E}" == f"{exp[lab]:.10E}"


def test_oracle_reproduces_x_only_run(oracle_mod):
    """results/amd_mp_roof_ex/log.txt:37-40: WENO5 in x only, y/z = order-1 copies."""
    exp = reference_checksums()["weno5_x_only"]
    o = oracle_mod
    m = n = p = 199
    nv, buff = 8, 6
    vf = o.fill_input_field(m, n, p, nv, buff)
    sums = []
    for d, off in enumerate((0.03, 0.05, 0.07)):
        vL, vR = o.order1_copy(vf, m, n, p, buff, d)
        if d == 0:
            rs = o.reshape(vf, m, n, p, buff, d)
            coefs = o.fill_coefficients(rs.shape[0] - 12, off)
            o.reconstruct(rs, coefs, 5, vL=vL, vR=vR)
        sums.append(o.checksum(vL) + o.checksum(vR))
    sums.append(sum(sums))
    for lab, val in zip("XYZT", sums):
        assert rel(val, exp[lab]) <= 1e-10, (lab, val, exp[lab])


def test_numpy_field_matches_oracle_fill(oracle_mod):
    from wenostandalone_b200 import fields
    a = fields.harness_field(9, 7, 5, 3, 6)
    b = oracle_mod.fill_input_field(9, 7, 5, 3, 6)
    assert a.shape == b.shape
    assert np.max(np.abs(a - b)) <= 1e-14


def test_numpy_coefficients_match_oracle(oracle_mod):
    from wenostandalone_b200 import fields
    for off in (0.03, 0.05, 0.07):
        A = fields.harness_coefficients(11, off)
        B = oracle_mod.fill_coefficients(11, off)
        for x, y in zip(A, B):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("order", [3, 5, 7])
def test_constant_field_is_reproduced(oracle_mod, order):
    """beta = eps everywhere, omega = d/sum(d): every candidate equals the constant."""
    from wenostandalone_b200 import fields
    rs = np.full((13 + 6, 4, 3, 2), 2.5, order="F")
    coefs = fields.uniform_weno_coefficients(order, 13 - 6)
    vL, vR = oracle_mod.reconstruct(rs, coefs, order)
    lo = 0 if order == 3 else 3
    hi = 13 if order == 3 else 10
    assert np.allclose(vL[lo:hi], 2.5, rtol=0, atol=1e-15)
    assert np.allclose(vR[lo:hi], 2.5, rtol=0, atol=1e-15)


@pytest.mark.parametrize("order", [3, 5, 7])
def test_linear_field_uniform_coefficients(oracle_mod, order):
    """Uniform-grid coefficients reproduce a linear profile exactly:
    vL = v_j - s/2 (left face), vR = v_j + s/2 (right face)."""
    from wenostandalone_b200 import fields
    ns = 20
    J = np.arange(ns + 6, dtype=float)
    rs = np.empty((ns + 6, 2, 2, 1), order="F")
    rs[:] = (0.3 * J + 1.0)[:, None, None, None]
    coefs = fields.uniform_weno_coefficients(order, ns - 6)
    vL, vR = oracle_mod.reconstruct(rs, coefs, order)
    o = np.arange(3, ns - 3)
    vj = 0.3 * (o + 3) + 1.0
    np.testing.assert_allclose(vL[3:ns - 3, 0, 0, 0], vj - 0.15, rtol=0, atol=1e-13)
    np.testing.assert_allclose(vR[3:ns - 3, 0, 0, 0], vj + 0.15, rtol=0, atol=1e-13)


def test_mp_leaves_monotone_weno_states(oracle_mod):
    """On a monotone linear profile the WENO5 states lie inside the MP bounds."""
    from wenostandalone_b200 import fields
    ns = 16
    J = np.arange(ns + 6, dtype=float)
    rs = np.empty((ns + 6, 1, 1, 1), order="F")
    rs[:, 0, 0, 0] = 0.7 * J - 2.0
    coefs = fields.uniform_weno_coefficients(5, ns - 6)
    vL, vR = oracle_mod.reconstruct(rs, coefs, 5)
    L0, R0 = vL.copy(), vR.copy()
    oracle_mod.preserve_monotonicity(rs, vL, vR)
    np.testing.assert_allclose(vL, L0, rtol=0, atol=1e-14)
    np.testing.assert_allclose(vR, R0, rtol=0, atol=1e-14)


def test_mp_clips_overshoot(oracle_mod):
    """A planted overshoot at a step is clipped back into [min, max] of the data."""
    ns = 16
    rs = np.zeros((ns + 6, 1, 1, 1), order="F")
    rs[11:, 0, 0, 0] = 1.0
    vL = np.full((ns, 1, 1, 1), 1.5, order="F")
    vR = np.full((ns, 1, 1, 1), -0.5, order="F")
    oracle_mod.preserve_monotonicity(rs, vL, vR)
    core = slice(3, ns - 3)
    assert vL[core].max() <= 1.0 and vR[core].min() >= 0.0


def test_weno3_teno_has_no_branch(oracle_mod):
    """The reference's WENO3 has no TENO branch: alpha stays 0 -> NaN."""
    from wenostandalone_b200 import fields
    rs = np.random.default_rng(0).random((19, 2, 2, 1)).copy(order="F")
    vL, vR = oracle_mod.reconstruct(rs, fields.uniform_weno_coefficients(3, 7), 3,
                                    scheme=oracle_mod.TENO)
    assert np.isnan(vL).all() and np.isnan(vR).all()
