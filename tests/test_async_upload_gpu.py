"""weno_sb_upload_async: v_vf crosses PCIe one variable at a time while the
folded sweeps of the variables already there run.  The results equal those
of the synchronous upload bit for bit (a face's arithmetic does not depend
on how the sweep is cut into launches), for face-independent and per-face
coefficients and back-to-back uploads of different fields; every other
handle call waits for the copy; FP32 handles take the synchronous path."""
import numpy as np
import pytest

from gpu_util import rel_err

pytestmark = pytest.mark.gpu


def _run(h, L, field, asynchronous, dirs=(0, 1, 2), flags=None, reshape=False):
    import torch
    import wenostandalone_b200 as wsb
    fl = (wsb.F_MP | wsb.F_FOLDED) if flags is None else flags
    if asynchronous:
        src = torch.from_numpy(np.asfortranarray(field).ravel(order="F").copy()).pin_memory()
        h.upload_async(L.A_V_VF, src)
    else:
        h.upload(L.A_V_VF, field)
    for d in dirs:
        if reshape:
            h.s_initialize_weno(d)
        h.weno(d, 5, fl)
    out = [(h.download(L.A_VL(d)), h.download(L.A_VR(d))) for d in dirs]
    sums = [h.checksum(L.A_VL(d)) + h.checksum(L.A_VR(d)) for d in dirs]
    return out, sums


@pytest.mark.parametrize("coefs", ["uniform", "varying"])
def test_async_upload_matches_synchronous(oracle_mod, coefs):
    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import _lib as L, fields
    from test_parity_gpu import varying_coefficients
    m, n, p, nv = 47, 31, 23, 4
    g = wsb.Grid(m, n, p, nv, 6)
    f1 = fields.smooth_jump_field(m, n, p, nv, 6, seed=31)
    f2 = fields.smooth_jump_field(m, n, p, nv, 6, seed=32)

    def coef(d):
        return (fields.uniform_weno_coefficients(5, g.nc(d)) if coefs == "uniform"
                else varying_coefficients(5, g.nc(d), seed=40 + d))
    with wsb.Harness(g) as h:
        for d in range(3):
            h.upload_coefficients(d, coef(d))
        ref1, s1 = _run(h, L, f1, False)
        ref2, s2 = _run(h, L, f2, False)
        for rnd in range(2):          # back to back, alternating fields
            got1, g1 = _run(h, L, f1, True)
            got2, g2 = _run(h, L, f2, True)
            for (a, b), (c, e) in zip(got1 + got2, ref1 + ref2):
                assert np.array_equal(a, c) and np.array_equal(b, e), rnd
            assert g1 == s1 and g2 == s2
        # and against the oracle
        for d in range(3):
            rs = oracle_mod.reshape(f2, m, n, p, 6, d)
            Lr, Rr = oracle_mod.order1_copy(f2, m, n, p, 6, d)
            oracle_mod.reconstruct(rs, coef(d), 5, vL=Lr, vR=Rr)
            oracle_mod.preserve_monotonicity(rs, Lr, Rr)
            core = slice(3, g.extents(d)[0] - 3)
            assert rel_err(got2[d][0][core], Lr[core]) <= 1e-12
            assert rel_err(got2[d][1][core], Rr[core]) <= 1e-12


def test_other_calls_wait_for_the_copy(oracle_mod):
    """After upload_async: the download of v_vf, the reshape with the
    non-folded sweep and the order-1 copy all see the new field."""
    import torch
    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import _lib as L, fields
    m, nv = 31, 3
    g = wsb.Grid(m, m, m, nv, 6)
    f0 = fields.smooth_jump_field(m, m, m, nv, 6, seed=1)
    f1 = fields.smooth_jump_field(m, m, m, nv, 6, seed=2)
    with wsb.Harness(g) as h:
        for d in range(3):
            h.upload_coefficients(d, fields.uniform_weno_coefficients(5, g.nc(d)))
        src = torch.from_numpy(f1.ravel(order="F").copy()).pin_memory()
        h.upload(L.A_V_VF, f0)
        h.upload_async(L.A_V_VF, src)
        assert np.array_equal(h.download(L.A_V_VF), f1)
        h.upload(L.A_V_VF, f0)
        h.upload_async(L.A_V_VF, src)
        h.s_initialize_weno(1)                         # reshape, then the non-folded sweep
        h.weno(1, 5, wsb.F_MP)
        rs = oracle_mod.reshape(f1, m, m, m, 6, 1)
        assert np.array_equal(h.download(L.A_RS(1)), rs)
        Lr, Rr = oracle_mod.reconstruct(rs, fields.uniform_weno_coefficients(5, g.nc(1)), 5)
        oracle_mod.preserve_monotonicity(rs, Lr, Rr)
        core = slice(3, g.extents(1)[0] - 3)
        assert rel_err(h.download(L.A_VL(1))[core], Lr[core]) <= 1e-12
        h.upload(L.A_V_VF, f0)
        h.upload_async(L.A_V_VF, src)
        h.s_order1_copy(2)
        Lc, _ = oracle_mod.order1_copy(f1, m, m, m, 6, 2)
        assert np.array_equal(h.download(L.A_VL(2)), Lc)


def test_fp32_handle_takes_the_synchronous_upload():
    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import _lib as L, fields
    m, nv = 23, 2
    g = wsb.Grid(m, m, m, nv, 6)
    f = fields.smooth_jump_field(m, m, m, nv, 6, seed=5)
    with wsb.Harness(g, precision=L.FP32) as h:
        for d in range(3):
            h.upload_coefficients(d, fields.uniform_weno_coefficients(5, g.nc(d)))
        # (FP32 handles sweep the reshaped FP32 copies: the folded form
        # reads the FP64 v_vf)
        ref, s_ref = _run(h, L, f, False, flags=wsb.F_MP, reshape=True)
        got, s_got = _run(h, L, f, True, flags=wsb.F_MP, reshape=True)
        for (a, b), (c, e) in zip(got, ref):
            assert np.array_equal(a, c) and np.array_equal(b, e)
        assert s_got == s_ref
