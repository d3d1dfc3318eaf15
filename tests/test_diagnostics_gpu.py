"""Device-side diagnostics through the C ABI: the Newton reciprocal used by
the JS normalisation against IEEE division, and the bounded mbarrier wait
of the pipelined sweeps (it must expire into WENO_SB_ERR_TIMEOUT, never hang).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ulp_dist(a, b):
    ia = a.view(np.int64)
    ib = b.view(np.int64)
    return np.abs(ia - ib)


def test_newton_reciprocal_within_one_ulp():
    import torch
    from wenostandalone_b200 import _lib as L
    rng = np.random.default_rng(7)
    x = np.concatenate([
        10.0 ** rng.uniform(-149, 149, 200000),      # the range the sweeps use
        rng.uniform(0.5, 2.0, 50000),
        np.array([1.0, 2.0, 0.5, 3.0, 1e-150, 1e150, np.nextafter(1.0, 2.0)]),
    ])
    dx = torch.from_numpy(x).cuda()
    fast = torch.empty_like(dx)
    ieee = torch.empty_like(dx)
    L.check(L.lib().weno_sb_selftest_rcp(dx.data_ptr(), fast.data_ptr(), ieee.data_ptr(), dx.numel(), None))
    torch.cuda.synchronize()
    d = _ulp_dist(fast.cpu().numpy(), ieee.cpu().numpy())
    assert d.max() <= 1, d.max()


def test_bounded_wait_expires_into_timeout_status():
    import torch
    from wenostandalone_b200 import _lib as L
    lib = L.lib()
    rc = lib.weno_sb_selftest_timeout(1_000_000, None)   # ~0.5 ms of SM clock
    assert rc == L.ERR_TIMEOUT, (rc, L.last_error())
    assert "timeout" in L.last_error()
    # the flag is cleared once reported, and the context is still usable
    assert lib.weno_sb_check_device(None) == L.OK
    t = torch.arange(10, dtype=torch.float64, device="cuda")
    assert float(t.sum()) == 45.0
