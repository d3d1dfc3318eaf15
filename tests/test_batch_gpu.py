"""Batches of uneven blocks in one persistent, graph-captured launch.

Seeded blocks with their own extents, v_size, order (3/5/7), weights
(JS/TENO), MP on/off, drop-in or folded input and FP64 / FP32-bulk storage;
every block's outputs are checked against the oracle (FP64: 1e-12 max-norm
relative; FP32-bulk: against the oracle on the FP32-rounded field, 1e-5),
after two graph launches and again after autotuning the tile shape.
"""
import numpy as np
import pytest

from gpu_util import from_dev, nan_dev, rel_err, teno_check, to_dev

pytestmark = pytest.mark.gpu


def _make_blocks(wsb, oracle_mod, n_blocks=14, seed=2024, lo=8, hi=40, vsizes=(2, 3, 5), uniform=False):
    import torch
    from wenostandalone_b200 import api, fields
    from test_parity_gpu import varying_coefficients
    rng = np.random.default_rng(seed)
    entries, checks = [], []
    for i in range(n_blocks):
        m, n, p = (int(x) - 1 for x in rng.integers(lo, hi + 1, 3))
        nv = int(rng.choice(vsizes))
        order = int(rng.choice([3, 5, 7]))
        scheme = int(rng.choice([0, 3])) if order != 3 else 0
        mp = bool(rng.integers(0, 2))
        folded = bool(rng.integers(0, 2))
        fp32 = bool(i % 4 == 3)
        d = int(rng.integers(0, 3))
        g = wsb.Grid(m, n, p, nv, 6, scheme=scheme)
        vf = fields.smooth_jump_field(m, n, p, nv, 6, seed=100 + i)
        if fp32:
            vf = vf.astype(np.float32).astype(np.float64)
        # face-independent coefficients take the marching items (WENO5 / WENO7
        # JS, WENO5 TENO in FP64); face-varying ones the per-face items
        coefs = (fields.uniform_weno_coefficients(order, g.nc(d)) if uniform
                 else varying_coefficients(order, g.nc(d), seed=200 + i))
        rs = oracle_mod.reshape(np.asfortranarray(vf), m, n, p, 6, d)
        Lr, Rr = oracle_mod.order1_copy(np.asfortranarray(vf), m, n, p, 6, d)
        Lr[:] = np.nan
        Rr[:] = np.nan
        oracle_mod.reconstruct(rs, coefs, order, scheme=scheme, vL=Lr, vR=Rr)
        if mp:
            oracle_mod.preserve_monotonicity(rs, Lr, Rr)
        dt = torch.float32 if fp32 else torch.float64
        if folded:
            v_in = to_dev(vf, dt)
        else:
            v_in = to_dev(rs, dt)
        L, R = nan_dev(g.face_shape(d), dt), nan_dev(g.face_shape(d), dt)
        flags = (wsb.F_MP if mp else 0) | (wsb.F_FOLDED if folded else 0)
        entries.append(dict(grid=g, dir=d, order=order, flags=flags, v_in=v_in,
                            coefs=tuple(to_dev(c) for c in coefs), vL=L, vR=R))
        mg = oracle_mod.teno_margin(rs, coefs, order) if scheme == 3 else None
        checks.append((g, d, scheme, fp32, Lr, Rr, mg))
    return entries, checks


def _check(entries, checks):
    for e, (g, d, scheme, fp32, Lr, Rr, mg) in zip(entries, checks):
        tol = 1e-5 if fp32 else 1e-12
        for got_t, ref in ((e["vL"], Lr), (e["vR"], Rr)):
            got = from_dev(got_t, g.face_shape(d))
            assert np.array_equal(np.isnan(got), np.isnan(ref)), "written faces differ from the sweep's faces"
            if scheme == 3:
                # every entry past tol is a cutoff flip on a borderline face
                teno_check(got, ref, mg, tol, (g, d, e["order"], fp32))
            else:
                assert rel_err(got, ref) <= tol, (g, d, e["order"], fp32)


def _relaunch_and_check(b, entries, checks):
    import torch
    for e in entries:
        e["vL"].fill_(float("nan"))
        e["vR"].fill_(float("nan"))
    for _ in range(2):
        b.launch()
    torch.cuda.synchronize()
    _check(entries, checks)


@pytest.mark.parametrize("coefficients", ["varying", "uniform"])
def test_batch_matches_oracle_per_block(oracle_mod, coefficients):
    """Every way of running a batch -- the persistent kernel (two tile
    shapes), the graph of per-block sweeps (1, 3 and 16 branches) and the
    grouped sweeps (8 to 4096 faces per work item, 1 to 3 branches) --
    then the autotuner's choice."""
    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import api
    entries, checks = _make_blocks(wsb, oracle_mod, uniform=coefficients == "uniform")
    b = api.Batch(entries)
    try:
        _relaunch_and_check(b, entries, checks)          # the default choice
        for cfg in ((0, 128, 8, 8), (0, 64, 32, 8), (1, 128, 8, 1), (1, 128, 8, 3), (1, 128, 8, 16),
                    (2, 128, 8, 1), (2, 128, 64, 3), (2, 128, 4096, 2)):
            b.configure(*cfg)
            q = b.query()
            if cfg[0] == 0:
                assert q == cfg
            elif cfg[0] == 1:
                assert q[0::3] == (1, cfg[3])
            else:
                assert (q[0], q[2], q[3]) == (2, cfg[2], cfg[3])
            _relaunch_and_check(b, entries, checks)
        t, u, ms = b.autotune()
        assert t in (64, 128, 256) and u in (4, 8, 16, 32) and ms > 0
        mode, _, _, nb = b.query()
        assert mode in (0, 1, 2) and 1 <= nb <= 16
        _relaunch_and_check(b, entries, checks)
    finally:
        b.close()


def test_batch_configure_rejects_bad_choices(oracle_mod):
    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import _lib as L, api
    entries, _ = _make_blocks(wsb, oracle_mod, n_blocks=2)
    b = api.Batch(entries)
    try:
        for cfg in ((3, 128, 8, 8), (-1, 128, 8, 8), (0, 96, 8, 8), (0, 128, 0, 8), (1, 128, 8, 0),
                    (1, 128, 8, 17), (2, 128, 7, 4), (2, 128, 4097, 4), (2, 128, 64, 0)):
            with pytest.raises(L.WenoError) as e:
                b.configure(*cfg)
            assert e.value.code == L.ERR_ARG
    finally:
        b.close()


def test_batch_rejects_bad_blocks(oracle_mod):
    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import _lib as L, api
    entries, _ = _make_blocks(wsb, oracle_mod, n_blocks=2)
    entries[1]["order"] = 4
    with pytest.raises(L.WenoError) as e:
        api.Batch(entries)
    assert e.value.code == L.ERR_ARG and "block 1" in L.last_error()


@pytest.mark.parametrize("fp32", [False, True])
def test_grouped_sweeps_mixed_layouts(oracle_mod, fp32):
    """Grouped sweeps whose entries differ in every per-entry property: odd
    and even extents (field rows loaded by TMA or per lane, face rows
    stored by TMA or with plain stores), x / y / z sweeps (row and column
    tiles), folded and drop-in inputs, and 8-face work items, so each warp
    runs many items of different entries in turn.  Against the oracle:
    FP64 1e-12, FP32-bulk 1e-5 on the FP32-rounded field."""
    import torch
    import wenostandalone_b200 as wsb
    from wenostandalone_b200 import api, fields
    rng = np.random.default_rng(77 if fp32 else 76)
    dt = torch.float32 if fp32 else torch.float64
    entries, checks = [], []
    for i in range(18):
        m, n, p = (int(x) - 1 for x in rng.integers(24, 47, 3))
        nv = int(rng.choice([3, 5]))
        order, scheme = [(5, 0), (5, 3), (7, 0), (3, 0)][i % 4]
        folded = i % 3 != 2
        d = i % 3
        g = wsb.Grid(m, n, p, nv, 6, scheme=scheme)
        vf = fields.smooth_jump_field(m, n, p, nv, 6, seed=300 + i)
        if fp32:
            vf = vf.astype(np.float32).astype(np.float64)
        coefs = fields.uniform_weno_coefficients(order, g.nc(d))
        rs = oracle_mod.reshape(np.asfortranarray(vf), m, n, p, 6, d)
        Lr, Rr = oracle_mod.order1_copy(np.asfortranarray(vf), m, n, p, 6, d)
        Lr[:] = np.nan
        Rr[:] = np.nan
        oracle_mod.reconstruct(rs, coefs, order, scheme=scheme, vL=Lr, vR=Rr)
        oracle_mod.preserve_monotonicity(rs, Lr, Rr)
        v_in = to_dev(vf if folded else rs, dt)
        L, R = nan_dev(g.face_shape(d), dt), nan_dev(g.face_shape(d), dt)
        entries.append(dict(grid=g, dir=d, order=order, flags=wsb.F_MP | (wsb.F_FOLDED if folded else 0),
                            v_in=v_in, coefs=tuple(to_dev(c) for c in coefs), vL=L, vR=R))
        mg = oracle_mod.teno_margin(rs, coefs, order) if scheme == 3 else None
        checks.append((g, d, scheme, fp32, Lr, Rr, mg))
    b = api.Batch(entries)
    try:
        for cfg in ((2, 128, 8, 1), (2, 128, 16, 4), (2, 128, 64, 2)):
            b.configure(*cfg)
            _relaunch_and_check(b, entries, checks)
    finally:
        b.close()
