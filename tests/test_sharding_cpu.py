"""Multi-rank host logic on CPU with the gloo backend (world_size 2 and 3):
the z-slab ghost exchange reproduces the undecomposed field, and the z sweep
on every slab then equals the undecomposed sweep bit for bit."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, m, n, p, nv, buff, q):
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import torch.distributed as dist
    import oracle
    from wenostandalone_b200 import fields, sharding
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        glob = fields.smooth_jump_field(m, n, p, nv, buff, seed=11)
        E1, E2, E3 = glob.shape[:3]
        G = sharding.ghost_planes(buff)
        z0, nz = sharding.slab_bounds(p, world, rank)
        # local slab: planes z0-G .. z0+nz+G-1 in global interior-cell coordinates,
        # i.e. global array planes z0 .. z0+nz+2G-1 (the array starts G planes below cell 0)
        loc = np.array(glob[:, :, z0:z0 + nz + 2 * G, :], order="F")
        # internal ghosts start as garbage; physical-boundary ghosts keep the global data
        if rank > 0:
            loc[:, :, :G, :] = -777.0
        if rank < world - 1:
            loc[:, :, nz + G:, :] = -777.0
        t = torch.from_numpy(loc.ravel(order="F").copy())
        sharding.exchange_z_ghosts(t, E1, E2, nz, nv, buff)
        got = t.numpy().reshape(loc.shape, order="F")
        ok_field = np.array_equal(got, glob[:, :, z0:z0 + nz + 2 * G, :])
        # z sweep (WENO5-JS + MP) on the slab vs on the global block
        pl = nz - 1  # local "p_cells"
        rs_loc = oracle.reshape(got, m, n, pl, buff, 2)
        coefs = fields.uniform_weno_coefficients(5, rs_loc.shape[0] - 12)
        Ll, Rl = oracle.reconstruct(rs_loc, coefs, 5)
        oracle.preserve_monotonicity(rs_loc, Ll, Rl)
        rs_g = oracle.reshape(glob, m, n, p, buff, 2)
        Lg, Rg = oracle.reconstruct(rs_g, fields.uniform_weno_coefficients(5, rs_g.shape[0] - 12), 5)
        oracle.preserve_monotonicity(rs_g, Lg, Rg)
        # local face o (core 3..ns_l-4) is global face o + z0
        ns_l = Ll.shape[0]
        sl = slice(3, ns_l - 3)
        ok_sweep = (np.array_equal(Ll[sl], Lg[3 + z0:ns_l - 3 + z0]) and
                    np.array_equal(Rl[sl], Rg[3 + z0:ns_l - 3 + z0]))
        q.put((rank, bool(ok_field), bool(ok_sweep), None))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # report to the parent instead of hanging it
        q.put((rank, False, False, repr(e)))


@pytest.mark.parametrize("world", [2, 3])
def test_z_slab_exchange_and_sweep_gloo(world, oracle_mod):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    m, n, p, nv, buff = 9, 7, 3 * world * 9 - 1, 2, 6
    procs = [ctx.Process(target=_worker, args=(r, world, port, m, n, p, nv, buff, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
    for rank, ok_field, ok_sweep, err in sorted(res):
        assert err is None, err
        assert ok_field, f"rank {rank}: ghost planes differ from the global field"
        assert ok_sweep, f"rank {rank}: slab z sweep differs from the global sweep"


def test_slab_bounds_cover_exactly():
    from wenostandalone_b200 import sharding
    for p in (0, 5, 199, 255):
        for w in (1, 2, 3, 8):
            cells = []
            for r in range(w):
                z0, nz = sharding.slab_bounds(p, w, r)
                cells.extend(range(z0, z0 + nz))
            assert cells == list(range(p + 1))


def test_lpt_assignment_balances():
    from wenostandalone_b200 import sharding
    rng = np.random.default_rng(0)
    costs = list(rng.integers(16, 113, 96) ** 3)
    parts = sharding.lpt_assign(costs, 8)
    assert sorted(i for p in parts for i in p) == list(range(96))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) / (sum(costs) / 8) < 1.15


def _bench_zslab_worker(rank, world, port, m, n, p, nv, buff, q):
    """The bench's --decomp zslab step (bench.zslab_local_field, zslab_step)
    on CPU tensors with gloo, the oracle standing in for the GPU sweeps."""
    import sys
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import torch
    import torch.distributed as dist
    import bench
    import oracle
    from wenostandalone_b200 import fields, sharding
    try:
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
        glob = fields.smooth_jump_field(m, n, p, nv, buff, seed=17)
        slab = sharding.ZSlab(m, n, p, nv, buff, world, rank)
        v = bench.zslab_local_field(slab, torch.from_numpy(glob.ravel(order="F").copy()))
        # the ghost planes shared with a neighbour start out poisoned: the exchange must fill them
        loc = v.view(nv, slab.E3, slab.E1 * slab.E2)
        if rank > 0:
            loc[:, :slab.G, :] = float("nan")
        if rank < world - 1:
            loc[:, slab.nz + slab.G:, :] = float("nan")
        shape = (slab.E1, slab.E2, slab.E3, nv)
        out = {}

        def sweep(d):
            f = np.asfortranarray(v.numpy().reshape(shape, order="F"))
            rs = oracle.reshape(f, m, n, slab.p_local, buff, d)
            L, R = oracle.reconstruct(rs, fields.uniform_weno_coefficients(5, rs.shape[0] - 12), 5)
            oracle.preserve_monotonicity(rs, L, R)
            out[d] = (L, R)

        bench.zslab_step(slab, v, sweep)
        lo, hi = slab.owned_cells()
        ok = []
        for d in range(3):
            rs = oracle.reshape(glob, m, n, p, buff, d)
            Lg, Rg = oracle.reconstruct(rs, fields.uniform_weno_coefficients(5, rs.shape[0] - 12), 5)
            oracle.preserve_monotonicity(rs, Lg, Rg)
            L, R = out[d]
            if d < 2:
                # x, y sweeps: the owned z planes (last axis of the face array before V)
                sl_l, sl_g = slice(lo, hi), slice(slab.z0 + lo, slab.z0 + hi)
                ok.append(np.array_equal(L[:, :, sl_l], Lg[:, :, sl_g]) and
                          np.array_equal(R[:, :, sl_l], Rg[:, :, sl_g]))
            else:
                # z sweep: the owned faces within the core
                ns_l = L.shape[0]
                a, b = max(lo, 3), min(hi, ns_l - 3)
                ok.append(np.array_equal(L[a:b], Lg[slab.z0 + a:slab.z0 + b]) and
                          np.array_equal(R[a:b], Rg[slab.z0 + a:slab.z0 + b]))
        q.put((rank, ok, (lo, hi), None))
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # report to the parent instead of hanging it
        q.put((rank, [False], None, repr(e)))


@pytest.mark.parametrize("world", [2, 3])
def test_bench_zslab_step_gloo(world, oracle_mod):
    """bench.py --decomp zslab's step on CPU ranks: every rank's owned
    results of the x, y and z sweeps equal the undecomposed block's, bit for
    bit, and the owned cells tile the block's z range exactly."""
    from wenostandalone_b200 import sharding
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    m, n, p, nv, buff = 8, 6, 11 * world - 1, 2, 6
    procs = [ctx.Process(target=_bench_zslab_worker, args=(r, world, port, m, n, p, nv, buff, q))
             for r in range(world)]
    for pr in procs:
        pr.start()
    res = [q.get(timeout=180) for _ in range(world)]
    for pr in procs:
        pr.join(timeout=60)
    cover = []
    for rank, ok, owned, err in sorted(res, key=lambda r: r[0]):
        assert err is None, err
        assert all(ok), f"rank {rank}: owned sweep results differ from the undecomposed block ({ok})"
        slab = sharding.ZSlab(m, n, p, nv, buff, world, rank)
        cover.extend(range(slab.z0 + owned[0], slab.z0 + owned[1]))
    # every z cell of the block (ghost layers included) has exactly one owner
    assert cover == list(range(p + 1 + 2 * buff))


def test_bench_batch_assignment_covers_every_block():
    import sys
    sys.path.insert(0, ROOT)
    import bench
    blocks = bench._batch_blocks()
    for world in (1, 2, 4, 8):
        parts = bench.batch_assignment(blocks, world)
        assert sorted(i for p in parts for i in p) == list(range(len(blocks)))
