"""Slab decomposition of a block along z, and the ghost-plane exchange.

The WENO path itself has no communication: every (a, b, v) column of a sweep
is independent, and a block's buff_size ghost layers (plus the harness's 3
pad cells) already hold the neighbours' data.  A multi-GPU run therefore
gives each rank its own block.  When one block is split into z-slabs, the x
and y sweeps stay local and only the z sweep needs the neighbours' planes:
G = buff_size + 3 planes per side, sent once per step before the sweeps
(MFC's halo exchange, here with torch.distributed point-to-point calls --
NCCL over NVLink on GPUs, gloo on CPU).

Arrays are 1-D tensors in Fortran order of the v_vf layout
(E1, E2, E3_local, V); a z-plane of one variable is E1*E2 contiguous values.
"""
from __future__ import annotations


def slab_bounds(p_cells: int, world: int, rank: int):
    """Interior z cells [z0, z0+nz) of rank `rank` when the p_cells+1 cells
    are split as evenly as possible."""
    total = p_cells + 1
    base, extra = divmod(total, world)
    nz = base + (1 if rank < extra else 0)
    z0 = rank * base + min(rank, extra)
    return z0, nz


def ghost_planes(buff_size: int) -> int:
    return buff_size + 3


def _planes(t, E1, E2, E3l, nv, k0, cnt):
    """View of planes [k0, k0+cnt) of every variable: shape (nv, cnt, E1*E2)."""
    return t.view(nv, E3l, E1 * E2)[:, k0:k0 + cnt, :]


def exchange_z_ghosts(v_local, E1: int, E2: int, nz: int, nv: int, buff_size: int, group=None) -> None:
    """Fill the G lower/upper ghost planes of every rank's slab from its
    neighbours' interior planes (ranks ordered along z).  Ranks at the ends
    keep their outer ghosts (physical boundary data).  Every rank posts the
    same sequence of sends and receives, so the exchange cannot deadlock."""
    import torch
    import torch.distributed as dist
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    G = ghost_planes(buff_size)
    if nz < G and world > 1:
        raise ValueError(f"slab of {nz} cells is thinner than the {G} ghost planes it must supply")
    E3l = nz + 2 * G
    ops = []
    recv_lo = recv_hi = None
    if rank > 0:
        send_lo = _planes(v_local, E1, E2, E3l, nv, G, G).contiguous()
        recv_lo = torch.empty_like(send_lo)
        ops.append(dist.P2POp(dist.isend, send_lo, rank - 1, group))
        ops.append(dist.P2POp(dist.irecv, recv_lo, rank - 1, group))
    if rank < world - 1:
        send_hi = _planes(v_local, E1, E2, E3l, nv, nz, G).contiguous()
        recv_hi = torch.empty_like(send_hi)
        ops.append(dist.P2POp(dist.isend, send_hi, rank + 1, group))
        ops.append(dist.P2POp(dist.irecv, recv_hi, rank + 1, group))
    if ops:
        for r in dist.batch_isend_irecv(ops):
            r.wait()
    if recv_lo is not None:
        _planes(v_local, E1, E2, E3l, nv, 0, G).copy_(recv_lo)
    if recv_hi is not None:
        _planes(v_local, E1, E2, E3l, nv, nz + G, G).copy_(recv_hi)


def lpt_assign(costs, world: int):
    """Longest-processing-time assignment of independent blocks to ranks:
    blocks sorted by cost, each given to the least-loaded rank.  Returns a
    list of block indices per rank."""
    loads = [0.0] * world
    out = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: -costs[k]):
        r = min(range(world), key=lambda q: (loads[q], q))
        loads[r] += costs[i]
        out[r].append(i)
    return out
