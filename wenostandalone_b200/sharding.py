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


class ZSlab:
    """One block of (m+1) x (n+1) x (p+1) cells split along z over `world`
    ranks: this rank's slab of nz cells, stored as a v_vf array of its own
    (E1, E2, nz + 2G, V) with G = buff_size + 3 ghost planes per side, so
    the library sweeps it as a block of p_cells = nz - 1.  The x and y
    sweeps need nothing from the neighbours; the z sweep needs the G planes
    next to the slab on each side, which exchange() fetches (MFC's halo
    exchange).  Neighbouring slabs overlap in buff_size cells on each side of
    a cut (the slab's own ghost layers), whose results both compute; each
    cell belongs to one rank (owned_cells)."""

    def __init__(self, m: int, n: int, p: int, nv: int, buff: int, world: int, rank: int):
        self.m, self.n, self.p, self.nv, self.buff = m, n, p, nv, buff
        self.world, self.rank = world, rank
        self.z0, self.nz = slab_bounds(p, world, rank)
        self.G = ghost_planes(buff)
        if world > 1 and self.nz < self.G:
            raise ValueError(f"{p + 1} cells over {world} ranks leaves slabs of {self.nz} cells, thinner than "
                             f"the {self.G} ghost planes each must supply")
        self.E1 = m + 2 * buff + 7
        self.E2 = n + 2 * buff + 7
        self.E3 = self.nz + 2 * self.G
        self.p_local = self.nz - 1

    def global_planes(self):
        """[first, last) planes of the global v_vf array that the slab holds
        (global plane k holds interior cell k - G)."""
        return self.z0, self.z0 + self.E3

    def exchange(self, v_local, group=None) -> None:
        exchange_z_ghosts(v_local, self.E1, self.E2, self.nz, self.nv, self.buff, group)

    def owned_cells(self):
        """[lo, hi) of the slab's z cells, in local indices 0 .. nz + 2 buff
        (local index k is global cell z0 + k - buff), whose results this rank
        owns: its nz interior cells, plus the lower ghost cells on the first
        rank and the upper ones on the last.  The x and y sweeps' face states
        of a z plane, and the z sweep's of a face (a face is indexed by its
        cell), belong to the owner of that cell; a neighbour's copy is
        identical.  (The z sweep writes core faces only: clip to
        [3, nz + 2 buff - 3).)"""
        lo = 0 if self.rank == 0 else self.buff
        hi = self.nz + 2 * self.buff if self.rank == self.world - 1 else self.buff + self.nz
        return lo, hi
