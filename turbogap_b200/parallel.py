"""Atom-range decomposition across ranks (one process per GPU).

The reference distributes central atoms over MPI ranks as contiguous ranges
(turbogap.f90:930-942): the first mod(n, ntasks) ranks get n/ntasks + 1 sites.
Each rank builds neighbour lists and SOAP/GAP work for its own sites only; the
per-atom energies, forces and the virial of all ranks are summed into every
atom (turbogap.f90:1876-1885). ``site_range`` restates the split; ``reduce_efv``
is the exchange step over torch.distributed (NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations


def site_range(n_sites: int, ntasks: int, rank: int):
    """0-based [beg, end) of the sites owned by ``rank`` (turbogap.f90:930-942)."""
    q, r = divmod(n_sites, ntasks)
    if rank < r:
        beg = rank * (q + 1)
        end = (rank + 1) * (q + 1)
    else:
        beg = r * (q + 1) + (rank - r) * q
        end = beg + q
    return beg, end


def reduce_efv(energies, forces, virial, group=None):
    """Sum per-rank partial energies (n), forces (n,3) and virial (3,3) in place
    (torch tensors) over the process group: the reference's mpi_reduce of E/F/W."""
    import torch.distributed as dist
    for t in (energies, forces, virial):
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return energies, forces, virial


def share_id(make_id, group=None) -> bytes:
    """The bytes ``make_id()`` returns on rank 0, on every rank of the group
    (a torch.distributed broadcast; any backend)."""
    import torch.distributed as dist
    box = [make_id() if dist.get_rank(group) == 0 else None]
    dist.broadcast_object_list(box, src=0, group=group)
    return bytes(box[0])


def shard_engine(engine, group=None):
    """Make ``engine`` (the same structure on every rank) one rank's shard: it
    evaluates this rank's contiguous range of central sites and sums forces,
    energies and the virial over the ranks with NCCL inside every step (the
    reference's MPI split and reduction, turbogap.f90:930-942, 1876-1885).
    Collective: every rank of ``group`` calls it. Returns (beg, end)."""
    import torch.distributed as dist
    from . import backend
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    beg, end = site_range(engine.n, world, rank)
    engine.set_site_range(beg, end)
    if world > 1:
        engine.set_comm(share_id(backend.nccl_unique_id, group), world, rank)
    return beg, end
