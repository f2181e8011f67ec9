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
