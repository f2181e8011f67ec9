"""Two ranks over gloo on CPU: the atom-range split of the reference
(turbogap.f90:930-942) with per-rank neighbour lists and SOAP/GAP work, followed
by the energy/force/virial reduction (turbogap.f90:1876-1885), reproduces the
single-process result. The oracle computes each rank's share."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from turbogap_b200.parallel import reduce_efv, site_range


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from _util import O, sparse_block
        from turbogap_b200.hypers import carbon_hypers
        from turbogap_b200.synth import random_structure
        h = carbon_hypers()
        blk = sparse_block(h, 60, seed=41, n_atoms=64, L=8.5, n_structs=1)
        st = random_structure(64, 8.5, 1.2, seed=42)
        beg, end = site_range(st.n, world, rank)
        e, f, v, _ = O.evaluate(st.positions, st.species, st.box, [blk], site_range=(beg, end))
        # e0 is zero here; each rank holds energies of its own sites only
        E, F, V = (torch.from_numpy(np.ascontiguousarray(x)) for x in (e, f, v))
        reduce_efv(E, F, V)
        if rank == 0:
            e1, f1, v1, _ = O.evaluate(st.positions, st.species, st.box, [blk])
            out.put((float(np.abs(E.numpy() - e1).max()), float(np.abs(F.numpy() - f1).max()),
                     float(np.abs(V.numpy() - v1).max())))
    finally:
        dist.destroy_process_group()


def test_site_range_matches_reference_split():
    n, ntasks = 10, 3
    got = [site_range(n, ntasks, r) for r in range(ntasks)]
    # Fortran: ranks 0 get 4 sites (1..4), rank 1 3 sites (5..7), rank 2 3 sites (8..10)
    assert got == [(0, 4), (4, 7), (7, 10)]
    assert sum(e - b for b, e in got) == n


def test_two_rank_decomposition_matches_single_process():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    de, df, dv = res
    assert de < 1e-12 and df < 1e-12 and dv < 1e-11


def _id_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from turbogap_b200.parallel import share_id
        made = []

        def make():
            made.append(rank)
            return bytes(range(128))

        got = share_id(make)
        out.put((rank, got, made))
    finally:
        dist.destroy_process_group()


def test_communicator_id_reaches_every_rank():
    """The NCCL id of a sharded engine is made on rank 0 only and every rank
    receives the same 128 bytes (the host half of parallel.shard_engine)."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_id_worker, args=(r, 3, port, q)) for r in range(3)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(3))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got, made in res:
        assert got == bytes(range(128))
        assert made == ([0] if rank == 0 else [])
