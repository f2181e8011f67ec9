"""The deadline of a sharded engine's exchange step, on CPU ranks (gloo).

NCCL's communicator is non-blocking in the backend: initialisation and every
grouped all-reduce are polled with a deadline (TGB_NCCL_TIMEOUT_S), after which
the communicator is aborted and the call returns TG_ERR_TIMEOUT. Here the NCCL
library is a stand-in (tests/fake_nccl, built with gcc; loaded through
TGB_NCCL_LIBRARY) whose initialisation completes once every rank has arrived.
Two gloo ranks that both join succeed; when rank 1 never joins, rank 0 gets
TG_ERR_TIMEOUT within the deadline and tells rank 1 on the host."""
import os
import shutil
import socket
import subprocess
import tempfile
import time

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
TG_OK, TG_ERR_TIMEOUT = 0, -6


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


@pytest.fixture(scope="module")
def fake_nccl(tmp_path_factory):
    if not shutil.which("gcc"):
        pytest.skip("gcc is needed to build the NCCL stand-in")
    out = tmp_path_factory.mktemp("fake_nccl") / "libfakenccl.so"
    subprocess.run(["gcc", "-shared", "-fPIC", "-O1", "-o", str(out),
                    os.path.join(HERE, "fake_nccl", "fake_nccl.c")], check=True)
    return str(out)


def _worker(rank, world, port, lib_path, marker_dir, absent, timeout_s, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["TGB_NCCL_LIBRARY"] = lib_path
    os.environ["FAKE_NCCL_DIR"] = marker_dir
    os.environ["TGB_NCCL_TIMEOUT_S"] = str(timeout_s)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        import ctypes as C

        from turbogap_b200 import backend as B
        from turbogap_b200._lib import lib
        from turbogap_b200.parallel import share_id
        nid = share_id(B.nccl_unique_id)             # made on rank 0, broadcast over gloo
        buf = C.create_string_buffer(nid, 128)
        if rank in absent:                           # this rank never joins the communicator
            rc, dt = None, 0.0
        else:
            t0 = time.monotonic()
            rc = lib().tgx_comm_probe(C.cast(buf, C.c_void_p), world, rank)
            dt = time.monotonic() - t0
        # the ranks learn each other's outcome on the host, not through NCCL
        box = [None] * world
        dist.all_gather_object(box, rc)
        out.put((rank, rc, dt, box))
    finally:
        dist.destroy_process_group()


def _run(world, lib_path, absent, timeout_s):
    marker_dir = tempfile.mkdtemp(prefix="fake_nccl_")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker,
                         args=(r, world, port, lib_path, marker_dir, absent, timeout_s, q))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shutil.rmtree(marker_dir, ignore_errors=True)
    return res


def test_every_rank_joins(fake_nccl):
    res = _run(2, fake_nccl, absent=(), timeout_s=20)
    for rank, rc, dt, box in res:
        assert rc == TG_OK and box == [TG_OK, TG_OK]


def test_absent_rank_gives_a_timeout_not_a_hang(fake_nccl):
    res = _run(2, fake_nccl, absent=(1,), timeout_s=1)
    (r0, rc0, dt0, box0), (r1, rc1, _, box1) = res
    assert rc0 == TG_ERR_TIMEOUT
    assert 0.9 < dt0 < 30.0                      # the deadline, not forever
    assert rc1 is None and box1 == [TG_ERR_TIMEOUT, None]   # rank 1 heard of it on the host


def _shard_worker(rank, world, port, lib_path, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    os.environ["TGB_NCCL_LIBRARY"] = lib_path
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        from turbogap_b200.parallel import shard_engine

        class Recorder:   # stands in for backend.Engine: records what the shard set-up asks
            n = 1000
            calls = []

            def set_site_range(self, beg, end):
                self.calls.append(("range", beg, end))

            def set_comm(self, nccl_id, n_ranks, rank):
                self.calls.append(("comm", bytes(nccl_id), n_ranks, rank))

        e = Recorder()
        beg, end = shard_engine(e)
        out.put((rank, beg, end, e.calls))
    finally:
        dist.destroy_process_group()


def test_bench_shard_setup_over_two_ranks(fake_nccl):
    """What `bench.py --gpus 2 --shard` does to its engine on each rank
    (parallel.shard_engine): contiguous central-site ranges that cover the
    structure (turbogap.f90:930-942), and one communicator id, made on rank 0,
    joined by both ranks."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, fake_nccl, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, b0, e0, c0), (r1, b1, e1, c1) = res
    assert (b0, e0, b1, e1) == (0, 500, 500, 1000)
    assert c0[0] == ("range", 0, 500) and c1[0] == ("range", 500, 1000)
    assert c0[1][0] == "comm" and c0[1][1] == c1[1][1]          # the same id
    assert c0[1][2:] == (2, 0) and c1[1][2:] == (2, 1)
