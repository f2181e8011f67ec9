"""tg_build_neighbors_list_noalloc (scratch in a fixed device array, nothing
allocated) against tg_build_neighbors_list on the same structures.

Both run the same cell-list kernels, so lists, distances and vectors must agree
bit for bit. Two different structures go through the no-allocation call back to
back (then the first again), so scratch left behind by one call cannot leak into
the next. Named to be collected last: it must pass after every other test as
well as alone."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from turbogap_b200 import backend as B
from turbogap_b200._lib import lib
from turbogap_b200.synth import random_structure

pytestmark = pytest.mark.gpu

RCUT = 3.7
MAX_SITES = 131072


def _reference(st):
    """The allocating entry point (host buffers, single unit cell)."""
    box = st.box
    return B.build_neighbors_list(st.positions, st.n, box[0], box[1], box[2], RCUT, [1, 1, 1],
                                  st.species)


def _noalloc(st, cap, stream):
    import torch

    dev = torch.device("cuda:0")
    n = st.n
    pos = torch.from_numpy(np.ascontiguousarray(st.positions, np.float64)).to(dev)
    n_neigh = torch.empty(n, dtype=torch.int32, device=dev)
    pstart = torch.empty(n + 1, dtype=torch.int64, device=dev)
    nbr = torch.empty(max(cap, 1), dtype=torch.int32, device=dev)
    rjs = torch.empty(max(cap, 1), dtype=torch.float64, device=dev)
    xyz = torch.empty((max(cap, 1), 3), dtype=torch.float64, device=dev)
    box = [np.ascontiguousarray(v, np.float64) for v in st.box]
    P = C.c_int64(-1)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    rc = lib().tg_build_neighbors_list_noalloc(
        n, pos.data_ptr(), box[0], box[1], box[2], RCUT, cap, n_neigh.data_ptr(),
        pstart.data_ptr(), nbr.data_ptr(), rjs.data_ptr(), xyz.data_ptr(), C.byref(P), stream)
    free1 = torch.cuda.mem_get_info(0)[0]
    out = None
    if rc == 0:
        k = int(P.value)
        out = dict(n_neigh=n_neigh.cpu().numpy(), pstart=pstart.cpu().numpy(),
                   neighbors_list=nbr[:k].cpu().numpy(), rjs=rjs[:k].cpu().numpy(),
                   xyz=xyz[:k].cpu().numpy())
    return rc, int(P.value), out, free0 - free1


def _same(ref, out):
    assert np.array_equal(ref["n_neigh"], out["n_neigh"])
    assert np.array_equal(np.concatenate([[0], np.cumsum(ref["n_neigh"])]), out["pstart"])
    assert np.array_equal(ref["neighbors_list"], out["neighbors_list"])
    assert np.array_equal(ref["rjs"], out["rjs"])
    assert np.array_equal(ref["xyz"], out["xyz"])


def test_noalloc_matches_allocating_entry_twice(gpu):
    import torch

    stream = torch.cuda.current_stream(0).cuda_stream
    st_a = random_structure(2000, 27.5, 1.2, seed=71)
    st_b = random_structure(3000, 31.0, 1.1, seed=72)
    ref_a, ref_b = _reference(st_a), _reference(st_b)
    cap = 60 * 3000
    # first call: the per-device set-up, which (lazy module loading) may load the
    # module and its fixed array, so its memory change is not checked
    rc, P, out_a, _ = _noalloc(st_a, cap, stream)
    assert rc == 0, lib().tg_last_error()
    assert P == len(ref_a["neighbors_list"])
    _same(ref_a, out_a)
    rc, P, out_b, grew_b = _noalloc(st_b, cap, stream)     # second call, other structure
    assert rc == 0, lib().tg_last_error()
    assert P == len(ref_b["neighbors_list"])
    _same(ref_b, out_b)
    rc, P, out_a2, grew_a = _noalloc(st_a, cap, stream)    # back to the first
    assert rc == 0, lib().tg_last_error()
    _same(ref_a, out_a2)
    assert grew_b == 0 and grew_a == 0, "device memory changed across a no-allocation call"


def test_noalloc_limits(gpu):
    import torch

    stream = torch.cuda.current_stream(0).cuda_stream
    st = random_structure(1500, 25.0, 1.2, seed=73)
    need = len(_reference(st)["neighbors_list"])
    rc, P, _, _ = _noalloc(st, need - 1, stream)             # caller arrays one pair short
    assert rc == -3 and P == need
    rc, P, out, _ = _noalloc(st, need, stream)               # exactly enough
    assert rc == 0 and P == need and out["pstart"][-1] == need
    nul = C.c_void_p()
    box = [np.eye(3)[k] * 80.0 for k in range(3)]
    Pn = C.c_int64(0)
    rc = lib().tg_build_neighbors_list_noalloc(MAX_SITES + 1, 1, box[0], box[1], box[2], RCUT,
                                               1, 1, 1, 1, 1, 1, C.byref(Pn), nul)
    assert rc == -3 and b"no-allocation limit" in lib().tg_last_error()
    tri = [np.array([20.0, 0, 0]), np.array([5.0, 20.0, 0]), np.array([0, 0, 20.0])]
    rc = lib().tg_build_neighbors_list_noalloc(10, 1, tri[0], tri[1], tri[2], RCUT,
                                               1, 1, 1, 1, 1, 1, C.byref(Pn), nul)
    assert rc == -1 and b"orthorhombic" in lib().tg_last_error()
    cube = [np.eye(3)[k] * 20.0 for k in range(3)]
    for bad in (0.0, -1.0, float("nan"), float("inf")):        # rcut_max checked first
        rc = lib().tg_build_neighbors_list_noalloc(10, 1, cube[0], cube[1], cube[2], bad,
                                                   1, 1, 1, 1, 1, 1, C.byref(Pn), nul)
        assert rc == -1 and b"rcut_max" in lib().tg_last_error()
    huge = [np.eye(3)[k] * 1e12 for k in range(3)]             # cells per axis overflow int
    rc = lib().tg_build_neighbors_list_noalloc(10, 1, huge[0], huge[1], huge[2], RCUT,
                                               1, 1, 1, 1, 1, 1, C.byref(Pn), nul)
    assert rc == -3 and b"no-allocation limit" in lib().tg_last_error()
