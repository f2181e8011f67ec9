"""Batched evaluation of independent structures of uneven size (the batched
kind) against the FP64 oracle, structure by structure: boxes below 2 rcut (several
images of a neighbour), between 2 and 3 rcut (minimum image) and above 3 rcut
(cell lists)."""
from __future__ import annotations

import numpy as np
import pytest

from _util import O, sparse_block
from turbogap_b200 import synth
from turbogap_b200.hypers import carbon_hypers

pytestmark = pytest.mark.gpu

E_TOL = 1e-6    # eV/atom
F_TOL = 1e-6    # eV/A
V_TOL = 1e-6    # relative to the largest virial component


def _cells():
    # (atoms, density g/cm3): L from 6.2 A (< 2 rcut) to 19 A (> 3 rcut)
    spec = [(64, 3.5), (64, 1.5), (120, 2.0), (300, 2.4), (700, 3.0), (150, 1.8)]
    out = []
    for k, (n, rho) in enumerate(spec):
        L = (n / synth.carbon_number_density(rho)) ** (1 / 3)
        out.append(synth.random_structure(n, L, 1.2, seed=500 + k))
    return out


def test_batch_matches_oracle_per_structure(gpu):
    h = carbon_hypers()
    blk = sparse_block(h, 300, seed=41)
    gpu.soap_backend_begin(blk, key=4242)
    cells = _cells()
    assert min(c.box[0, 0] for c in cells) < 2 * h.rcut_max < max(c.box[0, 0] for c in cells)
    bat = gpu.Batch(cells, [4242])
    e, f, v = bat.compute()
    e2, f2, v2 = bat.compute()            # second call replays the CUDA graph
    assert np.array_equal(e, e2) or np.max(np.abs(e - e2)) < 1e-12
    off = 0
    for s, st in enumerate(cells):
        eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, [blk])
        sl = slice(off, off + st.n)
        assert np.max(np.abs(e[sl] - eo)) < E_TOL, s
        assert np.max(np.abs(f[sl] - fo)) < F_TOL, s
        assert np.max(np.abs(v[s] - vo)) < V_TOL * max(1.0, np.max(np.abs(vo))), s
        off += st.n
    bat.close()


@pytest.mark.parametrize("slots", ["0", "8"])
def test_batch_list_builds_agree(gpu, monkeypatch, slots):
    """The one-pass list build (pairs counted into fixed rows, then compacted)
    against the two-pass build (TGB_BATCH_SLOTS=0) and against rows too short for
    every atom (8), where each step falls back to the second search: the same
    energies, forces and virials."""
    h = carbon_hypers()
    blk = sparse_block(h, 300, seed=41)
    gpu.soap_backend_begin(blk, key=4242)
    cells = _cells()
    ref = gpu.Batch(cells, [4242])
    e1, f1, v1 = ref.compute()
    ref.close()
    monkeypatch.setenv("TGB_BATCH_SLOTS", slots)
    bat = gpu.Batch(cells, [4242])
    for _ in range(2):                      # the second call replays the CUDA graph
        e, f, v = bat.compute()
        assert np.max(np.abs(e - e1)) < 1e-12 and np.max(np.abs(f - f1)) < 1e-9
        assert np.max(np.abs(v - v1)) < 1e-9
    bat.close()



def test_batch_dense_cell_rounds(gpu):
    """A cell structure dense enough (0.25 atoms/A^3, 4 cells per axis) that each
    cell's neighbourhood exceeds the 256 candidates the search stages at once,
    batched with a small one: per-structure parity with the oracle."""
    h = carbon_hypers()
    blk = sparse_block(h, 300, seed=41)
    gpu.soap_backend_begin(blk, key=4242)
    cells = [synth.random_structure(850, 15.0, 1.0, seed=531),
             synth.random_structure(64, 7.0, 1.2, seed=532)]
    bat = gpu.Batch(cells, [4242])
    e, f, v = bat.compute()
    off = 0
    for s, st in enumerate(cells):
        eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, [blk])
        sl = slice(off, off + st.n)
        assert np.max(np.abs(e[sl] - eo)) < E_TOL, s
        assert np.max(np.abs(f[sl] - fo)) < F_TOL, s
        # the virial per atom (its parity bound): a sum over about 50 000 pair
        # terms whose forces carry the 1e-6 eV/A bound
        assert np.max(np.abs(v[s] - vo)) / st.n < 1e-6, s
        off += st.n
    bat.close()
