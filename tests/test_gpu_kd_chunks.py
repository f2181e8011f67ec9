"""The GAP GEMMs over row chunks (a bounded kd scratch, gap.f90:168-185).

GEMM 1 writes the split kernel derivative kd of a chunk of central sites and
GEMM 2 reads it back before the next chunk, so kd holds one chunk (1 GiB by
default). The chunking changes no per-row arithmetic: energies, forces and the
virial must match a single chunk, in the plain form and in the mixed form's
exact path over the gated sites (gate 0: every site gated), to the 1e-12 that
FP64 force and virial atomics summed in no fixed order leave (and MD steps
carry into the positions)."""
from __future__ import annotations

import numpy as np
import pytest

from _util import sparse_block
from turbogap_b200 import synth
from turbogap_b200.hypers import ch_hypers

pytestmark = pytest.mark.gpu

L300 = (300 / 0.12) ** (1 / 3)


@pytest.fixture(scope="module")
def blocks(gpu):
    bC = sparse_block(ch_hypers(1), 500, seed=81, n_atoms=300, L=L300, d_min=1.0,
                      h_fraction=0.25, n_structs=4)
    bH = sparse_block(ch_hypers(2), 300, seed=82, n_atoms=300, L=L300, d_min=1.0,
                      h_fraction=0.25, n_structs=6)
    gpu.soap_backend_begin(bC, key=801)
    gpu.soap_backend_begin(bH, key=802)
    return bC, bH


def _structure():
    return synth.random_structure(600, (600 / 0.12) ** (1 / 3), 1.0, seed=83, h_fraction=0.25)


def _run(gpu, st, mlps=None, gate=0.0, steps=0):
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [801, 802])
    if mlps:
        for i, m in enumerate(mlps):
            gpu.engine_set_mlp(eng, i, m, gate_ev=gate)
    e, f, v = eng.compute()
    if steps:
        eng.set_state(st.positions, synth.maxwell_velocities(st.masses, 600.0, 84))
        eng.md(steps, 0.5)
        e, f, v = eng.compute()
    eng.close()
    return e, f, v


def test_chunked_gemms_match(gpu, blocks, monkeypatch):
    st = _structure()
    ref = _run(gpu, st, steps=3)
    monkeypatch.setenv("TGB_KD_CHUNK_ROWS", "128")   # 450 C sites: 4 chunks, the last short
    out = _run(gpu, st, steps=3)
    _same(ref, out)


def _same(ref, out):
    assert np.abs(ref[0] - out[0]).max() < 1e-12
    assert np.abs(ref[1] - out[1]).max() < 1e-12
    assert np.abs(ref[2] - out[2]).max() < 1e-12 * max(1.0, np.abs(ref[2]).max())


def test_chunked_gated_rows_match(gpu, blocks, monkeypatch):
    """Gate 0 sends every site through the exact kernel over the compacted rows,
    whose per-chunk counts are read on the device."""
    st = _structure()
    mlps = [gpu.Mlp(b.hypers.device_dim, 256, 4, seed=90 + i) for i, b in enumerate(blocks)]
    exact = _run(gpu, st)
    ref = _run(gpu, st, mlps, gate=0.0)
    monkeypatch.setenv("TGB_KD_CHUNK_ROWS", "128")
    out = _run(gpu, st, mlps, gate=0.0)
    for m in mlps:
        m.close()
    _same(ref, out)
    # and the gated path is the exact path (same GEMMs over permuted rows)
    assert np.abs(out[0] - exact[0]).max() < 1e-12
    assert np.abs(out[1] - exact[1]).max() < 1e-10
