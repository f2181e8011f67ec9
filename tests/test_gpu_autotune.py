"""The CTA-tile autotuner of the descriptor and force passes: every tile gives
the oracle's energies and forces (the descriptor does not depend on the tile),
the tuner picks one of them for every block, and the batched path reports its
picks. Tiles are pinned with TGB_SOAP_TILE for the comparison. Tile 4 is the
force pass's tensor-core kernel (TF32 hi/lo products; the descriptor keeps
tile 3 when 4 is pinned): the same bounds against the oracle, and forces within
1e-7 eV/A of the fp32 tiles."""
from __future__ import annotations

import os

import numpy as np
import pytest

from _util import O, sparse_block
from turbogap_b200 import synth
from turbogap_b200.hypers import carbon_hypers, ch_hypers
from turbogap_b200.synth import random_structure

pytestmark = pytest.mark.gpu

L = (300 / 0.12) ** (1 / 3)


@pytest.fixture(scope="module")
def ch(gpu):
    bC = sparse_block(ch_hypers(1), 300, seed=81, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=2)
    bH = sparse_block(ch_hypers(2), 200, seed=82, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=4)
    gpu.soap_backend_begin(bC, key=801)
    gpu.soap_backend_begin(bH, key=802)
    return bC, bH


def _with_env(name, value, fn):
    old = os.environ.get(name)
    os.environ[name] = value
    try:
        return fn()
    finally:
        if old is None:
            del os.environ[name]
        else:
            os.environ[name] = old


def test_every_tile_matches_the_oracle(gpu, ch):
    st = random_structure(300, L, 1.0, seed=83, h_fraction=0.25)
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, list(ch))
    first = None
    for t in range(5):
        def run():
            eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [801, 802])
            tiles = eng.tiles()
            out = eng.compute()
            eng.close()
            return tiles, out
        tiles, (e, f, v) = _with_env("TGB_SOAP_TILE", str(t), run)
        assert tiles == [(min(t, 3), t), (min(t, 3), t)]
        assert np.abs(e - eo).max() < 1e-6 and np.abs(f - fo).max() < 1e-6
        assert np.abs(v - vo).max() < 1e-6 * np.abs(vo).max()
        if first is None:
            first = (e, f)
        elif t < 4:   # the same descriptor and energies; forces up to the order of atomics
            assert np.abs(e - first[0]).max() < 1e-12
            assert np.abs(f - first[1]).max() < 1e-10
        else:         # the tensor-core tile rounds its products differently
            assert np.abs(e - first[0]).max() < 1e-12
            assert np.abs(f - first[1]).max() < 1e-7


def test_tuner_picks_a_tile_per_block(gpu, ch):
    st = random_structure(300, L, 1.0, seed=84, h_fraction=0.25)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [801, 802])
    tiles = eng.tiles()
    assert len(tiles) == 2 and all(0 <= a < 4 and 0 <= b < 5 for a, b in tiles)
    e, f, _ = eng.compute()
    eo, fo, _, _ = O.evaluate(st.positions, st.species, st.box, list(ch))
    assert np.abs(e - eo).max() < 1e-6 and np.abs(f - fo).max() < 1e-6
    eng.close()
    off = _with_env("TGB_AUTOTUNE", "0",
                    lambda: gpu.Engine(st.positions, st.species, st.masses, st.box, [801, 802]))
    assert off.tiles() == [(0, 0), (0, 0)]
    off.close()


def test_batch_reports_tuned_tiles(gpu):
    h = carbon_hypers()
    blk = sparse_block(h, 200, seed=85)
    gpu.soap_backend_begin(blk, key=803)
    structs = [synth.random_structure(n, L0, 1.2, seed=86 + k)
               for k, (n, L0) in enumerate([(64, 8.5), (150, 11.0), (40, 7.2)])]
    b = gpu.Batch(structs, [803])
    tiles = b.tiles()
    assert len(tiles) == 1 and 0 <= tiles[0][0] < 4 and 0 <= tiles[0][1] < 5
    e, f, v = b.compute()
    off = 0
    for s in structs:
        eo, fo, vo, _ = O.evaluate(s.positions, s.species, s.box, [blk])
        assert np.abs(e[off:off + s.n] - eo).max() < 1e-6
        assert np.abs(f[off:off + s.n] - fo).max() < 1e-6
        off += s.n
    b.close()
