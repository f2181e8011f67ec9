"""Edge cases the reference meets in production, against the FP64 oracle:
a block whose central species is absent (no central sites), atoms without
neighbours (only the self pair: the central weight alone makes the descriptor),
an empty batch of sites through get_gap_soap, and a one-atom cell (a supercell
of images only)."""
import numpy as np
import pytest

from _util import O, neighbor_data, sparse_block
from turbogap_b200.hypers import carbon_hypers, ch_hypers
from turbogap_b200.synth import Structure, random_structure

pytestmark = pytest.mark.gpu

L = (300 / 0.12) ** (1 / 3)


@pytest.fixture(scope="module")
def blocks(gpu):
    bC = sparse_block(ch_hypers(1), 200, seed=71, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=2)
    bH = sparse_block(ch_hypers(2), 150, seed=72, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=4)
    gpu.soap_backend_begin(bC, key=2001)
    gpu.soap_backend_begin(bH, key=2002)
    return bC, bH


def _check(gpu, st, blocks, keys):
    e0 = np.array([-0.5, -0.25])
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, list(blocks), e0=e0)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, keys, e0_by_species=e0)
    e, f, v = eng.compute()
    eng.close()
    assert np.all(np.isfinite(e)) and np.all(np.isfinite(f))
    assert np.abs(e - eo).max() < 1e-6
    assert np.abs(f - fo).max() < 1e-6
    # relative to the largest component, but at least 1e-7 absolute: the virial of
    # two small clusters is of order 1e-2
    assert np.abs(v - vo).max() <= 1e-6 * max(np.abs(vo).max(), 0.1)
    return e, f


def test_block_without_central_sites(gpu, blocks):
    """Only carbon: the H-centred block has no sites and adds nothing."""
    st = random_structure(200, (200 / 0.1) ** (1 / 3), 1.2, seed=73)
    assert np.all(st.species == 1)
    _check(gpu, st, blocks, [2001, 2002])


def test_isolated_atoms(gpu, blocks):
    """Two far-apart C/H clusters and two lone atoms in a 30 A box: the lone
    atoms' lists hold the self pair only."""
    rng = np.random.default_rng(74)
    box = np.eye(3) * 30.0
    pos, sp = [], []
    for k, centre in enumerate((np.array([5.0, 5.0, 5.0]), np.array([20.0, 20.0, 8.0]))):
        while len(pos) < 12 * (k + 1):   # 12 atoms per cluster
            p = centre + rng.uniform(-2.5, 2.5, 3)
            if all(np.linalg.norm(p - q) > 1.1 for q in pos):
                pos.append(p)
                sp.append(1 if rng.uniform() < 0.75 else 2)
    pos += [np.array([12.0, 27.0, 20.0]), np.array([27.0, 3.0, 25.0])]
    sp += [1, 2]
    st = Structure(np.array(pos), np.array(sp, np.int32), box)
    nl = neighbor_data(st, 3.7)
    assert nl["n_neigh"][-1] == 1 and nl["n_neigh"][-2] == 1
    e, f = _check(gpu, st, blocks, [2001, 2002])
    assert np.abs(f[-2:]).max() == 0.0


def test_empty_batch_of_sites(gpu, blocks):
    """get_gap_soap over zero sites leaves the outputs as they were."""
    bC, _ = blocks
    gpu.soap_backend_begin(bC, key=2001)
    st = random_structure(50, 9.0, 1.2, seed=75)
    e, f, v = gpu.get_gap_soap(st.n, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0),
                               np.zeros((0, 3)), np.zeros(0, np.int32), st.species)
    assert not e.any() and not f.any() and not v.any()


def test_one_atom_cell(gpu):
    """One C atom in a 2.5 A cube: every neighbour is an image of itself (the
    reference's supercell replication, then the brute-force list search)."""
    h = carbon_hypers()
    blk = sparse_block(h, 100, seed=76, n_atoms=64, L=8.5, n_structs=2)
    gpu.soap_backend_begin(blk, key=2003)
    st = Structure(np.array([[0.3, 0.4, 0.5]]), np.array([1], np.int32), np.eye(3) * 2.5)
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, [blk])
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [2003])
    e, f, v = eng.compute()
    eng.close()
    assert abs(e[0] - eo[0]) < 1e-6
    assert np.abs(f).max() < 1e-6 and np.abs(fo).max() < 1e-9   # a lattice: no net force
    assert np.abs(v - vo).max() <= 1e-6 * max(np.abs(vo).max(), 1e-3)
