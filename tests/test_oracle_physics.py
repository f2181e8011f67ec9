"""Self-consistency of the FP64 oracle, after tests/fd_gap of the reference:
analytic forces and virial against central finite differences of the oracle's
own energy (h = 1e-3 A, strain 1e-4, relative tolerance 1e-4 as in
tests/fd_gap/run.sh), plus the invariances a SOAP-GAP energy must have
(translation, rotation, permutation), zero net force and unit-norm descriptors."""
import numpy as np
import pytest

from _util import O, oracle_descriptors, sparse_block
from turbogap_b200.hypers import carbon_hypers, ch_hypers
from turbogap_b200.synth import random_structure

H_FD = 1e-3
STRAIN = 1e-4


@pytest.fixture(scope="module")
def carbon():
    h = carbon_hypers()
    blk = sparse_block(h, 120, seed=21, n_atoms=64, L=8.5, n_structs=3)
    st = random_structure(64, 8.5, 1.2, seed=22)
    return st, blk


@pytest.fixture(scope="module")
def two_species():
    L = (90 / 0.12) ** (1 / 3)
    bC = sparse_block(ch_hypers(1), 80, seed=23, n_atoms=90, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=3)
    bH = sparse_block(ch_hypers(2), 60, seed=24, n_atoms=90, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=4)
    st = random_structure(90, L, 1.0, seed=25, h_fraction=0.25)
    return st, [bC, bH]


def _energy(st, blocks, pos=None, box=None):
    e, _, _, _ = O.evaluate(st.positions if pos is None else pos, st.species,
                            st.box if box is None else box, blocks)
    return e.sum()


@pytest.mark.parametrize("which", ["carbon", "two_species"])
def test_forces_match_finite_differences(which, request):
    st, blocks = request.getfixturevalue(which)
    blocks = blocks if isinstance(blocks, list) else [blocks]
    _, f, _, _ = O.evaluate(st.positions, st.species, st.box, blocks)
    for i in (0, 7, 31):
        for q in range(3):
            p = st.positions.copy()
            p[i, q] += H_FD
            ep = _energy(st, blocks, pos=p)
            p[i, q] -= 2 * H_FD
            em = _energy(st, blocks, pos=p)
            fd = -(ep - em) / (2 * H_FD)
            assert abs(fd - f[i, q]) <= 1e-4 * max(abs(f[i, q]), 1e-3 * np.abs(f).max())


@pytest.mark.parametrize("which", ["carbon", "two_species"])
def test_virial_matches_strain_derivative(which, request):
    """virial_ab = -dE/d(eps_ab) under the homogeneous strain r -> (1 + eps) r."""
    st, blocks = request.getfixturevalue(which)
    blocks = blocks if isinstance(blocks, list) else [blocks]
    _, _, vir, _ = O.evaluate(st.positions, st.species, st.box, blocks)
    for a, b in ((0, 0), (1, 1), (0, 1), (1, 2)):
        def strained(s):
            eps = np.eye(3)
            eps[a, b] += s
            return _energy(st, blocks, pos=st.positions @ eps.T, box=st.box @ eps.T)
        dE = (strained(STRAIN) - strained(-STRAIN)) / (2 * STRAIN)
        assert abs(-dE - vir[a, b]) <= 1e-4 * np.abs(vir).max()


def test_invariances_and_sum_rules(carbon):
    st, blk = carbon
    e, f, v, _ = O.evaluate(st.positions, st.species, st.box, [blk])
    assert np.abs(f.sum(0)).max() < 1e-12
    assert np.allclose(v, v.T, atol=1e-12)
    # translation
    e2, f2, _, _ = O.evaluate(st.positions + np.array([0.3, -1.7, 2.2]), st.species, st.box, [blk])
    assert np.allclose(e2, e, atol=1e-12) and np.allclose(f2, f, atol=1e-11)
    # permutation of atom order
    perm = np.random.default_rng(0).permutation(st.n)
    e3, f3, _, _ = O.evaluate(st.positions[perm], st.species[perm], st.box, [blk])
    assert np.allclose(e3, e[perm], atol=1e-12) and np.allclose(f3, f[perm], atol=1e-11)


def test_rotation_invariance_of_descriptor():
    """A cubic-box rotation by 90 degrees about z (a lattice symmetry) leaves q unchanged
    and rotates forces."""
    h = carbon_hypers()
    blk = sparse_block(h, 50, seed=26, n_atoms=64, L=8.5, n_structs=1)
    st = random_structure(64, 8.5, 1.2, seed=27)
    R = np.array([[0.0, -1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]])
    pos_r = np.mod(st.positions @ R.T, 8.5)
    from turbogap_b200.synth import Structure
    st_r = Structure(pos_r, st.species, st.box)
    q, _, _ = oracle_descriptors(st, h)
    qr, _, _ = oracle_descriptors(st_r, h)
    # the oracle's radial sums carry ~1e-11 FP64 cancellation noise
    assert np.abs(q - qr).max() < 1e-10
    assert np.allclose(np.linalg.norm(q, axis=1), 1.0, atol=1e-14)
    _, f, _, _ = O.evaluate(st.positions, st.species, st.box, [blk])
    _, fr, _, _ = O.evaluate(st_r.positions, st.species, st.box, [blk])
    assert np.abs(fr - f @ R.T).max() < 1e-11


def test_energy_continuous_across_cutoff():
    """Moving a neighbour through rcut_hard changes the energy smoothly (buffer filter)."""
    h = carbon_hypers()
    blk = sparse_block(h, 40, seed=28, n_atoms=64, L=8.5, n_structs=1)
    from turbogap_b200.synth import Structure
    es = []
    for d in np.linspace(3.65, 3.75, 11):
        pos = np.array([[4.0, 4.0, 4.0], [4.0 + d, 4.0, 4.0]])
        es.append(O.evaluate(pos, np.array([1, 1], np.int32), np.eye(3) * 12.0, [blk])[0].sum())
    es = np.array(es)
    assert np.abs(np.diff(es)).max() < 1e-12


def test_triclinic_forces_and_virial_match_finite_differences():
    """A sheared cell through the reference's triclinic path (Gram-inverse
    get_distance, brute-force lists, supercell replicas): forces and virial
    against central finite differences of the oracle's own energy."""
    from turbogap_b200.hypers import SoapTurboHypers
    from turbogap_b200.synth import Structure
    h = SoapTurboHypers(species_z=[1, 2], alpha_max=[4, 4], l_max=4, central_species=1)
    L0 = (60 / 0.12) ** (1 / 3)
    blk = sparse_block(h, 40, seed=26, n_atoms=60, L=L0, d_min=1.0, h_fraction=0.25,
                       n_structs=2)
    cube = random_structure(60, L0, 1.0, seed=27, h_fraction=0.25)
    box = np.array([[1.0, 0.0, 0.0], [0.2, 1.0, 0.0], [-0.15, 0.1, 1.0]]) * L0
    st = Structure((cube.positions / L0) @ box, cube.species, box)
    _, f, vir, _ = O.evaluate(st.positions, st.species, st.box, [blk])
    for i in (0, 17, 42):
        for q in range(3):
            p = st.positions.copy()
            p[i, q] += H_FD
            ep = _energy(st, [blk], pos=p)
            p[i, q] -= 2 * H_FD
            em = _energy(st, [blk], pos=p)
            fd = -(ep - em) / (2 * H_FD)
            assert abs(fd - f[i, q]) <= 1e-4 * max(abs(f[i, q]), 1e-3 * np.abs(f).max())
    for a, b in ((0, 0), (0, 1), (2, 1)):
        def strained(s):
            eps = np.eye(3)
            eps[a, b] += s
            return _energy(st, [blk], pos=st.positions @ eps.T, box=st.box @ eps.T)
        dE = (strained(STRAIN) - strained(-STRAIN)) / (2 * STRAIN)
        assert abs(-dE - vir[a, b]) <= 1e-4 * np.abs(vir).max()
