"""SOAP compression on the CPU: the "trivial" recipe against the compress file
that the reference's own generator writes (tests/golden/make_compress_trivial.py),
the file forms and the .gap keywords, and the oracle's compressed descriptor:
the normalised map of the power spectrum, with forces and virial against
central finite differences of its energy (the tests/fd_gap methodology,
h = 1e-3 A, strain 1e-4, relative tolerance 1e-4)."""
import os

import numpy as np
import pytest

from _util import O, neighbor_data, oracle_descriptors, sparse_block
from turbogap_b200 import formats as F
from turbogap_b200.hypers import SoapCompression, SoapTurboHypers, trivial_compression
from turbogap_b200.synth import random_structure

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "compress_trivial_n6-6_l5.txt")
L = (90 / 0.12) ** (1 / 3)


def ch_small(central, compress=None):
    return SoapTurboHypers(species_z=[1, 2], alpha_max=[4, 4], l_max=4, central_species=central,
                           compress=compress)


def random_transformation(full_dim, dim, seed, per_row=3):
    """A P_transformation of dim rows with a few random entries each; some
    columns are hit by several rows."""
    rng = np.random.default_rng(seed)
    P_i = np.repeat(np.arange(1, dim + 1), per_row)
    P_j = rng.integers(1, full_dim + 1, size=dim * per_row)
    P_el = rng.normal(size=dim * per_row)
    return SoapCompression(dim, P_i, P_j, P_el)


def test_trivial_recipe_matches_the_reference_generator():
    spec = F.read_compress_file(GOLDEN, 2)
    assert spec.alpha_max == [6, 6] and spec.l_max == 5 and spec.dim == 138
    c = spec.compression()
    t = trivial_compression([6, 6], 5)
    assert t.dim == c.dim
    assert np.array_equal(t.P_i, c.P_i) and np.array_equal(t.P_j, c.P_j)
    assert np.array_equal(t.P_el, c.P_el)


def test_gap_keywords_give_the_compression(tmp_path):
    comp_file = tmp_path / "c.dat"
    comp_file.write_text("4 4 4 3\nP_transformation\n1 1 0.5\n1 5 0.5\n2 2 1.0\n3 7 -2.0\n"
                         "end_transformation\n")
    two = [1.0, 1.0]
    spec = F.SoapTurboSpec(n_species=2, species=["C", "H"], alpha_max=[4, 4],
                           rcut_hard=[3.7, 3.7], buffer=[0.5, 0.5], atom_sigma_r=[0.5, 0.5],
                           atom_sigma_t=[0.5, 0.5], atom_sigma_r_scaling=[0.0, 0.0],
                           atom_sigma_t_scaling=[0.0, 0.0], nf=[4.0, 4.0],
                           amplitude_scaling=two, central_weight=two, global_scaling=two,
                           l_max=4, compress_soap=True, file_compress=comp_file.name)
    c = spec.compression(str(tmp_path))
    assert c.dim == 3 and c.P_i.tolist() == [1, 1, 2, 3]
    assert c.P_el.tolist() == [0.5, 0.5, 1.0, -2.0]
    # a file takes precedence over the mode (read_files.f90:5162-5165)
    spec.compress_mode = "trivial"
    assert spec.compression(str(tmp_path)).dim == 3
    spec.file_compress = "none"
    t = spec.compression(str(tmp_path))
    assert t.dim == trivial_compression([4, 4], 4).dim
    h = spec.hypers(["C", "H"])
    h.compress = t
    assert h.uncompressed_dim == 180 and h.dim == t.dim and h.device_dim % 8 == 0
    spec.compress_mode = "something_else"
    with pytest.raises(NotImplementedError, match="trivial"):
        spec.compression(str(tmp_path))


@pytest.mark.parametrize("kind", ["trivial", "transformation"])
def test_compressed_descriptor_is_the_normalised_map(kind):
    st = random_structure(90, L, 1.0, seed=91, h_fraction=0.25)
    full = ch_small(1)
    comp = (trivial_compression([4, 4], 4) if kind == "trivial"
            else random_transformation(full.uncompressed_dim, 37, seed=92))
    nl = neighbor_data(st, 3.7)
    q, nrm, sites = oracle_descriptors(st, full, nl)
    qc, nrmc, sites_c = oracle_descriptors(st, ch_small(1, comp), nl)
    assert np.array_equal(sites, sites_c) and qc.shape == (len(sites), comp.dim)
    v = (q * nrm[:, None]) @ comp.matrix(full.uncompressed_dim).T
    assert np.allclose(nrmc, np.linalg.norm(v, axis=1), rtol=1e-12)
    assert np.allclose(qc, v / np.linalg.norm(v, axis=1)[:, None], atol=1e-13)


@pytest.fixture(scope="module")
def compressed_blocks():
    full = ch_small(1)
    cC = random_transformation(full.uncompressed_dim, 37, seed=93)
    cH = trivial_compression([4, 4], 4)
    bC = sparse_block(ch_small(1, cC), 60, seed=94, n_atoms=90, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=3)
    bH = sparse_block(ch_small(2, cH), 40, seed=95, n_atoms=90, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=4)
    st = random_structure(90, L, 1.0, seed=96, h_fraction=0.25)
    return st, [bC, bH]


def _energy(st, blocks, pos=None, box=None):
    e, _, _, _ = O.evaluate(st.positions if pos is None else pos, st.species,
                            st.box if box is None else box, blocks)
    return e.sum()


def test_compressed_forces_and_virial_match_finite_differences(compressed_blocks):
    st, blocks = compressed_blocks
    _, f, vir, _ = O.evaluate(st.positions, st.species, st.box, blocks)
    h = 1e-3
    for i in (0, 11, 40):
        for q in range(3):
            p = st.positions.copy()
            p[i, q] += h
            ep = _energy(st, blocks, pos=p)
            p[i, q] -= 2 * h
            em = _energy(st, blocks, pos=p)
            fd = -(ep - em) / (2 * h)
            assert abs(fd - f[i, q]) <= 1e-4 * max(abs(f[i, q]), 1e-3 * np.abs(f).max())
    for a, b in ((0, 0), (1, 2)):
        def strained(s):
            eps = np.eye(3)
            eps[a, b] += s
            return _energy(st, blocks, pos=st.positions @ eps.T, box=st.box @ eps.T)
        dE = (strained(1e-4) - strained(-1e-4)) / 2e-4
        assert abs(-dE - vir[a, b]) <= 1e-4 * np.abs(vir).max()


def test_repeated_entries_add():
    """Entries of a transformation add up (q_c(i) += P_el p(P_j) per entry, the
    loop the file format implies): a list with an entry split in two gives the
    same descriptor as the list with the summed weight."""
    st = random_structure(90, L, 1.0, seed=97, h_fraction=0.25)
    nl = neighbor_data(st, 3.7)
    full = ch_small(1)
    base = random_transformation(full.uncompressed_dim, 20, seed=98, per_row=2)
    split = SoapCompression(base.dim, np.concatenate([base.P_i, base.P_i[:5]]),
                            np.concatenate([base.P_j, base.P_j[:5]]),
                            np.concatenate([base.P_el * 1.0, np.zeros(5)]))
    split.P_el[:5] = base.P_el[:5] * 0.25
    split.P_el[-5:] = base.P_el[:5] * 0.75
    q1, n1, _ = oracle_descriptors(st, ch_small(1, base), nl)
    q2, n2, _ = oracle_descriptors(st, ch_small(1, split), nl)
    assert np.allclose(q1, q2, atol=1e-14) and np.allclose(n1, n2, rtol=1e-14)
