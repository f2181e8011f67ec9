"""distance_2b, angle_3b and core_pot on the GPU against the FP64 oracle
(gap.f90:400-1042): the add_*_contribution entry point on the oracle's own
neighbour lists, and the device engine (alone, with soap_turbo blocks, sharded
by site ranges, and over an NVE run)."""
from __future__ import annotations

import numpy as np
import pytest

from _util import O, make_families, neighbor_data, sparse_block
from turbogap_b200.hypers import ch_hypers
from turbogap_b200.parallel import site_range
from turbogap_b200.synth import maxwell_velocities, random_structure

pytestmark = pytest.mark.gpu

L = (300 / 0.12) ** (1 / 3)
E_TOL = 1e-6    # eV/atom
F_TOL = 1e-6    # eV/A


@pytest.fixture(scope="module")
def fams(gpu):
    fs = make_families(7)
    for k, f in enumerate(fs):
        gpu.family_begin(f, 500 + k)
    return fs


def test_get_family_matches_oracle(gpu, fams):
    st = random_structure(300, L, 1.0, seed=51, h_fraction=0.25)
    nl = neighbor_data(st, 4.0)
    for k, f in enumerate(fams):
        eo, fo, vo = O.family_energy_forces(f, nl["n_neigh"], nl["neighbors_list"], nl["rjs"],
                                            nl["xyz"], st.species, nl["neighbor_species"], st.n)
        e, fr, v = gpu.get_family(500 + k, st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"],
                                  nl["xyz"], st.species)
        assert np.abs(eo).max() > 1e-5, f.kind            # the family is not idle
        assert np.abs(e - eo).max() < 1e-10 * max(1.0, np.abs(eo).max()), f.kind
        assert np.abs(fr - fo).max() < 1e-10 * max(1.0, np.abs(fo).max()), f.kind
        assert np.abs(v - vo).max() < 1e-10 * max(1.0, np.abs(vo).max()), f.kind
    # add semantics: a second call adds the same contribution again
    e1, f1, v1 = gpu.get_family(500, st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"],
                                nl["xyz"], st.species)
    e2, f2, v2 = gpu.get_family(500, st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"],
                                nl["xyz"], st.species, energies0=e1.copy(), forces0=f1.copy(),
                                virial=v1.copy())
    assert np.allclose(e2, 2 * e1) and np.allclose(f2, 2 * f1) and np.allclose(v2, 2 * v1)


@pytest.fixture(scope="module")
def ch_blocks(gpu):
    bC = sparse_block(ch_hypers(1), 300, seed=52, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=2)
    bH = sparse_block(ch_hypers(2), 200, seed=53, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=4)
    gpu.soap_backend_begin(bC, key=511)
    gpu.soap_backend_begin(bH, key=512)
    return bC, bH


@pytest.mark.parametrize("with_soap", [False, True])
def test_engine_with_families_matches_oracle(gpu, fams, ch_blocks, with_soap):
    st = random_structure(300, L, 1.0, seed=54, h_fraction=0.25)
    e0 = np.array([-0.5, -0.25])
    blocks = list(ch_blocks) if with_soap else []
    keys = ([511, 512] if with_soap else []) + [500, 501, 502, 503]
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, blocks, e0=e0, families=fams)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, keys, e0_by_species=e0)
    e, f, v = eng.compute()
    assert np.abs(e - eo).max() < E_TOL
    assert np.abs(f - fo).max() < F_TOL
    assert np.abs(v - vo).max() < 1e-6 * np.abs(vo).max()
    # sharded: the shares of two site ranges sum to the whole
    es, fs, vs = np.zeros_like(e), np.zeros_like(f), np.zeros_like(v)
    for rank in range(2):
        beg, end = site_range(st.n, 2, rank)
        er = gpu.Engine(st.positions, st.species, st.masses, st.box, keys, e0_by_species=e0)
        er.set_site_range(beg, end)
        a, b, c = er.compute()
        es += a
        fs += b
        vs += c
        er.close()
    assert np.abs(es - e).max() < 1e-9 and np.abs(fs - f).max() < 1e-9
    assert np.abs(vs - v).max() < 1e-9 * np.abs(v).max()
    eng.close()


def test_engine_families_small_box_supercell(gpu, fams):
    # a box shorter than twice the cutoff: the supercell path of the lists
    st = random_structure(40, 6.5, 1.0, seed=55, h_fraction=0.25)
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, [], families=fams)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [500, 501, 502, 503])
    e, f, v = eng.compute()
    assert np.abs(e - eo).max() < E_TOL and np.abs(f - fo).max() < F_TOL
    assert np.abs(v - vo).max() < 1e-6 * np.abs(vo).max()
    eng.close()


def test_engine_families_nve(gpu, fams, ch_blocks):
    st = random_structure(300, L, 1.0, seed=56, h_fraction=0.25)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [511, 512, 500, 501, 502, 503])
    eng.set_state(st.positions, maxwell_velocities(st.masses, 300.0, 57))
    ep0, ek0 = eng.md(1, 0.25)
    ep1, ek1 = eng.md(200, 0.25)
    assert abs((ep1 + ek1) - (ep0 + ek0)) / st.n < 2e-5
    eng.close()


def test_family_key_space_is_shared(gpu, fams, ch_blocks):
    with pytest.raises(gpu.BackendError):
        gpu.family_begin(fams[0], 511)      # a soap_turbo block's key
    with pytest.raises(gpu.BackendError):
        gpu.soap_backend_begin(ch_blocks[0], key=500)   # a family's key
