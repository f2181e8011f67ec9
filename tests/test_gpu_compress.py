"""Compressed soap_turbo blocks on the GPU against the FP64 oracle.

A C-centred block under a random P_transformation of 301 rows (not a multiple
of 8: the device pads the rows it keeps) and an H-centred block under the
"trivial" recipe, both on the 2 x 8, l_max 8 shape. Tolerances: descriptors
1e-7, energies 1e-6 eV/atom, forces 1e-6 eV/A, as for the uncompressed plain
form; the virial 5e-6 relative to its largest component, because on these
300-atom C/H cells a single block's virial is a sum with much cancellation: the
uncompressed C block gives 1.5e-6 on the structure of test_get_gap_soap, the
compressed blocks 1.8e-6 to 2.0e-6. The engine with a gate of 0 (every site
back to exact GAP) reproduces the plain result."""
import numpy as np
import pytest

from _util import O, neighbor_data, oracle_descriptors, sparse_block
from turbogap_b200 import synth
from turbogap_b200.hypers import SoapCompression, ch_hypers, trivial_compression

pytestmark = pytest.mark.gpu

E_TOL = 1e-6
F_TOL = 1e-6
V_TOL = 5e-6
Q_TOL = 1e-7
L = (300 / 0.12) ** (1 / 3)


def random_transformation(full_dim, dim, seed, per_row=3):
    rng = np.random.default_rng(seed)
    P_i = np.repeat(np.arange(1, dim + 1), per_row)
    P_j = rng.integers(1, full_dim + 1, size=dim * per_row)
    return SoapCompression(dim, P_i, P_j, rng.normal(size=dim * per_row))


@pytest.fixture(scope="module")
def blocks(gpu):
    hC = ch_hypers(1)
    hC.compress = random_transformation(hC.uncompressed_dim, 301, seed=81)
    hH = ch_hypers(2)
    hH.compress = trivial_compression(hH.alpha_max, hH.l_max)
    bC = sparse_block(hC, 300, seed=82, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=2)
    bH = sparse_block(hH, 200, seed=83, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=4)
    assert hC.dim == 301 and hC.device_dim == 304
    gpu.soap_backend_begin(bC, key=1801)
    gpu.soap_backend_begin(bH, key=1802)
    return bC, bH


def test_descriptors(gpu, blocks):
    st = synth.random_structure(300, L, 1.0, seed=84, h_fraction=0.25)
    for key, b in zip((1801, 1802), blocks):
        h = b.hypers
        gpu.soap_backend_begin(b, key=key)
        nl = neighbor_data(st, h.rcut_max)
        q = gpu.get_soap(st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"], nl["xyz"],
                         st.species, st.species, h.dim)
        qo, _, _ = oracle_descriptors(st, h, nl)
        assert q.shape == qo.shape == (len(qo), h.dim)
        assert np.abs(q - qo).max() < Q_TOL
        assert np.allclose(np.linalg.norm(q, axis=1), 1.0, atol=1e-6)


def test_get_gap_soap(gpu, blocks):
    bC, _ = blocks
    st = synth.random_structure(300, L, 1.0, seed=85, h_fraction=0.25)
    gpu.soap_backend_begin(bC, key=1801)
    nl = neighbor_data(st, bC.hypers.rcut_max)
    e, f, v = gpu.get_gap_soap(st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"], nl["xyz"],
                               st.species, st.species)
    eo, fo, vo = O.get_gap_soap(O.HypersC(bC.hypers), st.n, nl["n_neigh"], nl["neighbors_list"],
                                nl["rjs"], nl["xyz"], st.species, st.species, bC.Qs, bC.alphas,
                                bC.delta, bC.zeta)
    assert np.abs(e - eo).max() < E_TOL
    assert np.abs(f - fo).max() < F_TOL
    assert np.abs(v - vo).max() < V_TOL * np.abs(vo).max()


def test_engine_and_gate_zero_mixed_form(gpu, blocks):
    bC, bH = blocks
    st = synth.random_structure(300, L, 1.0, seed=86, h_fraction=0.25)
    e0 = np.array([-0.5, -0.25])
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, list(blocks), e0=e0)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [1801, 1802], e0_by_species=e0)
    e, f, v = eng.compute()
    assert np.abs(e - eo).max() < E_TOL
    assert np.abs(f - fo).max() < F_TOL
    assert np.abs(v - vo).max() < V_TOL * np.abs(vo).max()
    # MD steps stay on the oracle's trajectory over a few steps
    vel = synth.maxwell_velocities(st.masses, 600.0, 87)
    eng.set_state(st.positions, vel)
    eng.md(5, 1.0)
    pos, _, frc = eng.get_state()
    eo2, fo2, _, _ = O.evaluate(pos, st.species, st.box, list(blocks), e0=e0)
    e2, f2, _ = eng.compute()
    assert np.abs(e2 - eo2).max() < E_TOL and np.abs(f2 - fo2).max() < F_TOL
    # the mixed form on compressed rows (the MLP input is the padded row): with a
    # gate of 0 every site goes back to the exact kernel
    m = gpu.Mlp(bC.hypers.device_dim, 128, 2, seed=3)
    gpu.engine_set_mlp(eng, 0, m, gate_ev=0.0)
    eg, fg, _ = eng.compute()
    assert gpu.engine_mlp_stats(eng, 0)[0] == int(np.sum(st.species == 1))
    assert np.abs(eg - e2).max() < 1e-9 and np.abs(fg - f2).max() < 1e-9
    gpu.engine_set_mlp(eng, 0, None)
    eng.close()
    m.close()


def test_batch(gpu, blocks):
    cells = [synth.random_structure(n, (n / 0.12) ** (1 / 3), 1.0, seed=880 + n, h_fraction=0.25)
             for n in (60, 150, 400)]
    bat = gpu.Batch(cells, [1801, 1802])
    e, f, v = bat.compute()
    off = 0
    for s, st in enumerate(cells):
        eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, list(blocks))
        sl = slice(off, off + st.n)
        assert np.max(np.abs(e[sl] - eo)) < E_TOL, s
        assert np.max(np.abs(f[sl] - fo)) < F_TOL, s
        assert np.max(np.abs(v[s] - vo)) < V_TOL * max(1.0, np.max(np.abs(vo))), s
        off += st.n
    bat.close()


def test_key_reuse_with_another_shape(gpu, blocks):
    """A begin under a cached key with another descriptor shape makes a new
    block (the cache holds only for the same shape), and engines made on the
    old block keep working."""
    bC, _ = blocks
    plain = sparse_block(ch_hypers(1), 300, seed=89, n_atoms=300, L=L, d_min=1.0,
                         h_fraction=0.25, n_structs=2)
    st = synth.random_structure(300, L, 1.0, seed=90, h_fraction=0.25)
    gpu.soap_backend_begin(plain, key=1803)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [1803])
    e_old, _, _ = eng.compute()
    gpu.soap_backend_begin(bC, key=1803)          # same key and n_sparse, compressed
    nl = neighbor_data(st, 3.7)
    q = gpu.get_soap(st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"], nl["xyz"],
                     st.species, st.species, bC.hypers.dim)
    qo, _, _ = oracle_descriptors(st, bC.hypers, nl)
    assert q.shape == qo.shape and np.abs(q - qo).max() < Q_TOL
    e_again, _, _ = eng.compute()                 # the engine still has the plain block
    assert np.array_equal(e_again, e_old)
    eng.close()



def test_repeated_entries_add(gpu):
    """A transformation with an entry split in two gives the descriptors of the
    one with the summed weight (entries add, in both CSR copies on the device)."""
    full = ch_hypers(1)
    rng = np.random.default_rng(91)
    # the first 80 components (n = 0 with every n', all l: the large ones) in
    # pairs with positive weights, so that |v| is of the size of |p| and the 1e-7
    # descriptor bar applies as for the power spectrum itself (a few random
    # small components would make |v| small and magnify the fp32 error of c)
    base = SoapCompression(40, np.repeat(np.arange(1, 41), 2), rng.permutation(80) + 1,
                           rng.uniform(0.2, 1.0, size=80))
    split = SoapCompression(base.dim, np.concatenate([base.P_i, base.P_i[:7]]),
                            np.concatenate([base.P_j, base.P_j[:7]]),
                            np.concatenate([base.P_el, base.P_el[:7] * 0.75]))
    split.P_el[:7] = base.P_el[:7] * 0.25
    st = synth.random_structure(300, L, 1.0, seed=92, h_fraction=0.25)
    nl = neighbor_data(st, 3.7)
    out = []
    for key, comp in ((1804, base), (1805, split)):
        h = ch_hypers(1)
        h.compress = comp
        b = sparse_block(h, 100, seed=93, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                         n_structs=1)
        gpu.soap_backend_begin(b, key=key)
        out.append(gpu.get_soap(st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"], nl["xyz"],
                                st.species, st.species, h.dim))
    h = ch_hypers(1)
    h.compress = base
    qo, _, _ = oracle_descriptors(st, h, nl)
    assert np.abs(out[0] - out[1]).max() < 1e-7
    assert np.abs(out[0] - qo).max() < Q_TOL and np.abs(out[1] - qo).max() < Q_TOL


def test_compressed_species_multiplicity(gpu):
    """A compressed block with carbon in both descriptor species (species
    multiplicity with the compression's raw-spectrum instantiations): descriptors
    and the engine's energies, forces and virial against the oracle."""
    from test_gpu_parity import multiplicity_hypers
    h = multiplicity_hypers(central=1)
    h.compress = random_transformation(h.uncompressed_dim, 301, seed=86)
    blk = sparse_block(h, 300, seed=87, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                       n_structs=2)
    gpu.soap_backend_begin(blk, key=1804)
    st = synth.random_structure(300, L, 1.0, seed=88, h_fraction=0.25)
    nl = neighbor_data(st, h.rcut_max)
    q = gpu.get_soap(st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"], nl["xyz"],
                     st.species, st.species, h.dim)
    qo, _, _ = oracle_descriptors(st, h, nl)
    assert np.abs(q - qo).max() < Q_TOL
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, [blk])
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [1804])
    e, f, v = eng.compute()
    assert np.abs(e - eo).max() < E_TOL
    assert np.abs(f - fo).max() < F_TOL
    assert np.abs(v - vo).max() < V_TOL * np.abs(vo).max()
    eng.close()
