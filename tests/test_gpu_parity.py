"""GPU parity: the CUDA backend, called through the C-ABI, against the FP64 oracle.

Tolerances (the plain bf16x3 form): neighbour indices, rjs and xyz bit-exact;
energies 1e-6 eV/atom and forces 1e-6 eV/A (max abs); virial 1e-6 relative to
its largest component; descriptor components 1e-7 (max abs). The mixed form
(single bf16 products) is held to 1 meV/atom and 30 meV/A.
"""
import numpy as np
import pytest

from _util import O, neighbor_data, oracle_descriptors, sparse_block
from turbogap_b200.hypers import SoapTurboHypers, carbon_hypers, ch_hypers
from turbogap_b200.synth import maxwell_velocities, random_structure

pytestmark = pytest.mark.gpu

E_TOL = 1e-6     # eV/atom
F_TOL = 1e-6     # eV/A
V_TOL = 1e-6     # relative
Q_TOL = 1e-7


def _bf16(x):
    u = np.asarray(x, np.float32).view(np.uint32)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


def _f32(u):
    return (u.astype(np.uint32) << 16).view(np.float32)


# the last two: more tiles than SMs with a short last column tile, where the
# waves rotate the column tiles over the CTAs
@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (257, 516, 192), (1000, 700, 640),
                                   (33, 1224, 3712), (10240, 324, 128), (7680, 700, 192)])
def test_tcgen05_gemm(gpu, M, N, K):
    rng = np.random.default_rng(M + N + K)
    A = _bf16(rng.normal(size=(M, K)))
    B = _bf16(rng.normal(size=(N, K)))
    C = gpu.gemm_bf16_tn(A, B)
    ref = _f32(A).astype(np.float64) @ _f32(B).astype(np.float64).T
    # fp32 accumulation over K terms of size ~1
    assert np.abs(C - ref).max() < 4e-6 * np.sqrt(K) * 8


CASES = [
    ("cells_3", lambda: random_structure(216, 12.91, 1.2, seed=1000)),
    ("cells_2", lambda: random_structure(40, 8.0, 1.2, seed=3)),
    ("supercell", lambda: random_structure(30, 6.0, 1.2, seed=4)),
    ("two_species", lambda: random_structure(300, (300 / 0.12) ** (1 / 3), 1.0, seed=11,
                                             h_fraction=0.25)),
    # 4 cells per axis of 13 atoms each: a 27-cell neighbourhood of about 350
    # candidates, more than the search stages at once (256), so it runs in rounds
    ("dense_rounds", lambda: random_structure(850, 15.0, 1.0, seed=12)),
]


@pytest.mark.parametrize("name,make", CASES)
def test_neighbor_list_bit_exact(gpu, name, make):
    st = make()
    ref = neighbor_data(st, 3.7)
    box = ref["box_sc"]
    g = gpu.build_neighbors_list(ref["pos_sc"], st.n, box[0], box[1], box[2], 3.7, ref["indices"],
                                 ref["sp_sc"])
    for k in ("n_neigh", "neighbors_list", "neighbor_species"):
        assert np.array_equal(ref[k], g[k]), k
    # FP64 geometry restated with the reference's rounding: identical bits
    assert np.array_equal(ref["rjs"].view(np.uint64), g["rjs"].view(np.uint64))
    assert np.array_equal(ref["xyz"].view(np.uint64), g["xyz"].view(np.uint64))
    # acos/atan2 of the device math library: a few ulp
    assert np.abs(ref["thetas"] - g["thetas"]).max() < 1e-14
    assert np.abs(ref["phis"] - g["phis"]).max() < 1e-14


def test_neighbor_list_do_list_and_capacity(gpu):
    st = random_structure(216, 12.91, 1.2, seed=1000)
    ref = neighbor_data(st, 3.7)
    dl = (np.arange(st.n) % 3 == 0).astype(np.int32)
    box = ref["box_sc"]
    orc = O.build_neighbors_list(ref["pos_sc"], st.n, box[0], box[1], box[2], 3.7,
                                 ref["indices"], ref["sp_sc"], dl)
    g = gpu.build_neighbors_list(ref["pos_sc"], st.n, box[0], box[1], box[2], 3.7,
                                 ref["indices"], ref["sp_sc"], do_list=dl, cap=16)
    assert np.array_equal(orc["n_neigh"], g["n_neigh"])
    assert np.array_equal(orc["neighbors_list"], g["neighbors_list"])


@pytest.fixture(scope="module")
def carbon_block(gpu):
    h = carbon_hypers()
    # 1000 sparse points from 5 further seeded 216-atom cells (carbon216 workload)
    return sparse_block(h, 1000, seed=17, n_structs=5)


def test_descriptor_parity(gpu, carbon_block):
    st = random_structure(216, 12.91, 1.2, seed=1000)
    h = carbon_block.hypers
    gpu.soap_backend_begin(carbon_block, key=101)
    nl = neighbor_data(st, h.rcut_max)
    q = gpu.get_soap(st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"], nl["xyz"], st.species,
                     st.species, h.dim)
    qo, _, _ = oracle_descriptors(st, h, nl)
    assert q.shape == qo.shape
    assert np.abs(q - qo).max() < Q_TOL
    assert np.allclose(np.linalg.norm(q, axis=1), 1.0, atol=1e-6)


def test_gap_soap_parity_carbon216(gpu, carbon_block):
    """carbon216: energies/forces/virial of get_gap_soap vs the oracle."""
    st = random_structure(216, 12.91, 1.2, seed=1000)
    h = carbon_block.hypers
    gpu.soap_backend_begin(carbon_block, key=101)
    nl = neighbor_data(st, h.rcut_max)
    e, f, v = gpu.get_gap_soap(st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"], nl["xyz"],
                               st.species, st.species)
    hc = O.HypersC(h)
    eo, fo, vo = O.get_gap_soap(hc, st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"],
                                nl["xyz"], st.species, st.species, carbon_block.Qs,
                                carbon_block.alphas, carbon_block.delta, carbon_block.zeta)
    assert np.abs(e - eo).max() < E_TOL
    assert np.abs(f - fo).max() < F_TOL
    assert np.abs(v - vo).max() < V_TOL * np.abs(vo).max()
    assert np.abs(f.sum(0)).max() < 1e-9


def test_gap_soap_batches_match_single_call(gpu, carbon_block):
    """Memory-budget batches (neighbors.f90:667-778) sum to the one-shot result."""
    st = random_structure(216, 12.91, 1.2, seed=1000)
    h = carbon_block.hypers
    gpu.soap_backend_begin(carbon_block, key=101)
    nl = neighbor_data(st, h.rcut_max)
    ib, ie, jb, je = O.atom_pair_batches(nl["n_neigh"], nl["rjs"], h.rcut_max, h.l_max, h.n_max,
                                         h.dim, h.n_species, 0.01)
    assert len(ib) > 1
    E = np.zeros(st.n)
    F = np.zeros((st.n, 3))
    V = np.zeros((3, 3))
    for a, b, c, d in zip(ib, ie, jb, je):
        e, f, v = gpu.get_gap_soap(st.n, nl["n_neigh"][a - 1:b], nl["neighbors_list"][c - 1:d],
                                   nl["rjs"][c - 1:d], nl["xyz"][c - 1:d], st.species[a - 1:b],
                                   st.species)
        E += e
        F += f
        V += v
    e1, f1, v1 = gpu.get_gap_soap(st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"],
                                  nl["xyz"], st.species, st.species)
    assert np.abs(E - e1).max() < 1e-12
    assert np.abs(F - f1).max() < 1e-9
    assert np.abs(V - v1).max() < 1e-8 * np.abs(v1).max()


@pytest.fixture(scope="module")
def ch_blocks(gpu):
    L = (300 / 0.12) ** (1 / 3)
    bC = sparse_block(ch_hypers(1), 400, seed=8, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=3)
    bH = sparse_block(ch_hypers(2), 300, seed=9, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=4)
    return bC, bH


def test_engine_parity_dense_rounds(gpu, carbon_block):
    """An engine on a structure dense enough that each cell's neighbourhood is
    staged in rounds (about 350 candidates against the 256 staged at once)."""
    st = random_structure(850, 15.0, 1.0, seed=12)
    gpu.soap_backend_begin(carbon_block, key=101)
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, [carbon_block])
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [101])
    e, f, v = eng.compute()
    assert np.abs(e - eo).max() < E_TOL
    assert np.abs(f - fo).max() < F_TOL
    assert np.abs(v - vo).max() / st.n < 1e-6   # the virial per atom (its parity bound)
    eng.close()


def test_engine_parity_two_species(gpu, ch_blocks):
    bC, bH = ch_blocks
    gpu.soap_backend_begin(bC, key=201)
    gpu.soap_backend_begin(bH, key=202)
    st = random_structure(300, (300 / 0.12) ** (1 / 3), 1.0, seed=11, h_fraction=0.25)
    e0 = np.array([-0.5, -0.25])
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, [bC, bH], e0=e0)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [201, 202], e0_by_species=e0)
    e, f, v = eng.compute()
    assert np.abs(e - eo).max() < E_TOL
    assert np.abs(f - fo).max() < F_TOL
    assert np.abs(v - vo).max() < V_TOL * np.abs(vo).max()
    eng.close()


def multiplicity_hypers(central=0):
    """Carbon (species 1) in both descriptor species of one block (species
    multiplicity 2, gap_interface.f90:180-199), each with its own cutoff,
    widths and central weight."""
    return SoapTurboHypers(species_z=[1, 1], alpha_max=[8, 8], l_max=8, rcut_hard=[3.7, 2.9],
                           buffer=[0.5, 0.4], atom_sigma_r=[0.5, 0.35], atom_sigma_t=[0.5, 0.4],
                           central_weight=[1.0, 0.6], central_species=central)


def test_descriptor_parity_species_multiplicity(gpu):
    h = multiplicity_hypers()
    blk = sparse_block(h, 200, seed=23, n_structs=2)
    gpu.soap_backend_begin(blk, key=231)
    st = random_structure(216, 12.91, 1.2, seed=1001)
    nl = neighbor_data(st, h.rcut_max)
    q = gpu.get_soap(st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"], nl["xyz"], st.species,
                     st.species, h.dim)
    qo, _, _ = oracle_descriptors(st, h, nl)
    assert np.abs(q - qo).max() < Q_TOL
    # the two descriptor species see the same atoms through different hypers
    half = h.alpha_max[0]
    assert np.abs(qo[:, : half * (half + 1) // 2]).max() > 0.0


def test_engine_parity_species_multiplicity(gpu):
    """C/H structure, a C-centred block with C in both descriptor species: H
    atoms are invisible to it; energies, forces and the virial against the oracle."""
    L = (300 / 0.12) ** (1 / 3)
    h = multiplicity_hypers(central=1)
    blk = sparse_block(h, 400, seed=24, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                       n_structs=3)
    gpu.soap_backend_begin(blk, key=232)
    st = random_structure(300, L, 1.0, seed=25, h_fraction=0.25)
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, [blk])
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [232])
    e, f, v = eng.compute()
    assert np.abs(e - eo).max() < E_TOL
    assert np.abs(f - fo).max() < F_TOL
    assert np.abs(v - vo).max() < V_TOL * np.abs(vo).max()
    assert (st.species == 2).any() and not f[st.species == 2].any()   # H is invisible to it
    # the mixed form on the multiplicity block: with a gate of 0 every site goes
    # back to the exact kernel, through the single-bf16 descriptor of the mixed form
    m = gpu.Mlp(h.device_dim, 64, 2, seed=5)
    gpu.engine_set_mlp(eng, 0, m, gate_ev=0.0)
    eg, fg, _ = eng.compute()
    assert gpu.engine_mlp_stats(eng, 0)[0] == int(np.sum(st.species == 1))
    assert np.abs(eg - e).max() < 1e-9 and np.abs(fg - f).max() < 1e-9
    gpu.engine_set_mlp(eng, 0, None)
    m.close()
    eng.close()


def test_mixed_precision_within_budget(gpu, ch_blocks):
    """Single-bf16 GEMMs (the mixed form): <= 1 meV/atom and <= 30 meV/A."""
    bC, bH = ch_blocks
    gpu.soap_backend_begin(bC, key=211, precision=gpu.TG_PREC_BF16)
    gpu.soap_backend_begin(bH, key=212, precision=gpu.TG_PREC_BF16)
    st = random_structure(300, (300 / 0.12) ** (1 / 3), 1.0, seed=12, h_fraction=0.25)
    eo, fo, _, _ = O.evaluate(st.positions, st.species, st.box, [bC, bH])
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [211, 212])
    e, f, _ = eng.compute()
    assert np.abs(e - eo).max() < 1e-3
    assert np.sqrt(((f - fo) ** 2).mean()) < 30e-3
    eng.close()


def test_velocity_verlet_bit_exact(gpu):
    rng = np.random.default_rng(3)
    n = 500
    args = [rng.normal(size=(n, 3)) for _ in range(5)]
    m = rng.uniform(1, 20, size=n)
    for first in (1, 0):
        a = [x.copy() for x in args]
        b = [x.copy() for x in args]
        O.velocity_verlet(a[0], a[1], a[2], a[3], a[4], m, 0.7, 0.5, first)
        gpu.velocity_verlet(b[0], b[1], b[2], b[3], b[4], m, 0.7, 0.5, first)
        for x, y in zip(a, b):
            assert np.array_equal(x.view(np.uint64), y.view(np.uint64))


def test_engine_nve_energy_conservation(gpu, ch_blocks):
    bC, bH = ch_blocks
    gpu.soap_backend_begin(bC, key=201)
    gpu.soap_backend_begin(bH, key=202)
    st = random_structure(300, (300 / 0.12) ** (1 / 3), 1.0, seed=11, h_fraction=0.25)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [201, 202])
    eng.set_state(st.positions, maxwell_velocities(st.masses, 300.0, 5))
    ep0, ek0 = eng.md(1, 0.5)
    ep1, ek1 = eng.md(300, 0.5)
    assert abs((ep1 + ek1) - (ep0 + ek0)) / st.n < 1e-5
    assert ek1 > 0
    eng.close()


@pytest.mark.parametrize("slots", ["0", "8"])
def test_engine_list_builds_agree(gpu, ch_blocks, monkeypatch, slots):
    """The engine's one-pass list build (pairs counted into fixed rows, then
    compacted) against the two-pass build (TGB_NL_SLOTS=0) and against rows too
    short for every site (8, each build falls back to the filling search): the
    same energies, forces and virial, also over MD steps."""
    bC, bH = ch_blocks
    gpu.soap_backend_begin(bC, key=201)
    gpu.soap_backend_begin(bH, key=202)
    st = random_structure(300, (300 / 0.12) ** (1 / 3), 1.0, seed=13, h_fraction=0.25)
    vel = maxwell_velocities(st.masses, 600.0, 14)
    out = []
    for env in (None, slots):
        if env is not None:
            monkeypatch.setenv("TGB_NL_SLOTS", env)
        eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [201, 202])
        e, f, v = eng.compute()
        eng.set_state(st.positions, vel)
        eng.md(3, 1.0)
        p, _, f2 = eng.get_state()
        out.append((e, f, v, p, f2))
        eng.close()
    (e1, f1, v1, p1, g1), (e2, f2, v2, p2, g2) = out
    assert np.abs(e1 - e2).max() < 1e-12 and np.abs(f1 - f2).max() < 1e-12
    assert np.abs(v1 - v2).max() < 1e-12
    assert np.abs(p1 - p2).max() < 1e-12 and np.abs(g1 - g2).max() < 1e-10


def test_engine_parity_real_zeta(gpu, carbon_block):
    """A non-integer zeta (gap.f90:115-121 keeps it real beyond 1e-5 of an
    integer): the real-power epilogue, whose padding columns must add nothing."""
    from turbogap_b200.hypers import GapBlock
    blk = GapBlock(carbon_block.hypers, carbon_block.Qs, carbon_block.alphas, delta=1.0, zeta=2.5)
    gpu.soap_backend_begin(blk, key=111)
    st = random_structure(216, 12.91, 1.2, seed=1000)
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, [blk])
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [111])
    e, f, v = eng.compute()
    eng.close()
    assert np.all(np.isfinite(eo))
    assert np.abs(e - eo).max() < E_TOL
    assert np.abs(f - fo).max() < F_TOL
    assert np.abs(v - vo).max() < V_TOL * np.abs(vo).max()
