"""GPU parity at the benchmarked hyperparameters, against the FP64 oracle.

The bf16x3 GAP GEMMs (gap.f90:137-138, K = q.Q_s^T; gap.f90:184-185, dE/dq)
carry a rounding error that grows with the sparse-set size M and the descriptor
length D, so the plain form's bound is checked where the benchmarks run:

  * two soap_turbo blocks (C and H centres, n_max 8+8, l_max 8: D = 1224) with
    M = 4000 sparse points each, on a whole 300-atom C/H cell and on one MPI
    rank's share of the 32,768-atom C/H benchmark structure (0.12 atoms/A^3);
  * one C block (D = 324) with M = 2000 sparse points, on uneven C cells of the
    batched workload (64-2048 atoms, 1.5-3.5 g/cm3) through the batch engine.

Bounds (plain form): 1e-6 eV/atom and 1e-6 eV/A (max abs). The virial is an
extensive energy: its bound is the per-atom energy bound, max |dW_ab| / N <=
1e-6 eV/atom. (Relative to its largest component the virial error at M = 4000
is about 2e-6; at M <= 1000 it stays under 1e-6, which the other parity tests
check.)
"""
import numpy as np
import pytest

from _util import O, sparse_block
from turbogap_b200 import synth
from turbogap_b200.hypers import carbon_hypers, ch_hypers
from turbogap_b200.synth import random_structure

pytestmark = pytest.mark.gpu

E_TOL = 1e-6     # eV/atom
F_TOL = 1e-6     # eV/A
W_TOL = 1e-6     # eV/atom: max |dW_ab| / N

L2048 = (2048 / 0.12) ** (1 / 3)
L300 = (300 / 0.12) ** (1 / 3)


@pytest.fixture(scope="module")
def ch_m4000(gpu):
    """C- and H-centred blocks with 4000 sparse points each, drawn from the
    oracle's descriptors of seeded 2048-atom C/H cells of the benchmark's kind."""
    bC = sparse_block(ch_hypers(1), 4000, seed=41, n_atoms=2048, L=L2048, d_min=1.0,
                      h_fraction=0.25)
    bH = sparse_block(ch_hypers(2), 4000, seed=42, n_atoms=2048, L=L2048, d_min=1.0,
                      h_fraction=0.25)
    assert bC.Qs.shape == (4000, 1224) and bH.Qs.shape == (4000, 1224)
    gpu.soap_backend_begin(bC, key=601)
    gpu.soap_backend_begin(bH, key=602)
    return bC, bH


def _check(e, f, v, eo, fo, vo, n_sites=None):
    n = n_sites or len(e)   # the central sites the virial sums over
    de, df = np.abs(e - eo).max(), np.abs(f - fo).max()
    dw = np.abs(v - vo).max() / n
    rel = np.abs(v - vo).max() / np.abs(vo).max()
    print(f"max dE {de:.2e} eV/atom, max dF {df:.2e} eV/A, virial {dw:.2e} eV/atom "
          f"({rel:.2e} of its largest component)")
    assert de < E_TOL, de
    assert df < F_TOL, df
    assert dw < W_TOL, (dw, rel)
    return de, df, dw


def test_ch_m4000_whole_cell(gpu, ch_m4000):
    st = random_structure(300, L300, 1.0, seed=43, h_fraction=0.25)
    e0 = np.array([-0.5, -0.25])
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, list(ch_m4000), e0=e0)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [601, 602], e0_by_species=e0)
    e, f, v = eng.compute()
    eng.close()
    _check(e, f, v, eo, fo, vo)


def test_ch_m4000_benchmark_structure_share(gpu, ch_m4000):
    """One rank's share (central sites 0..383) of the 32,768-atom benchmark
    structure: the engine's site range against the oracle's."""
    st = synth.workload_structure("ch32k")
    share = (0, 384)
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, list(ch_m4000),
                               site_range=share)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [601, 602])
    eng.set_site_range(*share)
    e, f, v = eng.compute()
    eng.close()
    assert np.count_nonzero(e) == share[1] - share[0]
    _check(e, f, v, eo, fo, vo, n_sites=share[1] - share[0])


def test_ch_m4000_after_md(gpu, ch_m4000):
    """The same bound after 10 NVE steps of the device engine: the oracle
    evaluates the engine's own positions."""
    st = random_structure(300, L300, 1.0, seed=44, h_fraction=0.25)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [601, 602])
    eng.set_state(st.positions, synth.maxwell_velocities(st.masses, 1000.0, 45))
    eng.md(10, 0.5)
    p, _, _ = eng.get_state()
    e, f, v = eng.compute()
    eng.close()
    eo, fo, vo, _ = O.evaluate(p, st.species, st.box, list(ch_m4000))
    _check(e, f, v, eo, fo, vo)


@pytest.fixture(scope="module")
def carbon_m2000(gpu):
    """A C block with 2000 sparse points from seeded C cells at 2.0-3.0 g/cm3."""
    h = carbon_hypers()
    qs = []
    for i, rho in enumerate((2.0, 2.5, 3.0)):
        n = 1000
        L = (n / synth.carbon_number_density(rho)) ** (1 / 3)
        st = random_structure(n, L, 1.2, seed=4700 + i)
        from _util import oracle_descriptors
        qs.append(oracle_descriptors(st, h)[0])
    Q = np.concatenate(qs)
    rng = np.random.default_rng(47)
    pick = rng.choice(len(Q), size=2000, replace=False)
    from turbogap_b200.hypers import GapBlock
    blk = GapBlock(h, Q[pick], rng.normal(0.0, 0.01, 2000), delta=1.0, zeta=4.0)
    gpu.soap_backend_begin(blk, key=611)
    return blk


def test_batched_cells_m2000(gpu, carbon_m2000):
    """Uneven cells of the batched workload, M = 2000: per-cell energies,
    forces and virials of the batch engine against the oracle, cell by cell
    (a small box among them takes the supercell path)."""
    sizes = synth.cells512_sizes()
    # the smallest cell, a mid-sized one and the largest of the first 64
    idx = [int(np.argmin(sizes)), int(np.argsort(sizes[:64])[32]), int(np.argmax(sizes[:64]))]
    cells = [synth.workload_structure("cells512", sub=i) for i in idx]
    bat = gpu.Batch(cells, [611])
    E, F, V = bat.compute()
    bat.close()
    off = 0
    for k, st in enumerate(cells):
        eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, [carbon_m2000])
        _check(E[off:off + st.n], F[off:off + st.n], V[k], eo, fo, vo)
        off += st.n
