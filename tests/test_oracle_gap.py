"""The oracle's GAP prediction and get_gap_soap remap against independent numpy
restatements of src/gap.f90:66-259 and src/gap_interface.f90:178-431."""
import numpy as np
import pytest

from _util import O, neighbor_data, sparse_block
from turbogap_b200.hypers import ch_hypers
from turbogap_b200.synth import random_structure


def numpy_gap(soap, soap_der, Qs, alphas, delta, zeta0, e0, n_neigh, nl, xyz, n_sites0):
    """gap.f90:66-259 in numpy (FP64): dgemm('t','n'), K^zeta, dgemm('n','t'), pair loop."""
    zeta = float(int(zeta0)) if abs(zeta0 - int(zeta0)) < 1e-5 else zeta0
    K = soap @ Qs.T
    e = delta ** 2 * (K ** zeta) @ alphas + e0
    Qss = -zeta * delta ** 2 * ((K ** (zeta - 1)) * alphas) @ Qs
    f = np.zeros((n_sites0, 3))
    vir = np.zeros((3, 3))
    l = 0
    for i in range(soap.shape[0]):
        for _ in range(n_neigh[i]):
            this = soap_der[l].T @ Qss[i]
            f[(nl[l] - 1) % n_sites0] += this
            vir += 0.5 * (np.outer(this, xyz[l]) + np.outer(xyz[l], this))
            l += 1
    return e, f, vir


@pytest.mark.parametrize("zeta", [4.0, 4.000003, 2.5])
def test_energy_and_forces_match_numpy_restatement(zeta):
    rng = np.random.default_rng(5)
    n, D, M = 12, 40, 30
    nn = rng.integers(1, 6, size=n).astype(np.int32)
    P = int(nn.sum())
    soap = np.abs(rng.normal(size=(n, D)))
    soap /= np.linalg.norm(soap, axis=1)[:, None]
    der = rng.normal(size=(P, D, 3))
    Qs = np.abs(rng.normal(size=(M, D)))
    Qs /= np.linalg.norm(Qs, axis=1)[:, None]
    al = rng.normal(0, 0.01, size=M)
    nl = rng.integers(1, 3 * n, size=P).astype(np.int32)
    xyz = rng.normal(size=(P, 3))
    e, f, v = O.soap_energy_and_forces(soap, der, Qs, al, 1.3, zeta, 0.2, nn, nl, xyz, n)
    e2, f2, v2 = numpy_gap(soap, der, Qs, al, 1.3, zeta, 0.2, nn, nl, xyz, n)
    assert np.allclose(e, e2, rtol=1e-13, atol=1e-14)
    assert np.allclose(f, f2, rtol=1e-12, atol=1e-13)
    assert np.allclose(v, v2, rtol=1e-12, atol=1e-13)


def test_get_gap_soap_central_filter_and_assignment():
    """Only central-species sites get energies; only atoms the block sees get forces;
    everything else in energies0/forces0 is left untouched (assignment, not addition)."""
    L = (120 / 0.12) ** (1 / 3)
    st = random_structure(120, L, 1.0, seed=31, h_fraction=0.25)
    bC = sparse_block(ch_hypers(1), 50, seed=32, n_atoms=120, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=2)
    nl = neighbor_data(st, 3.7)
    hc = O.HypersC(bC.hypers)
    e, f, v = O.get_gap_soap(hc, st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"], nl["xyz"],
                             st.species, st.species, bC.Qs, bC.alphas, bC.delta, bC.zeta)
    is_c = st.species == 1
    assert np.all(e[~is_c] == 0.0) and np.all(e[is_c] != 0.0)
    # every atom within rcut of a carbon is seen, so all of them carry a force here
    assert np.count_nonzero(np.abs(f).sum(1)) == st.n
    # block energies + e0 of the full evaluation with both blocks = sum of the blocks
    bH = sparse_block(ch_hypers(2), 40, seed=33, n_atoms=120, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=2)
    eH, fH, vH = O.get_gap_soap(O.HypersC(bH.hypers), st.n, nl["n_neigh"], nl["neighbors_list"],
                                nl["rjs"], nl["xyz"], st.species, st.species, bH.Qs, bH.alphas,
                                bH.delta, bH.zeta)
    e0 = np.array([-1.0, -0.5])
    et, ft, vt, _ = O.evaluate(st.positions, st.species, st.box, [bC, bH], e0=e0)
    assert np.allclose(et, e + eH + e0[st.species - 1], atol=1e-13)
    assert np.allclose(ft, f + fH, atol=1e-12)
    assert np.allclose(vt, v + vH, atol=1e-12)


def test_memory_budget_batches_only_change_summation_order():
    """get_number_of_atom_pairs batches: same energies/forces to round-off."""
    st = random_structure(120, 10.5, 1.2, seed=34)
    blk = sparse_block(ch_hypers(0).__class__(species_z=[1], alpha_max=[8]), 60, seed=35,
                       n_atoms=120, L=10.5, n_structs=1)
    e1, f1, v1, _ = O.evaluate(st.positions, st.species, st.box, [blk], max_gbytes=10.0)
    e2, f2, v2, _ = O.evaluate(st.positions, st.species, st.box, [blk], max_gbytes=0.005)
    nl = neighbor_data(st, 3.7)
    h = blk.hypers
    ib, _, _, _ = O.atom_pair_batches(nl["n_neigh"], nl["rjs"], 3.7, h.l_max, h.n_max, h.dim,
                                      h.n_species, 0.005)
    assert len(ib) > 3
    assert np.allclose(e1, e2, atol=1e-13)
    assert np.allclose(f1, f2, atol=1e-12)
    assert np.allclose(v1, v2, atol=1e-11)
