"""Local-property prediction (local_properties.f90:174-294, the Hirshfeld-volume
and dipole predictors' model) on the GPU against the oracle: per-site values
with the V0 offset and the clamp at zero, and dV_i/dr_j for every pair of the
caller's lists."""
from __future__ import annotations

import numpy as np
import pytest

from _util import O, neighbor_data, sparse_block
from turbogap_b200.hypers import SoapCompression, carbon_hypers
from turbogap_b200.synth import random_structure

pytestmark = pytest.mark.gpu


def _kept(st, h, nl):
    """The block's kept pairs per site (self first), with their global indices."""
    starts = np.concatenate([[0], np.cumsum(nl["n_neigh"])])
    nn, idx = [], []
    for i in range(st.n):
        c = 0
        for k in range(starts[i], starts[i + 1]):
            if nl["rjs"][k] < h.rcut_max:
                idx.append(k)
                c += 1
        nn.append(c)
    return np.array(nn, np.int32), np.array(idx)


def _transformation(full_dim, dim, seed):
    rng = np.random.default_rng(seed)
    P_i = np.concatenate([np.arange(1, dim + 1), rng.integers(1, dim + 1, size=dim)])
    P_j = rng.integers(1, full_dim + 1, size=2 * dim)
    return SoapCompression(dim, P_i, P_j, rng.uniform(0.2, 1.0, size=2 * dim))


@pytest.mark.parametrize("compressed", [False, True])
@pytest.mark.parametrize("offset", ["none", "median"])
def test_local_property_matches_oracle(gpu, offset, compressed):
    """compressed: the property's block under a 45-row P_transformation."""
    h = carbon_hypers()
    if compressed:
        h.compress = _transformation(h.uncompressed_dim, 45, seed=93)
    blk = sparse_block(h, 250, seed=91, sigma_alpha=0.002)
    gpu.soap_backend_begin(blk, key=903 if compressed else 901)
    st = random_structure(216, 12.91, 1.2, seed=92)
    nl = neighbor_data(st, h.rcut_max + 0.4)      # lists longer than the block's cutoff
    nn, idx = _kept(st, h, nl)
    q, sder, _ = O.get_soap(O.HypersC(h), nn, np.ones((len(idx), 1), np.int32), nl["rjs"][idx],
                            nl["xyz"][idx], derivatives=True)
    v0 = 0.0
    if offset == "median":   # half of the sites fall below zero and are clamped
        v0 = -float(np.median(O.local_property_predict(q, blk.Qs, blk.alphas, 0.0, blk.delta,
                                                       blk.zeta, sder, nn)[0]))
    vals, der = gpu.get_local_property(st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"],
                                       nl["xyz"], st.species, st.species, v0=v0)
    Vo, Do = O.local_property_predict(q, blk.Qs, blk.alphas, v0, blk.delta, blk.zeta, sder, nn)
    assert vals.shape == (st.n,)
    assert (Vo > 0.0).any()
    if offset == "median":
        assert (Vo == 0.0).sum() > st.n // 4              # the clamp and its zero derivatives
    assert np.abs(vals - Vo).max() < 1e-7
    full = np.zeros((len(nl["rjs"]), 3))
    full[idx] = Do
    assert np.abs(der - full).max() < 1e-6 * max(1.0, np.abs(full).max())
    # pairs beyond the block's cutoff carry nothing
    far = np.setdiff1d(np.arange(len(nl["rjs"])), idx)
    assert len(far) > 0 and not der[far].any()


def test_local_property_species_multiplicity(gpu):
    """A property block with carbon in both descriptor species (species
    multiplicity 2): each pair's dV/dr adds both species' terms."""
    from test_gpu_parity import multiplicity_hypers
    h = multiplicity_hypers()
    blk = sparse_block(h, 200, seed=97, sigma_alpha=0.002, n_structs=2)
    gpu.soap_backend_begin(blk, key=905)
    st = random_structure(216, 12.91, 1.2, seed=98)
    nl = neighbor_data(st, h.rcut_max)
    nn, idx = _kept(st, h, nl)
    q, sder, _ = O.get_soap(O.HypersC(h), nn, np.ones((len(idx), 2), np.int32), nl["rjs"][idx],
                            nl["xyz"][idx], derivatives=True)
    vals, der = gpu.get_local_property(st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"],
                                       nl["xyz"], st.species, st.species, v0=0.0)
    Vo, Do = O.local_property_predict(q, blk.Qs, blk.alphas, 0.0, blk.delta, blk.zeta, sder, nn)
    assert np.abs(vals - Vo).max() < 1e-7
    full = np.zeros((len(nl["rjs"]), 3))
    full[idx] = Do
    assert np.abs(der - full).max() < 1e-6 * max(1.0, np.abs(full).max())


@pytest.mark.parametrize("zeta", [4.0, 2.5])
def test_soap_dipole_matches_oracle(gpu, zeta):
    """get_soap_dipole (gap.f90:261-398): the self pair's gradient of a dipole
    GAP's fictitious local energy, mu_i = dE_i/dr_i, and E_i itself (no e0, no
    clamp), against the oracle's restatement on the materialised derivatives."""
    from turbogap_b200.hypers import GapBlock
    h = carbon_hypers()
    base = sparse_block(h, 200, seed=95, sigma_alpha=0.01)
    blk = GapBlock(h, base.Qs, base.alphas, delta=0.7, zeta=zeta)
    gpu.soap_backend_begin(blk, key=905 if zeta == 4.0 else 906)
    st = random_structure(216, 12.91, 1.2, seed=96)
    nl = neighbor_data(st, h.rcut_max + 0.3)
    nn, idx = _kept(st, h, nl)
    q, sder, _ = O.get_soap(O.HypersC(h), nn, np.ones((len(idx), 1), np.int32), nl["rjs"][idx],
                            nl["xyz"][idx], derivatives=True)
    mu, en = gpu.get_soap_dipole(st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"], nl["xyz"],
                                 st.species, st.species)
    mo, eo = O.soap_dipole(q, sder, blk.Qs, blk.alphas, blk.delta, blk.zeta, nn)
    assert mu.shape == (st.n, 3) and en.shape == (st.n,)
    assert np.abs(en - eo).max() < 1e-7
    assert np.abs(mu - mo).max() < 1e-6 * max(1.0, np.abs(mo).max())
    # the total dipole
    assert np.abs(mu.sum(0) - mo.sum(0)).max() < 1e-5 * max(1.0, np.abs(mo).max())
