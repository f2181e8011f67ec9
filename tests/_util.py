"""Shared helpers of the test-suite: structures, neighbour data and sparse sets
built with the FP64 oracle (the checker)."""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from turbogap_b200.hypers import GapBlock, SoapTurboHypers  # noqa: E402
from turbogap_b200.synth import Structure, random_structure  # noqa: E402


def neighbor_data(st: Structure, rcut: float):
    """Supercell + build_neighbors_list exactly as the reference driver does."""
    a, b, c = st.box
    ind = O.number_of_unit_cells(a, b, c, rcut)
    pos_sc, sp_sc = O.make_supercell(st.positions, st.species, a, b, c, ind)
    A, B, Cc = a * ind[0], b * ind[1], c * ind[2]
    nl = O.build_neighbors_list(pos_sc, st.n, A, B, Cc, rcut, ind, sp_sc)
    nl.update(indices=ind, pos_sc=pos_sc, sp_sc=sp_sc, box_sc=np.array([A, B, Cc]))
    return nl


def oracle_descriptors(st: Structure, h: SoapTurboHypers, nl=None):
    """q (n_central, dim) of the block's central atoms, |p| and the central atom ids."""
    if nl is None:
        nl = neighbor_data(st, h.rcut_max)
    n = st.n
    zfirst = {z: s + 1 for s, z in reversed(list(enumerate(h.species_z)))}
    starts = np.concatenate([[0], np.cumsum(nl["n_neigh"])])
    sites, nn, rjs, xyz, mask = [], [], [], [], []
    for i in range(n):
        if not (h.central_species == 0 or zfirst.get(int(st.species[i]), 0) == h.central_species):
            continue
        sites.append(i)
        cnt = 0
        for k in range(starts[i], starts[i + 1]):
            j = (nl["neighbors_list"][k] - 1) % n
            z = int(st.species[j])
            if nl["rjs"][k] < h.rcut_max and z in zfirst:
                cnt += 1
                rjs.append(nl["rjs"][k])
                xyz.append(nl["xyz"][k])
                mask.append([int(z == zz) for zz in h.species_z])
        nn.append(cnt)
    hc = O.HypersC(h)
    q, _, sdp = O.get_soap(hc, np.array(nn, np.int32), np.array(mask, np.int32),
                           np.array(rjs), np.array(xyz).reshape(-1, 3), derivatives=False)
    return q, sdp, np.array(sites)


def sparse_block(h: SoapTurboHypers, n_sparse: int, seed: int, n_atoms=216, L=12.91,
                 d_min=1.2, h_fraction=0.0, delta=1.0, zeta=4.0, sigma_alpha=0.01,
                 n_structs=None):
    """Sparse set of q vectors of random central atoms from seeded structures."""
    rng = np.random.default_rng(seed)
    qs = []
    i = 0
    while sum(len(x) for x in qs) < n_sparse * 2 and (n_structs is None or i < n_structs):
        st = random_structure(n_atoms, L, d_min, seed=seed * 100 + i, h_fraction=h_fraction)
        q, _, _ = oracle_descriptors(st, h)
        qs.append(q)
        i += 1
    Q = np.concatenate(qs)
    pick = rng.choice(len(Q), size=n_sparse, replace=False)
    alphas = rng.normal(0.0, sigma_alpha, size=n_sparse)
    return GapBlock(h, Q[pick], alphas, delta=delta, zeta=zeta)


def make_families(seed=0, rcut2=4.0, rcut3=3.2):
    """Seeded distance_2b (C-H), angle_3b (C centre, exp; H centre, pol) and
    core_pot (C-C) families on species C = 1, H = 2, with sparse points spread
    over the ranges their descriptors take in the C/H test structures."""
    from turbogap_b200 import families as FM
    rng = np.random.default_rng(seed)
    n2 = 24
    f2 = FM.Distance2b((1, 2), 0.6, 0.5, rcut2, rng.uniform(0.9, rcut2, n2),
                       rng.normal(0, 0.05, n2), rng.uniform(0.5, 1.0, n2))
    def sparse3(n):
        r1 = rng.uniform(1.0, rcut3, n)
        r2 = rng.uniform(1.0, rcut3, n)
        return np.stack([r1 + r2, (r1 - r2) ** 2, rng.uniform(1.0, r1 + r2)], axis=1)
    n3 = 40
    f3e = FM.Angle3b((1, 1, 2), 0.3, [1.5, 2.0, 1.2], rcut3, sparse3(n3), rng.normal(0, 0.05, n3),
                     rng.uniform(0.5, 1.0, n3), "exp")
    f3p = FM.Angle3b((2, 1, 1), 0.2, [4.0, 4.0, 4.0], rcut3, sparse3(n3), rng.normal(0, 0.05, n3),
                     rng.uniform(0.5, 1.0, n3), "pol")
    x = np.linspace(0.6, 2.6, 21)
    fc = FM.CorePot.from_table((1, 1), x, 3.0 * np.exp(-2.0 * x) / x, 1e50, 0.0,
                               cutoff=2.6, buffer=0.5)
    return [f2, f3e, f3p, fc]
