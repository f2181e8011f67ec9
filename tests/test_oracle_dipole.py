"""The oracle's get_soap_dipole (gap.f90:261-398) against its definition: the
local dipole mu_i is the derivative of the site's fictitious energy E_i with
respect to the central atom's own position (central differences, h = 1e-4 A),
and E_i carries no e0 and no clamp."""
import numpy as np

from _util import O, neighbor_data, sparse_block
from turbogap_b200.hypers import carbon_hypers
from turbogap_b200.synth import Structure, random_structure


def _site_data(st, h):
    nl = neighbor_data(st, h.rcut_max)
    starts = np.concatenate([[0], np.cumsum(nl["n_neigh"])])
    nn, idx = [], []
    for i in range(st.n):
        c = 0
        for k in range(starts[i], starts[i + 1]):
            if nl["rjs"][k] < h.rcut_max:
                idx.append(k)
                c += 1
        nn.append(c)
    idx = np.array(idx)
    return np.array(nn, np.int32), nl["rjs"][idx], nl["xyz"][idx]


def test_dipole_is_the_self_gradient_of_the_site_energy():
    h = carbon_hypers()
    blk = sparse_block(h, 50, seed=95, n_structs=1)
    st = random_structure(64, 8.5, 1.2, seed=96)
    hc = O.HypersC(h)
    nn, rjs, xyz = _site_data(st, h)
    q, sder, _ = O.get_soap(hc, nn, np.ones((len(rjs), 1), np.int32), rjs, xyz)
    mu, en = O.soap_dipole(q, sder, blk.Qs, blk.alphas, 0.8, 4.0, nn)

    def site_energies(pos):
        s2 = Structure(pos, st.species, st.box)
        n2, r2, x2 = _site_data(s2, h)
        q2, _, _ = O.get_soap(hc, n2, np.ones((len(r2), 1), np.int32), r2, x2, derivatives=False)
        return 0.8 ** 2 * (q2 @ blk.Qs.T) ** 4 @ blk.alphas

    step = 1e-4
    for i in (3, 40):
        fd = np.zeros(3)
        for c in range(3):
            p = st.positions.copy()
            p[i, c] += step
            e1 = site_energies(p)[i]
            p[i, c] -= 2 * step
            e2 = site_energies(p)[i]
            fd[c] = (e1 - e2) / (2 * step)
        assert np.abs(mu[i] - fd).max() < 1e-7 + 1e-5 * np.abs(fd).max()
