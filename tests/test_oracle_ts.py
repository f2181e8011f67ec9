"""The oracle's get_ts_energy_and_forces (vdw.f90:163-493) against its energy:
with fixed Hirshfeld volumes (no volume gradients) the TS energy is a pair
energy, and the forces it returns are minus its gradient (central differences,
h = 1e-4 A) when no pair lies in a buffer zone. Inside the buffers the
reference's slope of 1/r^6 (vdw.f90:287-300) is taken before the smoothing
factor is applied to r6, so there its forces are not the gradient of its
energy; the restatement keeps that, and the buffered case is checked against
the device instead (tests/test_gpu_ts.py)."""
import numpy as np
import pytest

from _util import O, neighbor_data
from turbogap_b200.synth import Structure, random_structure

C6 = np.array([46.6, 6.5]) * 0.0367     # eV A^6 scale; any positive numbers serve here
R0 = np.array([3.59, 3.10])
A0 = np.array([12.0, 4.5])


def _ts(st, vol, rcut, buffer, rin, bin_):
    nl = neighbor_data(st, rcut)
    nn = nl["n_neigh"]
    nb = nl["neighbors_list"]
    vn = vol[(nb - 1) % st.n]
    e, f, v, lv = O.ts_energy_and_forces(vol, np.zeros((len(nb), 3)), nn, nb,
                                         nl["neighbor_species"], rcut, buffer, rin, bin_,
                                         nl["rjs"], nl["xyz"], vn, 0.94, 20.0, C6, R0, A0, st.n,
                                         np.ones(st.n), 0.0, 1.0)
    return e, f, v


@pytest.mark.parametrize("buffers", [(0.0, 0.0)])
def test_ts_pair_forces_are_the_energy_gradient(buffers):
    buffer, bin_ = buffers
    rcut, rin = 6.0, 0.6
    st = random_structure(60, 10.0, 1.1, seed=7, h_fraction=0.3)
    vol = np.random.default_rng(8).uniform(0.6, 1.0, st.n)
    e, f, _ = _ts(st, vol, rcut, buffer, rin, bin_)
    assert np.all(np.isfinite(e)) and e.sum() < 0.0
    h = 1e-4
    for a in (0, 17, 41):
        for c in range(3):
            p = st.positions.copy()
            p[a, c] += h
            ep = _ts(Structure(p, st.species, st.box), vol, rcut, buffer, rin, bin_)[0].sum()
            p[a, c] -= 2 * h
            em = _ts(Structure(p, st.species, st.box), vol, rcut, buffer, rin, bin_)[0].sum()
            fd = -(ep - em) / (2 * h)
            assert abs(f[a, c] - fd) < 1e-7 + 1e-5 * abs(fd)
