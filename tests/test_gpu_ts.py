"""get_ts_energy_and_forces (vdw.f90:163-493) on the device against the oracle's
statement-by-statement restatement: a C/H cell with 6 A lists, inner and outer
buffers, Hirshfeld volumes and per-pair volume gradients (nonzero within the
3.7 A SOAP cutoff only, as the local-property predictor gives them), a
per-atom C6 scaling and the local-virial cut."""
import numpy as np
import pytest

from _util import O, neighbor_data
from turbogap_b200.synth import random_structure

pytestmark = pytest.mark.gpu

C6 = np.array([46.6, 6.5]) * 0.0367
R0 = np.array([3.59, 3.10])
A0 = np.array([12.0, 4.5])


@pytest.mark.parametrize("buffers", [(0.0, 0.0), (1.0, 0.5)])
def test_ts_matches_oracle(gpu, buffers):
    buffer, bin_ = buffers
    rcut, rin = 6.0, 0.6
    st = random_structure(300, (300 / 0.12) ** (1 / 3), 1.0, seed=31, h_fraction=0.25)
    rng = np.random.default_rng(32)
    vol = rng.uniform(0.6, 1.0, st.n)
    nl = neighbor_data(st, rcut)
    nb = nl["neighbors_list"]
    P = len(nb)
    vder = rng.normal(0.0, 0.02, (P, 3))
    vder[nl["rjs"] >= 3.7] = 0.0
    scale = rng.uniform(0.9, 1.1, st.n)
    args = (vol, vder, nl["n_neigh"], nb, nl["neighbor_species"], rcut, buffer, rin, bin_,
            nl["rjs"], nl["xyz"], vol[(nb - 1) % st.n], 0.94, 20.0, C6, R0, A0, st.n)
    e, f, v, lv = gpu.get_ts_energy_and_forces(*args, mbd_ts_scaling=scale, x_min=2.0, x_max=4.0)
    eo, fo, vo, lvo = O.ts_energy_and_forces(*args, scale, 2.0, 4.0)
    assert np.abs(e - eo).max() <= 1e-12 * max(1.0, np.abs(eo).max())
    assert np.abs(f - fo).max() <= 1e-10 * max(1.0, np.abs(fo).max())
    assert np.abs(v - vo).max() <= 1e-10 * max(1.0, np.abs(vo).max())
    assert np.abs(lv - lvo).max() <= 1e-10 * max(1.0, np.abs(lvo).max())
    # energies only
    e2, f2, _, _ = gpu.get_ts_energy_and_forces(*args, mbd_ts_scaling=scale, do_forces=False)
    assert f2 is None and np.abs(e2 - eo).max() <= 1e-12 * max(1.0, np.abs(eo).max())
