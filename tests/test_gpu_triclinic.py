"""Triclinic boxes in the device engine: the reference's O(N N_supercell) list
search (neighbors.f90:474-514, the triclinic get_distance :107-140) and its
triclinic wrap_pbc (md.f90:348-380). Energies, forces and the virial against
the FP64 oracle at 1e-6 (eV/atom, eV/A, relative), in a sheared cell and in a
small sheared cell that needs a supercell, and an NVE run against the oracle's
MD loop."""
import numpy as np
import pytest

from _util import O, sparse_block
from turbogap_b200.hypers import ch_hypers
from turbogap_b200.synth import Structure, maxwell_velocities, random_structure

pytestmark = pytest.mark.gpu

L = (300 / 0.12) ** (1 / 3)
SHEAR = np.array([[1.0, 0.0, 0.0], [0.22, 1.0, 0.0], [-0.13, 0.09, 1.0]])


def sheared(n, L0, seed):
    """A random C/H cell whose cube is sheared into a triclinic box (the
    fractional coordinates are kept)."""
    st = random_structure(n, L0, 1.0, seed=seed, h_fraction=0.25)
    box = SHEAR * L0
    pos = (st.positions / L0) @ box
    return Structure(pos, st.species, box)


@pytest.fixture(scope="module")
def ch(gpu):
    bC = sparse_block(ch_hypers(1), 300, seed=51, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=2)
    bH = sparse_block(ch_hypers(2), 200, seed=52, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=4)
    gpu.soap_backend_begin(bC, key=1901)
    gpu.soap_backend_begin(bH, key=1902)
    return bC, bH


@pytest.mark.parametrize("n,L0", [(300, L), (40, (40 / 0.12) ** (1 / 3))])
def test_engine_matches_oracle(gpu, ch, n, L0):
    st = sheared(n, L0, seed=53 + n)
    e0 = np.array([-0.5, -0.25])
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, list(ch), e0=e0)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [1901, 1902], e0_by_species=e0)
    e, f, v = eng.compute()
    assert np.abs(e - eo).max() < 1e-6
    assert np.abs(f - fo).max() < 1e-6
    assert np.abs(v - vo).max() < 1e-6 * np.abs(vo).max()
    eng.close()


def test_nve_follows_the_oracle_loop(gpu, ch):
    st = sheared(300, L, seed=57)
    vel = maxwell_velocities(st.masses, 900.0, 58)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [1901, 1902])
    eng.set_state(st.positions, vel)
    nsteps, dt = 6, 1.0
    eng.md(nsteps, dt)
    p_gpu, v_gpu, _ = eng.get_state()
    # the oracle in the reference's step order (turbogap_md.f90:161-297)
    pos, v = st.positions.copy(), vel.copy()
    pprev, fprev = np.zeros_like(pos), np.zeros_like(pos)
    a, b, c = st.box
    for step in range(nsteps):
        _, f, _, _ = O.evaluate(pos, st.species, st.box, list(ch))
        O.wrap_pbc(pos, a, b, c)
        O.remove_cm_vel(v, st.masses)
        O.velocity_verlet(pos, pprev, v, f, fprev, st.masses, dt, dt, step == 0)
    assert np.abs(p_gpu - pos).max() < 1e-7 and np.abs(v_gpu - v).max() < 1e-7
    # the wrapped positions of the last evaluated step lie in the cell
    frac = pprev @ np.linalg.inv(st.box)
    assert frac.min() > -1e-9 and frac.max() < 1.0 + 1e-9
    eng.close()
