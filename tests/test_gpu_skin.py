"""Neighbour lists kept between rebuilds when neighbors_buffer > 0
(turbogap_md.f90:451-470, neighbors.f90:544-590): the engine builds its lists to
rcut + buffer, recomputes the kept pairs' distances every step, and rebuilds
only once some atom's accumulated squared displacement exceeds buffer / 2.
Checked against an engine that rebuilds every step, against the oracle, and
against the reference's rebuild criterion replayed on the host."""
from __future__ import annotations

import numpy as np
import pytest

from _util import O, sparse_block
from turbogap_b200.hypers import ch_hypers
from turbogap_b200.synth import maxwell_velocities, random_structure

pytestmark = pytest.mark.gpu

L = (300 / 0.12) ** (1 / 3)


@pytest.fixture(scope="module")
def ch(gpu):
    bC = sparse_block(ch_hypers(1), 300, seed=71, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=2)
    bH = sparse_block(ch_hypers(2), 200, seed=72, n_atoms=300, L=L, d_min=1.0, h_fraction=0.25,
                      n_structs=4)
    gpu.soap_backend_begin(bC, key=701)
    gpu.soap_backend_begin(bH, key=702)
    return bC, bH


def _engine(gpu, st, buffer):
    return gpu.Engine(st.positions, st.species, st.masses, st.box, [701, 702],
                      neighbors_buffer=buffer)


def test_buffered_lists_follow_the_reference_criterion(gpu, ch):
    st = random_structure(300, L, 1.0, seed=73, h_fraction=0.25)
    vel = maxwell_velocities(st.masses, 1500.0, 74)
    buffer, dt, nsteps = 0.2, 1.0, 60
    eng = _engine(gpu, st, buffer)
    ref = _engine(gpu, st, 0.0)
    assert ref.neighbor_stats() == (-1, -1)
    for e in (eng, ref):
        e.set_state(st.positions, vel)
    disp = np.zeros((st.n, 3))
    expected = 1                      # the first evaluation builds
    for step in range(nsteps):
        ep, ek = eng.md(1, dt)
        rp, rk = ref.md(1, dt)
        assert abs(ep - rp) < 1e-8 * abs(rp) and abs(ek - rk) < 1e-8 * abs(rk), step
        # turbogap_md.f90:451-470 on the same doubles: positions after the step
        # minus the positions the step evaluated
        after, _, _ = eng.get_state()
        before = eng.get_frame()[0]
        disp = (disp + after) - before
        if step < nsteps - 1 and np.any(np.sum(disp * disp, axis=1) > buffer / 2.0):
            expected += 1
            disp[:] = 0.0
    builds, evals = eng.neighbor_stats()
    assert evals == nsteps
    assert builds == expected
    assert 1 < builds < nsteps        # lists were both kept and rebuilt in this run
    p1, v1, f1 = eng.get_state()
    p2, v2, f2 = ref.get_state()
    # a kept list walks its pairs in an older order than a fresh one, so the fp32
    # sums round differently and the two trajectories part slowly (chaos)
    assert np.abs(p1 - p2).max() < 1e-6 and np.abs(f1 - f2).max() < 1e-4
    # the kept lists give the oracle's energies and forces at the current positions
    e, f, _ = eng.compute()
    eo, fo, _, _ = O.evaluate(p1, st.species, st.box, list(ch))
    assert np.abs(e - eo).max() < 1e-6 and np.abs(f - fo).max() < 1e-6
    eng.close()
    ref.close()


def test_buffered_engine_single_point_and_set_state(gpu, ch):
    st = random_structure(300, L, 1.0, seed=75, h_fraction=0.25)
    eng = _engine(gpu, st, 0.5)
    e, f, v = eng.compute()
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, list(ch))
    assert np.abs(e - eo).max() < 1e-6 and np.abs(f - fo).max() < 1e-6
    assert np.abs(v - vo).max() < 1e-6 * np.abs(vo).max()
    # new positions from outside force a rebuild before the next evaluation
    st2 = random_structure(300, L, 1.0, seed=76, h_fraction=0.25)
    eng.set_state(st2.positions)
    e2, f2, _ = eng.compute()
    eo2, fo2, _, _ = O.evaluate(st2.positions, st.species, st.box, list(ch))
    assert np.abs(e2 - eo2).max() < 1e-6 and np.abs(f2 - fo2).max() < 1e-6
    assert eng.neighbor_stats() == (2, 2)
    eng.close()
