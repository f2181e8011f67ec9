"""A structure sharded by central-site ranges (the reference's MPI split,
turbogap.f90:930-942) on one GPU: the shares of disjoint ranges sum to the whole
structure's energies, forces and virial, and the in-step NCCL all-reduce on a
one-rank communicator leaves the MD trajectory unchanged. Ranks whose kernels
wait on one another are not run on one GPU; the multi-rank host logic is in
test_multirank_gloo.py."""
from __future__ import annotations

import numpy as np
import pytest

from _util import O, sparse_block
from turbogap_b200.hypers import ch_hypers
from turbogap_b200.parallel import site_range
from turbogap_b200.synth import maxwell_velocities, random_structure

pytestmark = pytest.mark.gpu

L300 = (300 / 0.12) ** (1 / 3)


@pytest.fixture(scope="module")
def ch(gpu):
    bC = sparse_block(ch_hypers(1), 400, seed=8, n_atoms=300, L=L300, d_min=1.0,
                      h_fraction=0.25, n_structs=3)
    bH = sparse_block(ch_hypers(2), 300, seed=9, n_atoms=300, L=L300, d_min=1.0,
                      h_fraction=0.25, n_structs=4)
    gpu.soap_backend_begin(bC, key=301)
    gpu.soap_backend_begin(bH, key=302)
    return bC, bH


def test_site_range_shares_sum_to_whole(gpu, ch):
    st = random_structure(300, L300, 1.0, seed=21, h_fraction=0.25)
    e0 = np.array([-0.5, -0.25])
    full = gpu.Engine(st.positions, st.species, st.masses, st.box, [301, 302], e0_by_species=e0)
    e, f, v = full.compute()
    eo, fo, vo, _ = O.evaluate(st.positions, st.species, st.box, list(ch), e0=e0)
    assert np.abs(e - eo).max() < 1e-6 and np.abs(f - fo).max() < 1e-6
    for world in (2, 3):
        es, fs, vs = np.zeros_like(e), np.zeros_like(f), np.zeros_like(v)
        pairs = 0
        for rank in range(world):
            beg, end = site_range(st.n, world, rank)
            eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [301, 302],
                             e0_by_species=e0)
            eng.set_site_range(beg, end)
            er, fr, vr = eng.compute()
            pairs += eng.n_pairs()   # each rank lists its own sites only
            assert np.all(er[:beg] == 0.0) and np.all(er[end:] == 0.0)
            # the oracle computes the same share (its site_range argument)
            eq, fq, vq, _ = O.evaluate(st.positions, st.species, st.box, list(ch), e0=e0,
                                       site_range=(beg, end))
            assert np.abs(er - eq).max() < 1e-6 and np.abs(fr - fq).max() < 1e-6
            es += er
            fs += fr
            vs += vr
            eng.close()
        assert pairs == full.n_pairs()
        assert np.abs(es - e).max() < 1e-9
        assert np.abs(fs - f).max() < 1e-9
        assert np.abs(vs - v).max() < 1e-9 * np.abs(v).max()
    full.close()


def test_site_range_arguments(gpu, ch):
    st = random_structure(300, L300, 1.0, seed=22, h_fraction=0.25)
    eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [301, 302])
    for beg, end in ((-1, 10), (20, 10), (0, 301)):
        with pytest.raises(gpu.BackendError):
            eng.set_site_range(beg, end)
    eng.set_site_range(0, 0)              # an empty share evaluates nothing
    e, f, v = eng.compute()
    assert not e.any() and not f.any() and not v.any()
    eng.close()


def test_one_rank_communicator_keeps_the_trajectory(gpu, ch):
    st = random_structure(300, L300, 1.0, seed=23, h_fraction=0.25)
    vel = maxwell_velocities(st.masses, 500.0, 24)
    runs = []
    for use_comm in (False, True):
        eng = gpu.Engine(st.positions, st.species, st.masses, st.box, [301, 302])
        eng.set_state(st.positions, vel)
        if use_comm:
            eng.set_comm(gpu.nccl_unique_id(), 1, 0)
        ep, ek = eng.md(6, 0.5)
        p, v, f = eng.get_state()
        runs.append((ep, ek, p, v, f))
        eng.set_comm(None)
        eng.close()
    a, b = runs
    # forces are summed with atomics, so two runs agree to rounding, not bit for bit
    assert abs(a[0] - b[0]) < 1e-9 * abs(a[0]) and abs(a[1] - b[1]) < 1e-9 * abs(a[1])
    for x, y in zip(a[2:], b[2:]):
        assert np.abs(x - y).max() < 1e-9
