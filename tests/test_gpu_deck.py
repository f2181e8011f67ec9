"""A deck written in the reference's file formats (input file, .gap with its
sparse-set files, extended XYZ) run through turbogap_b200.deck on the GPU,
against an MD loop of the FP64 oracle in the reference's step order
(turbogap_md.f90:161-380): thermo.log rows and trajectory frames."""
from __future__ import annotations

import numpy as np
import pytest

from _util import O, sparse_block
from turbogap_b200 import deck as D
from turbogap_b200 import formats as F
from turbogap_b200 import synth
from turbogap_b200.hypers import SoapCompression, carbon_hypers

pytestmark = pytest.mark.gpu


def _write_deck(d, nsteps, dt, e0, extra="", write_xyz=4, temperature=900.0, compress=None):
    h = carbon_hypers()
    h.compress = compress
    blk = sparse_block(h, 300, seed=61)
    F.write_sparse_set(blk, str(d / "desc_C.dat"), str(d / "alphas_C.dat"))
    if compress is not None:
        F.write_compress_file(str(d / "compress_C.dat"), compress, h.alpha_max, h.l_max)
    with open(d / "c.gap", "w") as fh:
        F.write_soap_block(fh, F.spec_from_block(blk, ["C"], "desc_C.dat", "alphas_C.dat",
                                                 "compress_C.dat" if compress else None))
    st = synth.random_structure(216, 12.91, 1.2, seed=62)
    m = np.full(st.n, 12.011 * F.AMU_TO_EV_FS2_A2)
    v = synth.maxwell_velocities(m, temperature, 63)
    F.write_extxyz(str(d / "atoms.xyz"), ["C"] * st.n, st.positions, st.box, step=0, time=0.0,
                   dt=dt, temperature=0.0, pressure=0.0, virial=np.zeros((3, 3)),
                   velocities=v)
    (d / "input").write_text(
        "atoms_file = 'atoms.xyz'\npot_file = 'c.gap'\nn_species = 1\nspecies = C\n"
        f"masses = 12.011\ne0 = {e0!r}\nmd_nsteps = {nsteps}\nmd_step = {dt!r}\n"
        f"write_thermo = 1\nwrite_xyz = {write_xyz}\n" + extra)
    # the deck's values after the round trip through the files
    fr = F.read_extxyz(str(d / "atoms.xyz"))[0]
    return blk, fr, m


def _oracle_md(blk, fr, m, nsteps, dt, e0):
    pos = fr.positions.copy()
    vel = fr.velocities.copy()
    pprev, fprev = np.zeros_like(pos), np.zeros_like(pos)
    sp = np.ones(fr.n, dtype=np.int32)
    a, b, c = fr.lattice
    vol = float(np.dot(np.cross(a, b), c))
    rows, frames = [], {}
    for step in range(nsteps + 1):
        e, f, vir, _ = O.evaluate(pos, sp, fr.lattice, [blk], e0=[e0])
        O.wrap_pbc(pos, a, b, c)
        O.remove_cm_vel(vel, m)
        O.velocity_verlet(pos, pprev, vel, f, fprev, m, dt, dt, step == 0)
        ek = 0.5 * float(np.sum(m[:, None] * vel * vel))
        rows.append((step, step * dt, F.instant_temperature(ek, fr.n), ek, float(e.sum()),
                     F.instant_pressure(ek, fr.n, vir, vol)))
        frames[step] = (pprev.copy(), vel.copy(), f.copy(), e.copy())
    return np.array(rows), frames


def _transformation(full_dim, dim, seed):
    rng = np.random.default_rng(seed)
    P_i = np.concatenate([np.arange(1, dim + 1), rng.integers(1, dim + 1, size=dim)])
    P_j = rng.integers(1, full_dim + 1, size=2 * dim)
    return SoapCompression(dim, P_i, P_j, rng.uniform(0.2, 1.0, size=2 * dim))


@pytest.mark.parametrize("compressed", [False, True])
def test_deck_md_matches_oracle(gpu, tmp_path, compressed):
    """compressed: the potential's block names a compress file (P_transformation
    of 50 rows over the 324 components), which the deck loader hands to the
    device with the sparse set."""
    nsteps, dt, e0 = 9, 1.0, -0.125
    comp = _transformation(324, 50, 65) if compressed else None
    blk, fr, m = _write_deck(tmp_path, nsteps, dt, e0, compress=comp)
    if compressed:
        g = F.read_gap_file(str(tmp_path / "c.gap"))
        assert g.soap_turbo[0].compress_soap and g.soap_turbo[0].file_compress == "compress_C.dat"
    out = tmp_path / "run"
    res = D.run_md(str(tmp_path / "input"), str(out))
    ref, frames = _oracle_md(blk, fr, m, nsteps, dt, e0)
    got = F.read_thermo(str(out / "thermo.log"))
    assert got.shape == (nsteps + 1, 6)
    assert np.array_equal(got[:, 0], ref[:, 0])
    n = fr.n
    # returned rows at full precision: 1e-6 eV/atom on E_pot; E_kin, T and P track it
    r = res["thermo"]
    assert np.abs(r[:, 4] - ref[:, 4]).max() < 1e-6 * n
    assert np.abs(r[:, 3] - ref[:, 3]).max() < 1e-6 * n
    assert np.abs(r[:, 2] - ref[:, 2]).max() < 1e-6 * np.abs(ref[:, 2]).max()
    assert np.abs(r[:, 5] - ref[:, 5]).max() < 1e-5 * np.abs(ref[:, 5]).max()
    # the file holds the same rows at its printed precision
    assert np.abs(got[:, 4] - r[:, 4]).max() < 1e-8 and np.abs(got[:, 2] - r[:, 2]).max() < 1e-4
    # trajectory: steps 0, 4, 8 and the last (9), positions at which forces were evaluated
    tr = F.read_extxyz(str(out / "trajectory_out.xyz"))
    assert [int(t.info["step"]) for t in tr] == [0, 4, 8, 9]
    for t in tr:
        p, v, f, e = frames[int(t.info["step"])]
        assert np.abs(t.positions - p).max() < 1e-7
        assert np.abs(t.velocities - v).max() < 1e-7
        assert abs(float(t.info["energy"]) - e.sum()) < 1e-6 * n
    assert abs(float(tr[0].info["time_step"]) - dt) < 1e-12


def test_deck_predict_frames(gpu, tmp_path):
    dt, e0 = 1.0, 0.0
    blk, fr, m = _write_deck(tmp_path, 1, dt, e0)
    st2 = synth.random_structure(216, 12.91, 1.2, seed=64)
    F.write_extxyz(str(tmp_path / "atoms.xyz"), ["C"] * 216, st2.positions, st2.box, step=10,
                   time=0.0, dt=dt, temperature=0.0, pressure=0.0, virial=np.zeros((3, 3)))
    res = D.run_predict(str(tmp_path / "input"), str(tmp_path / "p"))
    assert len(res) == 2
    sp = np.ones(216, dtype=np.int32)
    for r, pos in zip(res, (fr.positions, st2.positions)):
        eo, fo, vo, _ = O.evaluate(pos, sp, fr.lattice, [blk], e0=[e0])
        assert np.abs(r["energies"] - eo).max() < 1e-6
        assert np.abs(r["forces"] - fo).max() < 1e-6
    tr = F.read_extxyz(str(tmp_path / "p" / "trajectory_out.xyz"))
    assert [t.info["i_config"] for t in tr] == ["1", "2"]


def test_warm_lists_match_cold_prediction(gpu, tmp_path):
    """tests/mc_mpi_neighbors of the reference, for MD with kept lists: every
    frame of a run whose lists live across steps (neighbors_buffer > 0) carries
    the forces and local energies it was given; a cold prediction of the same
    frames, with lists built from scratch, must reproduce them (1e-5 eV/A on
    force components, 1e-6 eV on local energies, as there)."""
    # The reference rebuilds once a squared displacement exceeds buffer / 2, so an
    # atom may move sqrt(buffer / 2) first and two atoms closing in on each other
    # 2 sqrt(buffer / 2); no pair can enter rcut unseen only when that is at most
    # the buffer, i.e. buffer >= 2 A. A smaller buffer follows the reference and
    # can drop a pair near the cutoff.
    nsteps, dt = 30, 1.0
    _write_deck(tmp_path, nsteps, dt, 0.0, extra="neighbors_buffer = 2.0\n", write_xyz=1,
                temperature=2500.0)
    D.run_md(str(tmp_path / "input"), str(tmp_path / "run"))
    traj = F.read_extxyz(str(tmp_path / "run" / "trajectory_out.xyz"))
    assert len(traj) == nsteps + 1
    text = (tmp_path / "input").read_text().replace("atoms_file = 'atoms.xyz'",
                                                    "atoms_file = 'run/trajectory_out.xyz'")
    (tmp_path / "input_cold").write_text(text)
    cold = D.run_predict(str(tmp_path / "input_cold"), str(tmp_path / "cold"))
    assert len(cold) == len(traj)
    for k, (fr, c) in enumerate(zip(traj, cold)):
        assert np.abs(c["forces"] - fr.arrays["forces"]).max() < 1e-5, k
        assert np.abs(c["energies"] - fr.arrays["local_energy"]).max() < 1e-6, k
