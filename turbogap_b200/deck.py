"""Run a TurboGAP deck (input file + .gap potential + extended XYZ) on the device.

``run_md`` follows ``turbogap md <input>`` for NVE velocity Verlet on soap_turbo
blocks: steps 0..md_nsteps (turbogap.f90:664-676), each an evaluation at x(t)
followed by the integrator; ``thermo.log`` rows at step 0, the last step and
every ``write_thermo`` steps (turbogap_md.f90:299-330); trajectory frames at
step 0, the last step and every ``write_xyz`` steps, holding the positions the
forces were evaluated at (turbogap_md.f90:357-380). ``run_predict`` evaluates
every frame of the atoms file (``turbogap predict``).

soap_turbo blocks (compressed ones included) and the distance_2b, angle_3b and
core_pot families run on the device, in orthorhombic and triclinic boxes. Decks
that need anything else (thermostats, barostats, adaptive time steps) are
refused with the keyword that needs it. Velocities drawn here (no velocity
column, or ``randomize_velocities``) follow md.f90:95-158 with numpy's
generator, so they differ from the reference's random stream.
"""
from __future__ import annotations

import os
import zlib
from typing import Dict, List, Optional

import numpy as np

from . import backend
from . import formats as F
from .hypers import GapBlock


def block_key(block: GapBlock) -> int:
    """A key from the block's content: the backend keeps one device copy of a
    sparse set per key, so equal keys must mean equal blocks."""
    h = block.hypers
    c = zlib.crc32(block.Qs.tobytes())
    c = zlib.crc32(block.alphas.tobytes(), c)
    c = zlib.crc32(repr((vars(h), float(block.delta), float(block.zeta))).encode(), c)
    return int(c & 0x3FFFFFFF) + 1


def family_key(f) -> int:
    """A content key for a 2b / 3b / core_pot family (disjoint from block keys
    in practice: a different hash input)."""
    c = zlib.crc32(repr((f.kind, tuple(f.species))).encode())
    for name in ("Qs", "alphas", "cutoff", "x", "V"):
        if hasattr(f, name):
            c = zlib.crc32(np.ascontiguousarray(getattr(f, name)).tobytes(), c)
    for name in ("delta", "sigma", "rcut", "kernel_type", "yp1", "ypn"):
        if hasattr(f, name):
            c = zlib.crc32(repr(getattr(f, name)).encode(), c)
    return int(c & 0x3FFFFFFF) + 0x40000000


def _remove_cm_vel(v: np.ndarray, m: np.ndarray) -> np.ndarray:
    """md.f90:316-344: subtract the centre-of-mass velocity."""
    return v - (m[:, None] * v).sum(0) / m.sum()


def draw_velocities(masses: np.ndarray, t_beg: float, distribution: str,
                    seed: int) -> np.ndarray:
    """md.f90:95-158. "maxwell": N(0, kT/m) per component, centre of mass
    removed, no rescale. "uniform": U[0, 1) per component, centre of mass
    removed, rescaled to t_beg. Fewer than two atoms get zero velocities."""
    n = len(masses)
    if n < 2:
        return np.zeros((n, 3))
    rng = np.random.default_rng(seed)
    if distribution == "maxwell":
        v = rng.normal(size=(n, 3)) * np.sqrt(F.KB_EV * t_beg / masses)[:, None]
        return _remove_cm_vel(v, masses)
    v = _remove_cm_vel(rng.random((n, 3)), masses)
    ek = 0.5 * float(np.sum(masses[:, None] * v * v))
    t = F.instant_temperature(ek, n)
    return v * np.sqrt(t_beg / t)


class Deck:
    """An input deck resolved against its files: species, masses, blocks, frame."""

    def __init__(self, input_path: str):
        self.input = F.read_input_file(input_path)
        d = self.input
        self.base = d.base_dir
        if d.pot_file is None or d.atoms_file is None:
            raise ValueError("the input file needs pot_file and atoms_file")
        self.gap = F.read_gap_file(os.path.join(self.base, d.pot_file))
        raw = self.gap.distance_2b + self.gap.angle_3b + self.gap.core_pot
        if not self.gap.soap_turbo and not raw:
            raise ValueError(f"{d.pot_file} has no GAP block")
        off = d.off_path()
        if off:
            raise NotImplementedError("not on the device path: " + "; ".join(off))
        self.species_types = d.species
        self.blocks: List[GapBlock] = [s.load(self.species_types, self.base)
                                       for s in self.gap.soap_turbo]
        self.families = [b.load(self.species_types, self.base, d.core_pot_cutoff,
                                d.core_pot_buffer) for b in raw]
        self.frames = F.read_extxyz(os.path.join(self.base, d.atoms_file))
        if not self.frames:
            raise ValueError(f"{d.atoms_file} holds no structure")

    def species_ids(self, frame: F.Frame) -> np.ndarray:
        """1-based indices into the input's species list (read_files.f90:245-268)."""
        ids = np.zeros(frame.n, dtype=np.int32)
        for i, s in enumerate(frame.species):
            if s not in self.species_types:
                raise ValueError(f"atom {i + 1} has no known species ({s!r})")
            ids[i] = self.species_types.index(s) + 1
        return ids

    def masses(self, frame: F.Frame, ids: np.ndarray) -> np.ndarray:
        """eV fs^2 / A^2. A mass column of the XYZ file wins over the input's masses."""
        if frame.masses is not None:
            return frame.masses * F.AMU_TO_EV_FS2_A2
        amu = self.input.masses_amu
        if amu is None:
            raise ValueError("no masses: give `masses` in the input file or a masses column "
                             "in the XYZ file (the element database is not included)")
        return np.asarray(amu)[ids - 1] * F.AMU_TO_EV_FS2_A2

    def begin(self) -> List[int]:
        keys = []
        for b in self.blocks:
            keys.append(block_key(b))
            backend.soap_backend_begin(b, keys[-1])
        backend.soap_backend_end()
        for f in self.families:
            keys.append(family_key(f))
            backend.family_begin(f, keys[-1])
        return keys

    def engine(self, frame: F.Frame, keys: List[int]) -> backend.Engine:
        ids = self.species_ids(frame)
        return backend.Engine(frame.positions, ids, self.masses(frame, ids), frame.lattice, keys,
                              e0_by_species=self.input.e0,
                              neighbors_buffer=self.input.neighbors_buffer)


def run_md(input_path: str, out_dir: Optional[str] = None) -> Dict[str, object]:
    """Run the deck's MD and write thermo.log and trajectory_out.xyz to out_dir
    (default: the deck's directory). Returns the thermo rows as an array."""
    deck = Deck(input_path)
    d = deck.input
    out = out_dir or deck.base
    os.makedirs(out, exist_ok=True)
    frame = deck.frames[0]
    ids = deck.species_ids(frame)
    masses = deck.masses(frame, ids)
    if frame.velocities is None or d.randomize_velocities:
        vel = draw_velocities(masses, d.t_beg, d.velocity_distribution, d.random_seed)
    else:
        vel = frame.velocities
    if frame.fix_atoms is not None and frame.fix_atoms.any():
        raise NotImplementedError("fix_atoms is not on the device path")
    keys = deck.begin()
    eng = deck.engine(frame, keys)
    eng.set_state(frame.positions, vel)
    vol = float(np.dot(np.cross(frame.lattice[0], frame.lattice[1]), frame.lattice[2]))
    n, nsteps, dt = frame.n, d.md_nsteps, d.md_step
    wt, wx = max(d.write_thermo, 0), max(d.write_xyz, 0)

    def wanted(step, every):
        return step == 0 or step == nsteps or (every > 0 and step % every == 0)

    thermo_path = os.path.join(out, "thermo.log")
    traj_path = os.path.join(out, "trajectory_out.xyz")
    rows = []
    with open(thermo_path, "w") as th:
        th.write(F.THERMO_HEADER + "\n")
        step = 0
        while step <= nsteps:
            # run quietly up to the next step that writes something
            nxt = step
            while nxt < nsteps and not (wanted(nxt, wt) or wanted(nxt, wx)):
                nxt += 1
            if nxt > step:
                eng.md(nxt - step, dt, energies=False)
                step = nxt
            e_pot, e_kin = eng.md(1, dt)
            t = step * dt
            if wanted(step, wt) or wanted(step, wx):
                pos, v, f, e, vir = eng.get_frame()
                temp = F.instant_temperature(e_kin, n)
                pres = F.instant_pressure(e_kin, n, vir, vol)
                if wanted(step, wt):
                    rows.append((step, t, temp, e_kin, e_pot, pres))
                    th.write(F.thermo_row(step, t, temp, e_kin, e_pot, pres) + "\n")
                if wanted(step, wx):
                    F.write_extxyz(traj_path, frame.species, pos, frame.lattice, step=step,
                                   time=t, dt=dt, temperature=temp, pressure=pres,
                                   virial=vir, velocities=v, forces=f, local_energies=e,
                                   masses_amu=frame.masses)
            step += 1
    eng.close()
    return {"thermo": np.array(rows), "thermo_path": thermo_path, "trajectory_path": traj_path}


def run_predict(input_path: str, out_dir: Optional[str] = None) -> List[Dict[str, np.ndarray]]:
    """Energies, forces and virial of every frame of the atoms file, written to
    trajectory_out.xyz as configurations i_config = 1, 2, ..."""
    deck = Deck(input_path)
    out = out_dir or deck.base
    os.makedirs(out, exist_ok=True)
    traj_path = os.path.join(out, "trajectory_out.xyz")
    keys = deck.begin()
    res = []
    for k, frame in enumerate(deck.frames):
        ids = deck.species_ids(frame)
        eng = deck.engine(frame, keys)
        e, f, vir = eng.compute()
        eng.close()
        F.write_extxyz(traj_path, frame.species, frame.positions, frame.lattice, step=-(k + 1),
                       time=0.0, dt=0.0, temperature=0.0, pressure=0.0, virial=vir, forces=f,
                       local_energies=e, masses_amu=frame.masses, overwrite=(k == 0))
        res.append({"energies": e, "forces": f, "virial": vir, "species": ids})
    return res
