"""Seeded synthetic inputs for the benchmark workloads (no datasets exist).

Every structure is a periodic cubic box filled with uniformly random atoms
subject to a minimum pair distance under the minimum-image convention.
Seeds: workload k uses 1000 + k; sub-structures use (1000 + k) * 100 + i.

Workloads:
  carbon216   216 C, L = 12.91 A (2.0 g/cm^3), d_min 1.2 A          (k = 0)
  ch32k       32,768 atoms C:H = 3:1, 0.12 atoms/A^3, d_min 1.0 A   (k = 1)
  cells512    512 C cells, N log-uniform 64..2048, 1.5..3.5 g/cm^3  (k = 2)
  carbon131k  131,072 C at 2.0 g/cm^3                               (k = 3)
  ch1m        1,048,576 atoms C:H = 3:1 at 0.12 atoms/A^3           (k = 4)
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

# md units: masses in eV fs^2 / A^2 = amu * 103.6426965268 (read_files.f90:1301)
AMU_TO_EVFS2A2 = 103.6426965268
KB_EV = 8.6173303e-5          # md.f90:104
MASS_AMU = {1: 12.011, 2: 1.008}
GCM3_TO_AMU_A3 = 0.602214076  # 1 g/cm^3 in amu / A^3


@dataclass
class Structure:
    positions: np.ndarray   # (n, 3) float64, Cartesian A, inside [0, L)
    species: np.ndarray     # (n,) int32 global species ids (1 = C, 2 = H)
    box: np.ndarray         # (3, 3) float64, rows = lattice vectors a, b, c

    @property
    def n(self) -> int:
        return int(self.positions.shape[0])

    @property
    def masses(self) -> np.ndarray:
        """Per-atom masses in eV fs^2 / A^2."""
        lut = np.zeros(max(MASS_AMU) + 1)
        for z, v in MASS_AMU.items():
            lut[z] = v * AMU_TO_EVFS2A2
        return lut[self.species]


def carbon_number_density(rho_gcm3: float) -> float:
    return rho_gcm3 * GCM3_TO_AMU_A3 / MASS_AMU[1]


def random_structure(n: int, L: float, d_min: float, seed: int, h_fraction: float = 0.0,
                     max_rounds: int = 10000) -> Structure:
    """Uniform random atoms in a cubic periodic box, all MIC distances >= d_min.

    Conflicting atoms are redrawn round by round (the later index of each close
    pair moves) until no pair is closer than d_min."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, L, size=(n, 3))
    for _ in range(max_rounds):
        pos = np.mod(pos, L)
        pos[pos >= L] = 0.0
        tree = cKDTree(pos, boxsize=L)
        pairs = tree.query_pairs(d_min, output_type="ndarray")
        if len(pairs) == 0:
            break
        bad = np.unique(pairs.max(axis=1))
        pos[bad] = rng.uniform(0.0, L, size=(len(bad), 3))
    else:
        raise RuntimeError("could not place atoms with the requested minimum distance")
    species = np.ones(n, dtype=np.int32)
    n_h = int(round(n * h_fraction))
    if n_h:
        species[rng.permutation(n)[:n_h]] = 2
    return Structure(positions=pos, species=species, box=np.eye(3) * L)


WORKLOAD_NAMES = ("carbon216", "ch32k", "carbon131k", "ch1m", "cells512")


def workload_structure(name: str, sub: int | None = None) -> Structure:
    """The seeded structure of a named workload (sub-structure index for cells512)."""
    if name == "carbon216":
        return random_structure(216, 12.91, 1.2, seed=1000)
    if name == "ch32k":
        n = 32768
        return random_structure(n, (n / 0.12) ** (1 / 3), 1.0, seed=1001, h_fraction=0.25)
    if name == "carbon131k":
        n = 131072
        return random_structure(n, (n / carbon_number_density(2.0)) ** (1 / 3), 1.2, seed=1003)
    if name == "ch1m":
        n = 1048576
        return random_structure(n, (n / 0.12) ** (1 / 3), 1.0, seed=1004, h_fraction=0.25)
    if name == "cells512":
        rng = np.random.default_rng(1002)
        ns = np.rint(np.exp(rng.uniform(np.log(64), np.log(2048), size=512))).astype(int)
        rho = rng.uniform(1.5, 3.5, size=512)
        i = int(sub)
        L = (ns[i] / carbon_number_density(rho[i])) ** (1 / 3)
        return random_structure(int(ns[i]), L, 1.2, seed=1002 * 100 + i)
    raise KeyError(name)


def cells512_sizes() -> np.ndarray:
    rng = np.random.default_rng(1002)
    return np.rint(np.exp(rng.uniform(np.log(64), np.log(2048), size=512))).astype(int)


def maxwell_velocities(masses: np.ndarray, T: float, seed: int) -> np.ndarray:
    """N(0, kT/m) per component, centre-of-mass velocity removed (md.f90:95-158,
    distribution "maxwell"; no rescaling)."""
    rng = np.random.default_rng(seed)
    v = rng.standard_normal((len(masses), 3)) * np.sqrt(KB_EV * T / masses)[:, None]
    cm = (masses[:, None] * v).sum(0) / masses.sum()
    return v - cm


def sparse_alphas(n_sparse: int, seed: int, sigma: float = 0.01) -> np.ndarray:
    """alpha_s ~ N(0, sigma) eV (sigma read as the standard deviation)."""
    return np.random.default_rng(seed).normal(0.0, sigma, size=n_sparse)
