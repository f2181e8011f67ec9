"""The other GAP families: distance_2b, angle_3b and core_pot.

Their parameters as the reference holds them after reading a .gap file
(types.f90 distance_2b, angle_3b, core_pot; read_files.f90:5238-5505), with
species as global ids (1-based positions in the input's species list). The
device evaluates them next to the soap_turbo blocks (gap.f90:400-1042).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Sequence, Tuple

import numpy as np


@dataclass
class Distance2b:
    species: Tuple[int, int]
    delta: float
    sigma: float
    rcut: float
    Qs: np.ndarray          # (n,) sparse distances
    alphas: np.ndarray      # (n,)
    cutoff: np.ndarray      # (n,) the second column of the alphas file
    kind: str = "distance_2b"

    def __post_init__(self):
        self.Qs = np.ascontiguousarray(self.Qs, dtype=np.float64).reshape(-1)
        self.alphas = np.ascontiguousarray(self.alphas, dtype=np.float64)
        self.cutoff = np.ascontiguousarray(self.cutoff, dtype=np.float64)
        if not (len(self.Qs) == len(self.alphas) == len(self.cutoff)):
            raise ValueError("Qs, alphas and cutoff need the same length")


@dataclass
class Angle3b:
    species: Tuple[int, int, int]   # center, species1, species2
    delta: float
    sigma: Sequence[float]          # 3
    rcut: float
    Qs: np.ndarray                  # (n, 3): (r_ij + r_ik, (r_ij - r_ik)^2, r_jk)
    alphas: np.ndarray
    cutoff: np.ndarray
    kernel_type: str = "exp"        # "exp" or "pol"
    kind: str = "angle_3b"

    def __post_init__(self):
        self.Qs = np.ascontiguousarray(self.Qs, dtype=np.float64).reshape(-1, 3)
        self.alphas = np.ascontiguousarray(self.alphas, dtype=np.float64)
        self.cutoff = np.ascontiguousarray(self.cutoff, dtype=np.float64)
        self.sigma = [float(x) for x in self.sigma]
        if len(self.sigma) != 3:
            raise ValueError("angle_3b needs three sigmas")
        if self.kernel_type not in ("exp", "pol"):
            raise ValueError(f"kernel_type {self.kernel_type!r}: exp or pol")
        if not (len(self.Qs) == len(self.alphas) == len(self.cutoff)):
            raise ValueError("Qs, alphas and cutoff need the same length")


@dataclass
class CorePot:
    species: Tuple[int, int]
    x: np.ndarray           # table nodes (A), increasing
    V: np.ndarray           # pair energy at the nodes (eV)
    yp1: float              # end slopes as in the file (> 0.99e30: natural end)
    ypn: float
    kind: str = "core_pot"

    def __post_init__(self):
        self.x = np.ascontiguousarray(self.x, dtype=np.float64)
        self.V = np.ascontiguousarray(self.V, dtype=np.float64)
        if len(self.x) < 2 or len(self.x) != len(self.V):
            raise ValueError("core_pot needs at least two (x, V) nodes")

    @property
    def rcut(self) -> float:
        return float(self.x[-1])

    @staticmethod
    def from_table(species, x, V, yp1, ypn, cutoff=1e10, buffer=1.0) -> "CorePot":
        """Nodes beyond ``cutoff`` dropped and V tapered by 1/2 (cos(pi (x - cutoff
        + buffer) / buffer) + 1) over the last ``buffer`` (read_files.f90:5425-5447;
        core_pot_cutoff and core_pot_buffer default to 1e10 and 1)."""
        x = np.asarray(x, dtype=np.float64)
        V = np.asarray(V, dtype=np.float64)
        keep = x <= cutoff
        x, V = x[keep], V[keep].copy()
        t = x > cutoff - buffer
        V[t] = V[t] * 0.5 * (np.cos(math.pi / buffer * (x[t] - cutoff + buffer)) + 1.0)
        return CorePot(tuple(species), x, V, float(yp1), float(ypn))


def rcut_of(f) -> float:
    return float(f.rcut)
