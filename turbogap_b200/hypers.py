"""soap_turbo hyperparameters and GAP sparse-set blocks.

Mirrors ``type soap_turbo`` (types.f90:75-134) and the defaults that
``read_gap_hypers`` applies while parsing a soap_turbo block
(read_files.f90:4648-4667): nf 4, buffer 0.5, sigma scalings 0,
amplitude_scaling 1, central_weight 1, global_scaling 1, basis poly3,
scaling_mode polynomial, radial_enhancement 0, central_species 0.
``rcut_soft`` is stored as the reference stores it after the block closes:
rcut_hard - buffer (read_files.f90:5101-5108).
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np


@dataclass
class SoapCompression:
    """soap_turbo compression (``compress_P_*``, types.f90:92-110, filled at
    read_files.f90:5166-5231): the descriptor has ``dim`` components,
    q_c(i) = sum of P_el(k) p(P_j(k)) over the entries k with P_i(k) = i
    (1-based; p in the uncompressed order n <= n', l), normalised after the map."""
    dim: int
    P_i: np.ndarray
    P_j: np.ndarray
    P_el: np.ndarray

    def __post_init__(self):
        self.dim = int(self.dim)
        self.P_i = np.ascontiguousarray(self.P_i, dtype=np.int32)
        self.P_j = np.ascontiguousarray(self.P_j, dtype=np.int32)
        self.P_el = np.ascontiguousarray(self.P_el, dtype=np.float64)
        if not (self.P_i.shape == self.P_j.shape == self.P_el.shape) or self.P_i.ndim != 1:
            raise ValueError("compression entries need matching P_i, P_j, P_el")
        if self.dim < 1 or len(self.P_el) < 1:
            raise ValueError("compression needs dim >= 1 and at least one entry")

    def matrix(self, full_dim: int) -> np.ndarray:
        """The dense (dim, full_dim) transformation."""
        P = np.zeros((self.dim, full_dim))
        np.add.at(P, (self.P_i.astype(np.int64) - 1, self.P_j.astype(np.int64) - 1), self.P_el)
        return P


def trivial_compression(alpha_max: Sequence[int], l_max: int) -> SoapCompression:
    """compress_mode "trivial", as the reference's generator of compress files
    writes it (tools/compress_indices/compress_indices.py:39-57): keep the
    components (n, n', l), n <= n', in which n or n' is the first radial
    channel of some species; P_el = 1."""
    nmax = [int(a) for a in alpha_max]
    pivots = set(np.cumsum([0] + nmax[:-1]).tolist())    # 0-based first channel per species
    ntot = sum(nmax)
    keep = []
    k = 0
    for n in range(ntot):
        for n2 in range(n, ntot):
            for _ in range(l_max + 1):
                k += 1
                if n in pivots or n2 in pivots:
                    keep.append(k)
    d = len(keep)
    return SoapCompression(d, np.arange(1, d + 1), np.array(keep), np.ones(d))


@dataclass
class SoapTurboHypers:
    species_z: List[int]            # global species ids of the descriptor's species
    alpha_max: List[int]            # n_max per species
    l_max: int = 8
    rcut_hard: List[float] = None
    buffer: List[float] = None
    nf: List[float] = None
    atom_sigma_r: List[float] = None
    atom_sigma_t: List[float] = None
    atom_sigma_r_scaling: List[float] = None
    atom_sigma_t_scaling: List[float] = None
    amplitude_scaling: List[float] = None
    central_weight: List[float] = None
    global_scaling: List[float] = None
    radial_enhancement: int = 0
    central_species: int = 0        # 1-based index into species_z; 0 = every atom
    basis: str = "poly3"
    scaling_mode: str = "polynomial"
    compress: Optional[SoapCompression] = None

    def __post_init__(self):
        n = len(self.species_z)

        def fill(v, default):
            if v is None:
                return [float(default)] * n
            v = [float(x) for x in v]
            if len(v) != n:
                raise ValueError("per-species hyperparameter lists need n_species entries")
            return v

        self.rcut_hard = fill(self.rcut_hard, 3.7)
        self.buffer = fill(self.buffer, 0.5)
        self.nf = fill(self.nf, 4.0)
        self.atom_sigma_r = fill(self.atom_sigma_r, 0.5)
        self.atom_sigma_t = fill(self.atom_sigma_t, 0.5)
        self.atom_sigma_r_scaling = fill(self.atom_sigma_r_scaling, 0.0)
        self.atom_sigma_t_scaling = fill(self.atom_sigma_t_scaling, 0.0)
        self.amplitude_scaling = fill(self.amplitude_scaling, 1.0)
        self.central_weight = fill(self.central_weight, 1.0)
        self.global_scaling = fill(self.global_scaling, 1.0)
        self.alpha_max = [int(a) for a in self.alpha_max]
        if len(self.alpha_max) != n:
            raise ValueError("alpha_max needs n_species entries")
        if not (0 <= self.radial_enhancement <= 2):
            raise ValueError("radial_enhancement must be 0, 1 or 2")
        if self.basis != "poly3":
            raise ValueError(f"basis {self.basis!r}: only poly3 is implemented")
        if self.scaling_mode != "polynomial":
            raise ValueError("only scaling_mode polynomial is implemented")

    @property
    def n_species(self) -> int:
        return len(self.species_z)

    @property
    def rcut_soft(self) -> List[float]:
        # read_files.f90:5101-5108: buffer 0 means rcut_soft = rcut_hard
        return [h if b == 0.0 else h - b for h, b in zip(self.rcut_hard, self.buffer)]

    @property
    def rcut_max(self) -> float:
        return max(self.rcut_hard)

    @property
    def n_max(self) -> int:
        return int(sum(self.alpha_max))

    @property
    def uncompressed_dim(self) -> int:
        # read_files.f90:5233-5235
        n = self.n_max
        return n * (n + 1) // 2 * (self.l_max + 1)

    @property
    def dim(self) -> int:
        """Components of the descriptor the kernel sees: the compressed dim when
        the block is compressed (read_files.f90:5171, 5213-5216)."""
        return self.compress.dim if self.compress is not None else self.uncompressed_dim

    @property
    def device_dim(self) -> int:
        """Row length of descriptor and dE/dq rows on the device (the input size
        of a mixed-form MLP): dim, or a compressed dim rounded up to a multiple
        of 8 with zero components."""
        return self.dim if self.compress is None else (self.dim + 7) // 8 * 8

    @property
    def n_lm(self) -> int:
        return (self.l_max + 1) ** 2


@dataclass
class GapBlock:
    """One soap_turbo descriptor block with its sparse set (delta, zeta, Qs, alphas)."""
    hypers: SoapTurboHypers
    Qs: np.ndarray                  # (n_sparse, dim) float64 (row = one sparse point)
    alphas: np.ndarray              # (n_sparse,) float64
    delta: float = 1.0
    zeta: float = 4.0

    def __post_init__(self):
        self.Qs = np.ascontiguousarray(self.Qs, dtype=np.float64)
        self.alphas = np.ascontiguousarray(self.alphas, dtype=np.float64)
        if self.Qs.ndim != 2 or self.Qs.shape[1] != self.hypers.dim:
            raise ValueError(f"Qs must be (n_sparse, {self.hypers.dim})")
        if self.alphas.shape != (self.Qs.shape[0],):
            raise ValueError("alphas must have n_sparse entries")

    @property
    def n_sparse(self) -> int:
        return int(self.Qs.shape[0])


def carbon_hypers(n_max: int = 8, l_max: int = 8) -> SoapTurboHypers:
    """Single-species carbon block: rcut 3.7, buffer 0.5, sigmas 0.5, nf 4."""
    return SoapTurboHypers(species_z=[1], alpha_max=[n_max], l_max=l_max)


def ch_hypers(central: int, n_max: int = 8, l_max: int = 8) -> SoapTurboHypers:
    """Two-species (C=1, H=2) block centred on descriptor species ``central``."""
    return SoapTurboHypers(species_z=[1, 2], alpha_max=[n_max, n_max], l_max=l_max,
                           central_species=central)


def blocks_species_cutoff(blocks: Sequence[GapBlock]) -> float:
    return max(b.hypers.rcut_max for b in blocks)
