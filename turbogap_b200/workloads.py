"""Benchmark workloads: seeded structures and sparse sets built on the GPU.

A workload fixes the structure (see synth.py), the soap_turbo blocks and their
sparse sets, and the MD settings. Sparse sets are the descriptors of central
atoms of further seeded structures of the same kind, computed by this backend
(get_soap), n_sparse of them drawn without replacement; alphas ~ N(0, 0.01) eV.

  carbon216  1 block  (C),      D = 324,  M = 1000, dt 1.0 fs, 300 K
  ch32k      2 blocks (C and H), D = 1224, M = 4000 each, dt 1.0 fs, 300 K
  carbon131k 1 block  (C),      D = 324,  M = 1000, dt 1.0 fs, 300 K
  ch1m       2 blocks (C and H), D = 1224, M = 4000 each, dt 0.5 fs, 300 K
  cells512   512 independent C cells (64-2048 atoms, 1.5-3.5 g/cm3), 1 block D = 324,
             M = 2000; one step = energies and forces of every cell (batched)
  ch32k_trivial  the ch32k structure and seeds with both blocks under the
             "trivial" SOAP compression (D = 279 of 1224), M = 4000 each
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, List

import numpy as np

from . import synth
from .hypers import GapBlock, SoapTurboHypers, carbon_hypers, ch_hypers, trivial_compression


@dataclass
class Workload:
    name: str
    index: int                    # seed base 1000 + index
    hypers: List[SoapTurboHypers]
    n_sparse: List[int]
    dt: float
    temperature: float
    description: str
    source: Callable[[int], synth.Structure] = field(repr=False, default=None)

    @property
    def seed(self) -> int:
        return 1000 + self.index

    def structure(self, replica: int = 0) -> synth.Structure:
        if replica == 0:
            if self.name in synth.WORKLOAD_NAMES:
                return synth.workload_structure(self.name)
            return self.source(self.seed)
        return self.source(self.seed * 100 + 50 + replica)


def _ch(n: int, seed: int) -> synth.Structure:
    return synth.random_structure(n, (n / 0.12) ** (1 / 3), 1.0, seed=seed, h_fraction=0.25)


def _c(n: int, seed: int, rho: float = 2.0) -> synth.Structure:
    L = (n / synth.carbon_number_density(rho)) ** (1 / 3)
    return synth.random_structure(n, L, 1.2, seed=seed)


WORKLOADS = {
    "carbon216": Workload("carbon216", 0, [carbon_hypers()], [1000], 1.0, 300.0,
                          "216 C, L=12.91 A (2.0 g/cm3), poly3 n_max 8 l_max 8 (D=324), "
                          "zeta 4, delta 1, M=1000", source=lambda s: _c(216, s)),
    "ch32k": Workload("ch32k", 1, [ch_hypers(1), ch_hypers(2)], [4000, 4000], 1.0, 300.0,
                      "32768 atoms C:H=3:1 at 0.12 /A3, two blocks (C, H centres) n_max 8+8 "
                      "l_max 8 (D=1224 each), zeta 4, M=4000 per block",
                      source=lambda s: _ch(32768, s)),
    "ch16k": Workload("ch16k", 5, [ch_hypers(1), ch_hypers(2)], [4000, 4000], 1.0, 300.0,
                      "16384 atoms C:H=3:1 at 0.12 /A3, ch32k blocks (D=1224, M=4000 per "
                      "block); the small case for full profiler captures",
                      source=lambda s: _ch(16384, s)),
    "carbon131k": Workload("carbon131k", 3, [carbon_hypers()], [1000], 1.0, 300.0,
                           "131072 C at 2.0 g/cm3, D=324, M=1000",
                           source=lambda s: _c(131072, s)),
    "ch1m": Workload("ch1m", 4, [ch_hypers(1), ch_hypers(2)], [4000, 4000], 0.5, 300.0,
                     "1048576 atoms C:H=3:1 at 0.12 /A3, D=1224 per block, M=4000 per block",
                     source=lambda s: _ch(1048576, s)),
}


def _trivial(h: SoapTurboHypers) -> SoapTurboHypers:
    h.compress = trivial_compression(h.alpha_max, h.l_max)
    return h


WORKLOADS["ch32k_trivial"] = Workload(
    "ch32k_trivial", 1, [_trivial(ch_hypers(1)), _trivial(ch_hypers(2))], [4000, 4000], 1.0,
    300.0, "the ch32k structure with both blocks under the trivial SOAP compression "
    "(D=279 of 1224 each), zeta 4, M=4000 per block", source=lambda s: _ch(32768, s))


def uneven_cells(n_cells: int, seed: int):
    """Independent C cells: atoms log-uniform in 64..2048, density uniform in
    1.5..3.5 g/cm3, minimum distance 1.2 A (seeded)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_cells):
        n = int(round(np.exp(rng.uniform(np.log(64), np.log(2048)))))
        rho = rng.uniform(1.5, 3.5)
        L = (n / synth.carbon_number_density(rho)) ** (1 / 3)
        out.append(synth.random_structure(n, L, 1.2, seed=seed * 1000 + k))
    return out


WORKLOADS["cells512"] = Workload(
    "cells512", 2, [carbon_hypers()], [2000], 1.0, 300.0,
    "512 independent C cells, atoms log-uniform 64-2048, 1.5-3.5 g/cm3, D=324, M=2000; "
    "energies and forces of all cells per step (batched)",
    source=lambda s: _c(216, s))


def _source_structures(w: Workload):
    """Further seeded structures of the workload's kind, for the sparse sets."""
    if w.name in ("carbon216",):
        return [w.source(w.seed * 100 + i) for i in range(5)]
    if w.name == "cells512":
        return [_c(1000, w.seed * 100 + i, rho=2.0 + 0.5 * i) for i in range(3)]
    if w.name == "carbon131k":
        return [_c(4096, w.seed * 100 + i) for i in range(1)]
    return [_ch(32768, w.seed * 100 + 0)]


def unit_cells(box: np.ndarray, rcut: float) -> np.ndarray:
    """number_of_unit_cells_for_given_cutoff for orthorhombic boxes."""
    L = np.diag(box)
    return np.maximum(1, np.ceil(2.0 * rcut / L - 1e-12)).astype(np.int32)


def supercell(st: synth.Structure, ind) -> tuple:
    """read_files.f90:347-363 replica order (a-index slowest)."""
    reps = []
    for i2 in range(ind[0]):
        for j2 in range(ind[1]):
            for k2 in range(ind[2]):
                reps.append(st.positions + i2 * st.box[0] + j2 * st.box[1] + k2 * st.box[2])
    return np.concatenate(reps), np.tile(st.species, int(np.prod(ind)))


def descriptors_gpu(backend, h: SoapTurboHypers, st: synth.Structure, key: int) -> np.ndarray:
    """q of the central atoms of ``st`` for block hypers ``h`` through the backend."""
    dummy = GapBlock(h, np.zeros((1, h.dim)), np.zeros(1))
    backend.soap_backend_begin(dummy, key=key)
    ind = unit_cells(st.box, h.rcut_max)
    pos_sc, sp_sc = supercell(st, ind)
    box = st.box * ind[:, None]
    nl = backend.build_neighbors_list(pos_sc, st.n, box[0], box[1], box[2], h.rcut_max, ind, sp_sc)
    q = backend.get_soap(st.n, nl["n_neigh"], nl["neighbors_list"], nl["rjs"], nl["xyz"],
                         st.species, st.species, h.dim)
    backend.soap_backend_end()
    return q


def build_blocks(w: Workload, describe: Callable[[SoapTurboHypers, synth.Structure], np.ndarray]
                 ) -> List[GapBlock]:
    """Sparse-set blocks of a workload; ``describe(h, structure)`` returns the q rows
    of the structure's central atoms (the backend on the GPU arm, the oracle on the
    CPU reference arm)."""
    blocks = []
    sources = _source_structures(w)
    for b, (h, M) in enumerate(zip(w.hypers, w.n_sparse)):
        qs = np.concatenate([describe(h, st) for st in sources])
        rng = np.random.default_rng(w.seed * 100 + 90 + b)
        pick = rng.choice(len(qs), size=M, replace=False)
        alphas = synth.sparse_alphas(M, seed=w.seed * 100 + 95 + b)
        blocks.append(GapBlock(h, qs[pick], alphas, delta=1.0, zeta=4.0))
    return blocks
