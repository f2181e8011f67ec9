"""Training data for the learned surrogate of the mixed form.

The ensembles learn from (q, E_GAP, dE/dq) triples that the exact GAP path
produces during NVE MD of separate, smaller cells of the target's kind at a
spread of temperatures, not from the structure they are then run on:

  * carbon: cells of 216 to 4,096 C atoms at 2.0 g/cm3 (minimum distance 1.2 A);
  * C/H:    cells of 216 to 4,096 atoms, C:H = 3:1 at 0.12 atoms/A3 (1.0 A);

sizes log-uniform over the range, temperatures log-uniform over 300-5,000 K
(Maxwell velocities, centre of mass removed), a snapshot every ``stride`` steps
until the cell's share of the sample budget is reached. Every snapshot adds one
triple per central site of every block (tg_mlp_add_engine_samples).
"""
from __future__ import annotations

import os
import time
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

from . import synth


@dataclass
class Cell:
    structure: synth.Structure
    temperature: float


def training_cells(kind: str, n_cells: int, seed: int, sizes=(216, 4096),
                   temperatures=(300.0, 5000.0)) -> List[Cell]:
    """Seeded cells of the given kind ("C" or "CH") with log-uniform sizes and
    temperatures."""
    rng = np.random.default_rng(seed)
    lo, hi = np.log(sizes[0]), np.log(sizes[1])
    tlo, thi = np.log(temperatures[0]), np.log(temperatures[1])
    out = []
    for k in range(n_cells):
        n = int(round(np.exp(rng.uniform(lo, hi))))
        T = float(np.exp(rng.uniform(tlo, thi)))
        s = seed * 1000 + k
        if kind == "C":
            L = (n / synth.carbon_number_density(2.0)) ** (1 / 3)
            st = synth.random_structure(n, L, 1.2, seed=s)
        elif kind == "CH":
            st = synth.random_structure(n, (n / 0.12) ** (1 / 3), 1.0, seed=s, h_fraction=0.25)
        else:
            raise ValueError(f"unknown cell kind {kind!r}")
        out.append(Cell(st, T))
    return out


def collect(backend, mlps: Sequence, keys: Sequence[int], cells: Sequence[Cell],
            n_samples: int, dt: float, stride: int = 2, seed: int = 0,
            max_steps_per_cell: int = 4000) -> dict:
    """Runs exact GAP MD of every cell and adds a snapshot's triples to the
    ensembles (mlps[i] learns block i) every ``stride`` steps, until about
    n_samples site triples (all blocks together) are collected, spread evenly
    over the cells. Returns what was collected."""
    t0 = time.time()
    quota = int(np.ceil(n_samples / max(len(cells), 1)))
    snapshots, steps, skipped = 0, 0, 0
    old = os.environ.get("TGB_AUTOTUNE")
    os.environ["TGB_AUTOTUNE"] = "0"      # small cells: the default tiles
    try:
        for k, c in enumerate(cells):
            st = c.structure
            eng = backend.Engine(st.positions, st.species, st.masses, st.box, list(keys))
            try:
                eng.set_state(st.positions,
                              synth.maxwell_velocities(st.masses, c.temperature, seed + k))
                got, n_steps = 0, 0
                while got < quota and n_steps < max_steps_per_cell:
                    eng.md(stride, dt, energies=False)
                    n_steps += stride
                    for i, m in enumerate(mlps):
                        m.add_engine_samples(eng, i)
                    got += st.n
                    snapshots += 1
                steps += n_steps
            except RuntimeError:   # a cell whose MD left the device's bounds is dropped
                skipped += 1
            finally:
                eng.close()
    finally:
        if old is None:
            del os.environ["TGB_AUTOTUNE"]
        else:
            os.environ["TGB_AUTOTUNE"] = old
    return {"cells": len(cells), "skipped_cells": skipped, "snapshots": snapshots,
            "md_steps": steps, "samples": [int(m.n_samples()) for m in mlps],
            "seconds": time.time() - t0}
