"""Command line: ``python -m turbogap_b200 {md,predict} <input> [--out DIR] [--device K]``.

Mirrors ``turbogap md <input>`` and ``turbogap predict <input>`` for decks that
stay on the device path (soap_turbo blocks, NVE velocity Verlet); thermo.log and
trajectory_out.xyz are written to DIR (default: the input file's directory).
"""
from __future__ import annotations

import argparse
import sys


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m turbogap_b200")
    ap.add_argument("mode", choices=("md", "predict"))
    ap.add_argument("input")
    ap.add_argument("--out", default=None)
    ap.add_argument("--device", type=int, default=0)
    a = ap.parse_args(argv)
    from . import backend, deck
    backend.gpu_context_init(0, a.device)
    try:
        if a.mode == "md":
            res = deck.run_md(a.input, a.out)
            print(f"{len(res['thermo'])} thermo rows -> {res['thermo_path']}; "
                  f"trajectory -> {res['trajectory_path']}")
        else:
            res = deck.run_predict(a.input, a.out)
            for k, r in enumerate(res):
                print(f"config {k + 1}: energy {r['energies'].sum():.8f} eV")
    finally:
        backend.gpu_context_finalize()
    return 0


if __name__ == "__main__":
    sys.exit(main())
