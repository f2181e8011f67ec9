"""Build libtgb200.so in-tree with nvcc for sm_100a (B200).

    python -m turbogap_b200.build [--force] [--verbose]

Every CUDA translation unit is compiled for ``-gencode arch=compute_100a,code=sm_100a``
with ``-lineinfo``; the geometry/MD unit additionally with ``--fmad=false`` so its
FP64 arithmetic rounds like the reference Fortran. The shared library lands next
to this file (turbogap_b200/libtgb200.so) so it ships with the source tree.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libtgb200.so")

SOURCES = {
    "tgb_neighbors.cu": ["--fmad=false"],
    "tgb_soap.cu": [],
    "tgb_gemm.cu": [],
    "tgb_mlp.cu": [],
    "tgb_capi.cu": [],
    "tgb_noalloc.cu": ["--fmad=false"],
    "tgb_comm.cu": [],
    "tgb_family.cu": [],
    "tgb_vdw.cu": [],
}

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr",
          "-Xptxas", "-warn-spills"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found (CUDA toolkit required to build the backend)")


def _deps(src: str):
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps.append(os.path.join(ROOT, "include", "tgb200.h"))
    return [src] + deps


def _stale(out: str, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _compile(name: str, extra, force: bool, verbose: bool, ptxas_v: bool):
    src = os.path.join(CSRC, name)
    obj = os.path.join(BUILD, name.replace(".cu", ".o"))
    if not os.path.exists(src):
        return None
    if not force and not _stale(obj, _deps(src)):
        return obj
    cmd = [nvcc()] + ARCH + COMMON + extra + (["-Xptxas", "-v"] if ptxas_v else []) + [
        "-I", os.path.join(ROOT, "include"), "-c", src, "-o", obj]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {name}:\n{r.stdout}\n{r.stderr}")
    if verbose or ptxas_v:
        msg = (r.stdout + r.stderr).strip()
        if msg:
            print(msg, flush=True)
    return obj


def build(force: bool = False, verbose: bool = False, ptxas_v: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        futs = [ex.submit(_compile, n, e, force, verbose, ptxas_v) for n, e in SOURCES.items()]
        objs = [f.result() for f in futs]
    objs = [o for o in objs if o]
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static", "-ldl"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-v", action="store_true", help="print register/spill usage")
    a = ap.parse_args(argv)
    print(build(a.force, a.verbose, a.ptxas_v))
    return 0


if __name__ == "__main__":
    sys.exit(main())
