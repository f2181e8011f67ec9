#!/usr/bin/env python
"""SOAP-GAP E+F atom-steps/s on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload ch1m] [--precision bf16x3|bf16]

One step is one NVE velocity-Verlet MD step of the workload through the
device-resident engine: neighbour list rebuild, every soap_turbo block
(descriptor, tcgen05 GAP GEMMs, adjoint forces/virial), wrap_pbc,
remove_cm_vel and velocity_verlet, replayed from a CUDA graph. ``value`` is
atoms x steps / device time (CUDA events on the engine's stream, max over
ranks). ``e2e`` is the same metric through the public C-ABI with host buffers:
each step uploads the positions from pinned host memory and reads energies,
forces and virial back. N > 1 runs one independent replica per GPU (weak
scaling; no data-path collective); with ``--shard`` the ranks share ONE
structure by central-site ranges and sum forces, energies and the virial with
an NCCL all-reduce inside every step (strong scaling). ``--impl reference``
times the FP64 CPU port
of the reference path on the host cores (the Fortran reference cannot be built
here).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from turbogap_b200 import synth  # noqa: E402
from turbogap_b200.workloads import WORKLOADS, build_blocks, descriptors_gpu  # noqa: E402

# value: the plain (bf16x3, FP64-faithful) form; the line's "mixed" object holds
# the mixed+MLP form on the same workload with its error against the plain path
METRIC = "SOAP-GAP E+F atom-steps/s on 1 B200: plain vs mixed+MLP at \u22641 meV/atom"
UNIT = "atom-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="ch1m", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="bf16x3", choices=["bf16x3", "bf16"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=10)
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed (MLP + gate) leg")
    ap.add_argument("--mixed-steps", type=int, default=200)
    ap.add_argument("--mlp-samples", type=int, default=2000000,
                    help="(q, E, dE/dq) site triples the MLPs are trained on")
    ap.add_argument("--mlp-cells", type=int, default=16,
                    help="separate training cells of the workload's kind")
    ap.add_argument("--mlp-epochs", type=int, default=10)
    ap.add_argument("--mlp-hidden", type=int, default=0,
                    help="hidden width H of each member (D -> H -> H -> 1); 0: 64")
    ap.add_argument("--gate-ev", type=float, default=0.005)
    ap.add_argument("--shard", action="store_true",
                    help="N > 1: shard ONE structure over the ranks by central-site ranges "
                         "(in-step NCCL all-reduce; strong scaling) instead of N replicas")
    ap.add_argument("--neighbors-buffer", type=float, default=0.0,
                    help="list skin (A): lists kept until an atom moved sqrt(buffer/2); "
                         "0 (the reference default) rebuilds every step")
    return ap.parse_args()


# ------------------------------------------------------------------ helpers
class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-i", str(self.device), "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return world, rank, local, dist


def max_over_ranks(x, dist):
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gemm_flops_per_step(blocks, structure, sites_only=False):
    """Algorithmic FLOPs of ONE of the two GAP GEMMs per step: 2 D M per central
    atom (K = q.Q_s^T in GEMM 1, dE/dq in GEMM 2); the pair does 4 D M. With
    sites_only, the number of central sites over all blocks instead."""
    tot = 0
    for b in blocks:
        h = b.hypers
        zs = set(h.species_z) if h.central_species == 0 else {h.species_z[h.central_species - 1]}
        nb = int(np.isin(structure.species, list(zs)).sum())
        tot += nb if sites_only else 2 * h.dim * b.n_sparse * nb
    return tot


# DRAM bytes per central site of one GEMM launch, from the ncu capture of the
# 12288-site C block of ch16k (dram__bytes_read.sum + dram__bytes_write.sum
# divided by its sites); traffic grows with the sites at fixed D and M.
GEMM1_DRAM_BYTES_PER_SITE = (222.311424e6 + 264.274176e6) / 12288
GEMM2_DRAM_BYTES_PER_SITE = (417.493760e6 + 42.420736e6) / 12288


# ------------------------------------------------------------------ mixed form
def mixed_leg(B, eng, blocks, keys, w, a, ext, dist, plain_ms):
    """The mixed form: per block a 4-member MLP ensemble replaces the GAP GEMMs;
    sites whose ensemble spread exceeds the gate go back to the exact kernel.
    The ensembles are trained on the GPU from about 2M (q, E, dE/dq) triples of
    exact GAP MD of separate cells of the workload's kind (216-4096 atoms,
    300-5000 K; turbogap_b200.learned), never from the benchmark structure.
    Accuracy is measured on the benchmark structure against the exact bf16x3
    path (which matches the FP64 oracle to 1e-6 eV/atom), on a hot held-out
    cell, and against the oracle itself in the parity leg."""
    import torch
    from turbogap_b200 import learned
    t0 = time.time()
    hidden = [a.mlp_hidden or 64 for b in blocks]
    mlps = [B.Mlp(b.hypers.device_dim, hidden[i], 4, seed=100 + i) for i, b in enumerate(blocks)]
    kind = "CH" if len(blocks) > 1 else "C"
    cells = learned.training_cells(kind, a.mlp_cells, seed=w.seed * 100 + 61)
    data = learned.collect(B, mlps, keys, cells, a.mlp_samples, dt=w.dt, stride=2, seed=17)
    t_data = time.time() - t0
    losses = [m.train(a.mlp_epochs, batch=512, lr=1e-3, force_weight=1.0, seed=7 + i)
              for i, m in enumerate(mlps)]
    t_train = time.time() - t0 - t_data

    def errors():
        for i in range(len(mlps)):
            B.engine_set_mlp(eng, i, None)
        e_ref, f_ref, _ = eng.compute()
        for i, m in enumerate(mlps):
            B.engine_set_mlp(eng, i, m, gate_ev=a.gate_ev)
        e_mix, f_mix, _ = eng.compute()
        gated = sum(B.engine_mlp_stats(eng, i)[0] for i in range(len(mlps)))
        return (float(np.sqrt(np.mean((e_mix - e_ref) ** 2))),
                float(np.sqrt(np.mean((f_mix - f_ref) ** 2))), gated)

    err_fresh = errors()                    # the benchmark structure: never in the training data
    eng.md(max(a.warmup, 3), w.dt, energies=False)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    eng.md(a.mixed_steps, w.dt, energies=False)
    e1.record(ext)
    e1.synchronize()
    t_max = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist)
    prof = eng.profile(3, w.dt)
    err_after = errors()                    # at the end of the mixed-form trajectory
    hot = _hot_cell(B, mlps, keys, kind, w, a.gate_ev)
    for i in range(len(mlps)):
        B.engine_set_mlp(eng, i, None)
    n = eng.n
    ms = 1e3 * t_max / a.mixed_steps
    out = {
        "value": n * a.mixed_steps * (dist.get_world_size() if dist else 1) / t_max,
        "unit": UNIT, "ms_per_step": ms, "steps": a.mixed_steps,
        "speedup_vs_plain": plain_ms / ms,
        "gate_ev": a.gate_ev,
        "rmse_e_mev_per_atom": 1e3 * err_fresh[0], "rmse_f_mev_per_A": 1e3 * err_fresh[1],
        "gated_sites": err_fresh[2], "sites": n,
        "after_mixed_md": {"rmse_e_mev_per_atom": 1e3 * err_after[0],
                           "rmse_f_mev_per_A": 1e3 * err_after[1], "gated_sites": err_after[2]},
        "reference": "exact bf16x3 GPU path at the same configurations (the benchmark "
                     "structure is not in the training data)",
        "mlp": f"4 members x (D -> H -> H -> 1, SiLU) per block, H = {hidden}, bf16 GEMMs, "
               f"fp32 accumulation",
        "training": {"samples": [m.n_samples() for m in mlps], "protocol":
                     f"exact GAP NVE MD of {data['cells']} separate {kind} cells, 216-4096 "
                     f"atoms, 300-5000 K, a snapshot every 2 steps", "data": data,
                     "epochs": a.mlp_epochs,
                     "batch": 512, "data_seconds": t_data, "train_seconds": t_train,
                     "final_loss": [float(l_[-1]) for l_ in losses]},
        "held_out_cells": hot,
        "ms_per_step_by_pass": prof,
    }
    return out, mlps


def _hot_cell(B, mlps, keys, kind, w, gate_ev):
    """Two held-out 4096-atom cells of the training kind, against the exact path
    with the mixed form's gate: one after 20 NVE steps from 5000 K (inside the
    training range), and one at 1.6 times the density (outside it, where the
    ensemble's spread should send sites back to the exact kernel)."""
    from turbogap_b200 import learned
    out = {}
    for name, dens, T in (("hot_5000K", 1.0, 5000.0), ("dense_1.6x", 1.6, 300.0)):
        c = learned.training_cells(kind, 1, seed=w.seed * 100 + 77, sizes=(4096, 4096),
                                   temperatures=(T, T))[0]
        st = c.structure
        if dens != 1.0:   # the same atoms in a box scaled to the new density
            f = dens ** (-1.0 / 3.0)
            st = synth.Structure(st.positions * f, st.species, st.box * f)
        e2 = B.Engine(st.positions, st.species, st.masses, st.box, list(keys))
        try:
            e2.set_state(st.positions, synth.maxwell_velocities(st.masses, T, 5))
            e2.md(20, w.dt, energies=False)
            er, fr, _ = e2.compute()
            for i, m in enumerate(mlps):
                B.engine_set_mlp(e2, i, m, gate_ev=gate_ev)
            em, fm, _ = e2.compute()
            gated = sum(B.engine_mlp_stats(e2, i)[0] for i in range(len(mlps)))
            for i, m in enumerate(mlps):
                B.engine_set_mlp(e2, i, m, gate_ev=1e9)   # no gate: the networks alone
            eu, fu, _ = e2.compute()
        finally:
            e2.close()
        rms = lambda x: 1e3 * float(np.sqrt(np.mean(np.square(x))))   # noqa: E731
        out[name] = {"atoms": st.n, "density_factor": dens, "temperature_K": T,
                     "md_steps": 20, "gated_sites": int(gated),
                     "rmse_e_mev_per_atom": rms(em - er), "rmse_f_mev_per_A": rms(fm - fr),
                     "ungated": {"rmse_e_mev_per_atom": rms(eu - er),
                                 "rmse_f_mev_per_A": rms(fu - fr)}}
    return out


# ------------------------------------------------------------------ CPU (oracle)
def oracle_blocks(w):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from _util import oracle_descriptors
    return build_blocks(w, lambda h, st: oracle_descriptors(st, h)[0])


def time_oracle_sample(O, st, blocks, n_sites):
    t0 = time.perf_counter()
    O.evaluate(st.positions, st.species, st.box, blocks, site_range=(0, n_sites))
    return time.perf_counter() - t0


def calibrate_sample(O, st, blocks, target_s):
    """(n, per-site seconds, fixed seconds) for a share of central sites 0..n-1
    whose per-site work takes about target_s with the oracle's current threads.
    Two sample sizes far enough apart that the per-site part dominates the noise
    of the fixed, structure-wide part of a call (the cell grid over every atom);
    the sample stays bounded whatever the estimate says."""
    na, nb = min(256, st.n), min(1280, st.n)
    t_a = time_oracle_sample(O, st, blocks, na)
    t_b = time_oracle_sample(O, st, blocks, nb)
    per = (t_b - t_a) / (nb - na) if nb > na else 0.0
    if not per > 0.0:
        per = t_b / nb                      # an upper bound on the per-site cost
    fixed = min(max(t_a - na * per, 0.0), t_a)
    n_max = min(st.n, max(nb, int(3 * target_s / (t_b / nb))))
    return int(max(na, min(n_max, round(target_s / per)))), per, fixed


def cpu_baseline_leg(w, st, blocks, target_s=15.0, single_core_s=5.0):
    """The FP64 oracle port on the host cores: E+F of central sites 0..n-1 of the
    workload's structure (one MPI rank's share, all blocks, the share's lists),
    with the sparse sets the GPU arm uses, so the same share on the GPU is a
    parity check. The sample is sized to about target_s; the rate is sites per
    second, a full step of the structure taking N / rate. Also a single-thread
    rate on a smaller share. Returns the cpu_baseline object and the oracle's
    share (n, energies, forces, virial)."""
    import oracle as O
    cores = O.set_threads(0)
    n, per, fixed = calibrate_sample(O, st, blocks, target_s)
    t0 = time.perf_counter()
    e, f, v, _ = O.evaluate(st.positions, st.species, st.box, blocks, site_range=(0, n))
    t = time.perf_counter() - t0
    O.set_threads(1)
    try:   # one thread: the same two-point split of a smaller share
        n1b = int(max(32, min(n, 512, round(single_core_s / (per * cores)))))
        t1a = time_oracle_sample(O, st, blocks, 16)
        t1 = time_oracle_sample(O, st, blocks, n1b)
        n1 = n1b
        per1 = (t1 - t1a) / max(n1b - 16, 1)
        if not per1 > 0.0:
            per1 = t1 / n1b
    finally:
        O.set_threads(cores)
    rate = n / max(t - fixed, 1e-9)
    rate1 = 1.0 / per1
    cpu = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
           "sample": f"E+F of central sites 0..{n - 1} of the {w.name} structure (one MPI "
                     f"rank's share, all blocks), FP64 oracle port, {cores} OpenMP threads: "
                     f"{t:.1f} s, of which {fixed:.2f} s is the structure-wide cell grid; the "
                     f"rate is sites per second of the per-site work, so a full step of the "
                     f"{st.n}-atom structure would take about {st.n / rate + fixed:.0f} s",
           "host_cpu": _host_cpu(),
           "single_core": {"value": rate1, "unit": UNIT, "cores": 1,
                           "sample": f"central sites 0..{n1 - 1} against 0..15, 1 thread, "
                                     f"{t1:.1f} s; the per-site slope"}}
    return cpu, (n, e, f, v)


def _host_cpu():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def parity_leg(B, eng, st, oracle_share, blocks, keys, mlps, gate_ev):
    """The plain form against the FP64 oracle on the CPU baseline's share (the
    same central sites, the same structure and sparse sets): max |dE| per site,
    max |dF| over the share's force contributions, the virial relative to its
    largest component. The mixed form on the same share (energy RMSE over the
    share's sites), and the mixed form's full-force RMSE on a held-out cell of
    the workload's kind (2048 atoms, another seed), where the oracle evaluates
    every site."""
    import oracle as O
    n, eo, fo, vo = oracle_share
    eng.set_state(st.positions, np.zeros_like(st.positions))
    eng.set_site_range(0, n)
    e, f, v = eng.compute()
    out = {"sites": n, "structure": "the benchmark structure at its initial positions",
           "max_dE_eV_per_atom": float(np.abs(e - eo)[:n].max()),
           "max_dF_eV_per_A": float(np.abs(f - fo).max()),
           "virial_rel": float(np.abs(v - vo).max() / max(np.abs(vo).max(), 1e-300)),
           "virial_dev_eV_per_atom": float(np.abs(v - vo).max() / n),
           "bounds": {"dE_eV_per_atom": 1e-6, "dF_eV_per_A": 1e-6,
                      "virial_dev_eV_per_atom": 1e-6}}
    if mlps:
        for i, m in enumerate(mlps):
            B.engine_set_mlp(eng, i, m, gate_ev=gate_ev)
        em, fm, _ = eng.compute()
        gated = sum(B.engine_mlp_stats(eng, i)[0] for i in range(len(mlps)))
        for i in range(len(mlps)):
            B.engine_set_mlp(eng, i, None)
        out["mixed_share"] = {"rmse_e_mev_per_atom": 1e3 * float(np.sqrt(np.mean((em - eo)[:n] ** 2))),
                              "max_e_mev_per_atom": 1e3 * float(np.abs(em - eo)[:n].max()),
                              "gated_sites": int(gated)}
        # held-out cell: full forces
        held = _held_out_cell(st)
        if held is not None:
            eh, fh, _, _ = O.evaluate(held.positions, held.species, held.box, blocks)
            e2 = B.Engine(held.positions, held.species, held.masses, held.box, keys)
            ep, fp, _ = e2.compute()
            for i, m in enumerate(mlps):
                B.engine_set_mlp(e2, i, m, gate_ev=gate_ev)
            em2, fm2, _ = e2.compute()
            g2 = sum(B.engine_mlp_stats(e2, i)[0] for i in range(len(mlps)))
            e2.close()
            out["held_out_cell"] = {
                "atoms": held.n,
                "plain_max_dE_eV_per_atom": float(np.abs(ep - eh).max()),
                "plain_max_dF_eV_per_A": float(np.abs(fp - fh).max()),
                "mixed_rmse_e_mev_per_atom": 1e3 * float(np.sqrt(np.mean((em2 - eh) ** 2))),
                "mixed_rmse_f_mev_per_A": 1e3 * float(np.sqrt(np.mean((fm2 - fh) ** 2))),
                "mixed_gated_sites": int(g2),
                "mixed_bounds": {"rmse_e_mev_per_atom": 1.0, "rmse_f_mev_per_A": 30.0}}
    eng.set_site_range(0, st.n)
    return out


def _held_out_cell(st):
    """A 2048-atom cell of the benchmark structure's kind (density, composition,
    minimum distance), from another seed; None for kinds not covered."""
    n = 2048
    dens = st.n / abs(np.linalg.det(st.box))
    hfrac = float(np.mean(st.species == 2))
    dmin = 1.0 if hfrac > 0 else 1.2
    return synth.random_structure(n, (n / dens) ** (1 / 3), dmin, seed=777001,
                                  h_fraction=round(hfrac, 4))


def run_reference_batch(a, w, world):
    cells = batch_cells(w)
    for _ in range(a.warmup):
        oracle_batch_sample(w, cells[:1], 0.0)
    atoms, t, k = 0, 0.0, 0
    for _ in range(a.steps):
        na, tt, k = oracle_batch_sample(w, cells, 2.0)
        atoms += na
        t += tt
    value = atoms / t
    cores = os.cpu_count()
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * t / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": {"workload": f"{w.name}: {w.description}",
                                        "sample_cells": k},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"each step: E+F of the first {k} cells, FP64 port of the "
                                   f"reference CPU path; the Fortran reference cannot be built here"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)
    return 0


def run_reference(a):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import oracle as O
    w = WORKLOADS[a.workload]
    if w.name in BATCH_WORKLOADS:
        return run_reference_batch(a, w, world)
    st = w.structure()
    blocks = oracle_blocks(w)
    n, per, fixed = calibrate_sample(O, st, blocks, 2.0)
    for _ in range(a.warmup):
        time_oracle_sample(O, st, blocks, n)
    # each step evaluates the share 0..n-1; a full step of the N-atom structure on
    # these cores is fixed + N x (the step's per-site time), the rate N / that
    t_full = 0.0
    t_sample = 0.0
    for _ in range(a.steps):
        ts = time_oracle_sample(O, st, blocks, n)
        t_sample += ts
        t_full += fixed + st.n * max(ts - fixed, 1e-9) / n
    value = st.n * a.steps / t_full
    cores = os.cpu_count()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * t_full / a.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": f"{w.name}: {w.description}", "sample_sites": n},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"each step: E+F of central sites 0..{n - 1} of {w.name} "
                                   f"(one MPI rank's share, {t_sample / a.steps:.2f} s, of which "
                                   f"{fixed:.2f} s is the structure-wide cell grid), FP64 port "
                                   f"of the reference CPU path on {cores} threads; the full "
                                   f"{st.n}-atom step is that grid plus {st.n} sites at the "
                                   f"step's per-site time; the Fortran reference cannot be "
                                   f"built here"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------ batches
BATCH_WORKLOADS = {"cells512": 512}


def batch_cells(w, replica=0):
    from turbogap_b200.workloads import uneven_cells
    return uneven_cells(BATCH_WORKLOADS[w.name], w.seed + 7919 * replica)


def oracle_batch_sample(w, cells, target_s):
    """Oracle E+F of the first cells until about target_s of CPU time."""
    import oracle as O
    blocks = oracle_blocks(w)
    t, atoms, k = 0.0, 0, 0
    while k < len(cells) and t < target_s:
        st = cells[k]
        t0 = time.perf_counter()
        O.evaluate(st.positions, st.species, st.box, blocks)
        t += time.perf_counter() - t0
        atoms += st.n
        k += 1
    return atoms, t, k


def run_batch(a, w, world, rank, local, dist):
    """Energies and forces of every cell of a batch per step (no MD)."""
    import torch
    from turbogap_b200 import backend as B
    torch.cuda.set_device(local)
    B.gpu_context_init(rank, local)
    blocks = build_blocks(w, lambda h, st: descriptors_gpu(B, h, st, key=900))
    keys = []
    for i, b in enumerate(blocks):
        B.soap_backend_begin(b, key=i + 1)
        keys.append(i + 1)
    cells = batch_cells(w, rank)
    bat = B.Batch(cells, keys)
    n = bat.n
    ext = torch.cuda.ExternalStream(bat.stream())
    for _ in range(max(a.warmup, 3)):
        bat.compute_device()
    kernels = bat.graph_kernels()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(ext)
        for _ in range(a.steps):
            bat.compute_device()
        e1.record(ext)
        e1.synchronize()
    t_max = max_over_ranks(e0.elapsed_time(e1) / 1e3, dist)
    value = n * a.steps * world / t_max
    prof = bat.profile(a.profile_steps)
    peaks, peak_kind = measured_peaks()
    peak = float(peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops")))
    h = blocks[0].hypers
    flops = 2 * h.dim * blocks[0].n_sparse * n
    achieved = flops / (prof["gemm1"] / 1e3) / 1e12
    # e2e: host positions in, host energies / forces / virials out, every step
    pos = np.ascontiguousarray(np.concatenate([c.positions for c in cells]))
    pos_h = torch.from_numpy(pos).pin_memory()
    en_h = torch.empty(n, dtype=torch.float64, pin_memory=True)
    f_h = torch.empty((n, 3), dtype=torch.float64, pin_memory=True)
    v_h = torch.empty((len(cells), 9), dtype=torch.float64, pin_memory=True)
    lib = B.lib()
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(ext)
    for _ in range(a.e2e_steps):
        B.check(lib.tg_batch_set_positions(bat.handle, pos_h.numpy()))
        B.check(lib.tg_batch_compute(bat.handle, C.c_void_p(en_h.data_ptr()),
                                     C.c_void_p(f_h.data_ptr()), C.c_void_p(v_h.data_ptr())))
    e3.record(ext)
    e3.synchronize()
    t_e2e = max_over_ranks(e2.elapsed_time(e3) / 1e3, dist)
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        atoms, t, k = oracle_batch_sample(w, cells, 15.0)
        cpu = {"value": atoms / t, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": f"E+F of the first {k} cells ({atoms} atoms), FP64 oracle port, "
                         f"{os.cpu_count()} OpenMP threads, {t:.1f} s"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * t_max / a.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "bf16x3", "data": "synthetic",
        "config": {"workload": f"{w.name}: {w.description}", "cells": len(cells),
                   "atoms_per_gpu": n, "pairs": bat.n_pairs(),
                   "step": "energies, forces and virials of every cell (batched, one CUDA graph)",
                   "l2": "inputs larger than L2",
                   "soap_tiles": _tiles_desc(bat.tiles()),
                   "parallelism": f"{world} independent replica(s), one per GPU"},
        "roofline": {"kernel": "k_gemm_tn<GAP>: tcgen05 GEMM 1 (all cells' sites)", "bound": "tensor",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak, "traffic": None,
                     "peak_source": f"{peak_kind} bf16 dense (sustained), of measured",
                     "ms_per_step_by_pass": prof},
        "cpu_baseline": cpu,
        "e2e": {"value": n * a.e2e_steps * world / t_e2e, "unit": UNIT,
                "h2d_bytes_per_step": int(pos.nbytes),
                "d2h_bytes_per_step": int((en_h.numel() + f_h.numel() + v_h.numel()) * 8),
                "api": "tg_batch_set_positions + tg_batch_compute (host buffers)"},
        "gpu_launches": kernels * a.steps,
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    bat.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------------ GPU
def run_ours(a):
    world, rank, local, dist = dist_setup(a.gpus)
    if a.workload in BATCH_WORKLOADS:
        return run_batch(a, WORKLOADS[a.workload], world, rank, local, dist)
    import torch
    from turbogap_b200 import backend as B
    from turbogap_b200.workloads import descriptors_gpu

    torch.cuda.set_device(local)
    B.gpu_context_init(rank, local)
    w = WORKLOADS[a.workload]
    prec = B.TG_PREC_BF16X3 if a.precision == "bf16x3" else B.TG_PREC_BF16
    blocks = build_blocks(w, lambda h, st: descriptors_gpu(B, h, st, key=900))
    keys = []
    for i, b in enumerate(blocks):
        B.soap_backend_begin(b, key=i + 1, precision=prec)
        keys.append(i + 1)
    shard = a.shard and world > 1
    st = w.structure(replica=0 if shard else rank)
    eng = B.Engine(st.positions, st.species, st.masses, st.box, keys,
                   neighbors_buffer=a.neighbors_buffer)
    eng.set_state(st.positions, synth.maxwell_velocities(st.masses, w.temperature, w.seed))
    if shard:   # one structure over the ranks: central-site ranges, in-step NCCL all-reduce
        from turbogap_b200.parallel import shard_engine
        shard_engine(eng)
    n_pairs = eng.n_pairs()
    ext = torch.cuda.ExternalStream(eng.stream())

    # warm-up: first step eager, then the step graph is captured and replayed
    eng.md(max(a.warmup, 3), w.dt, energies=False)
    kernels_per_step = eng.graph_kernels()

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(ext)
        eng.md(a.steps, w.dt, energies=False)
        e1.record(ext)
        e1.synchronize()
    torch.cuda.synchronize()
    t_dev = e0.elapsed_time(e1) / 1e3
    t_max = max_over_ranks(t_dev, dist)
    # replicas: every rank steps its own structure; shard: the ranks step one
    value = st.n * a.steps * (1 if shard else world) / t_max
    clocks = clk.summary()

    # per-pass CUDA-event profile (eager steps on the same stream)
    prof = eng.profile(a.profile_steps, w.dt)
    peaks, peak_kind = measured_peaks()
    flops = gemm_flops_per_step(blocks, st)
    achieved = flops / (prof["gemm1"] / 1e3) / 1e12        # GEMM 1: the dominant kernel
    achieved2 = flops / (prof["gemm2"] / 1e3) / 1e12
    peak = float(peaks.get("bf16_tflops_sustained", peaks.get("bf16_tflops")))
    nsplit = 3 if a.precision == "bf16x3" else 1
    n_central = gemm_flops_per_step(blocks, st, sites_only=True)

    # e2e through the C-ABI with pinned host buffers
    n = st.n
    pos_h = torch.empty((n, 3), dtype=torch.float64, pin_memory=True)
    en_h = torch.empty(n, dtype=torch.float64, pin_memory=True)
    f_h = torch.empty((n, 3), dtype=torch.float64, pin_memory=True)
    v_h = torch.empty(9, dtype=torch.float64, pin_memory=True)
    p_now, _, _ = eng.get_state()
    pos_h.copy_(torch.from_numpy(p_now))
    lib = B.lib()
    h = eng.handle
    for _ in range(2):
        B.check(lib.tg_engine_set_state(h, C.c_void_p(pos_h.data_ptr()), None))
        B.check(lib.tg_engine_compute(h, C.c_void_p(en_h.data_ptr()), C.c_void_p(f_h.data_ptr()),
                                      C.c_void_p(v_h.data_ptr())))
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(ext)
    for _ in range(a.e2e_steps):
        B.check(lib.tg_engine_set_state(h, C.c_void_p(pos_h.data_ptr()), None))
        B.check(lib.tg_engine_compute(h, C.c_void_p(en_h.data_ptr()), C.c_void_p(f_h.data_ptr()),
                                      C.c_void_p(v_h.data_ptr())))
    e3.record(ext)
    e3.synchronize()
    t_e2e = max_over_ranks(e2.elapsed_time(e3) / 1e3, dist)
    e2e = {"value": n * a.e2e_steps * (1 if shard else world) / t_e2e, "unit": UNIT,
           "h2d_bytes_per_step": int(pos_h.numel() * 8),
           "d2h_bytes_per_step": int((en_h.numel() + f_h.numel() + v_h.numel()) * 8),
           "api": "tg_engine_set_state + tg_engine_compute (host positions in, host energies/"
                  "forces/virial out)"}

    mixed, mlps = None, []
    if not a.no_mixed and not shard:
        mixed, mlps = mixed_leg(B, eng, blocks, keys, w, a, ext, dist, 1e3 * t_max / a.steps)

    cpu, parity = None, None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            cpu, share = cpu_baseline_leg(w, st, blocks)
        except Exception as ex:  # keep the bench line even if the oracle cannot run
            cpu, share = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                          "sample": f"failed: {ex}"}, None
        if share is not None:
            parity = parity_leg(B, eng, st, share, blocks, keys, mlps, a.gate_ev)
    for m in mlps:
        m.close()

    # the per-site DRAM bytes were captured at D = 1224, M = 4000 (ch16k)
    same_gemm = all(b.hypers.dim == 1224 and b.n_sparse == 4000 for b in blocks)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1e3 * t_max / a.steps, "higher_is_better": True,
        "scaling": "strong" if shard else "weak", "vs_baseline": None, "dtype": a.precision,
        "data": "synthetic",
        "config": {"workload": f"{w.name}: {w.description}", "atoms_per_gpu": st.n,
                   "pairs": n_pairs, "dt_fs": w.dt, "md": "NVE velocity-Verlet, neighbour list " + (
                       "rebuilt every step" if a.neighbors_buffer <= 0 else
                       f"built to rcut + {a.neighbors_buffer} A, kept until an atom moved "
                       f"sqrt({a.neighbors_buffer}/2) A"), "precision": a.precision,
                   "l2": "inputs larger than L2 (GEMM operands and kd scratch > 126 MB)",
                   "soap_tiles": _tiles_desc(eng.tiles()),
                   "parallelism": (f"one structure over {world} GPUs: central-site ranges, "
                                   f"in-step NCCL all-reduce of forces, energies and virial"
                                   if shard else f"{world} independent replica(s), one per GPU")},
        "roofline": {"kernel": "k_gemm_tn<GAP>: tcgen05 GEMM 1, K = q.Q_s^T with the fused "
                               "K^zeta energy and kd epilogue (all blocks of a step)",
                     "bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak,
                     "traffic": GEMM1_DRAM_BYTES_PER_SITE * n_central if same_gemm else None,
                     "traffic_source": ("ncu dram bytes of the ch16k C-block launch, per site, "
                                        "times the central sites of a step") if same_gemm else
                                       "no capture at this D and M",
                     "peak_source": f"{peak_kind} bf16 dense (sustained), of measured",
                     "algorithmic_flops_per_step": flops,
                     "issue_rate_tflops": achieved * nsplit,
                     "gemm2": {"kernel": "k_gemm_tn<STORE>: dE/dq = (kd - kcoef).(Q_s - mu)",
                               "achieved": achieved2, "frac": achieved2 / peak,
                               "traffic": (GEMM2_DRAM_BYTES_PER_SITE * n_central
                                           if same_gemm else None),
                               "issue_rate_tflops": achieved2 * nsplit},
                     "ms_per_step_by_pass": prof},
        "cpu_baseline": cpu,
        "parity": parity,
        "mixed": mixed,
        "e2e": e2e,
        "gpu_launches": kernels_per_step * a.steps,
        "clocks": clocks,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def _tiles_desc(tiles):
    """Autotuned CTA tiles of the descriptor and force passes, per block."""
    name = {0: "4 sites/CTA, >=4 CTAs/SM", 1: "4 sites/CTA, >=3 CTAs/SM", 2: "2 sites/CTA, >=8 CTAs/SM",
            3: "8 sites/CTA, >=2 CTAs/SM", 4: "tensor cores (mma.sync TF32), 4 sites/CTA"}
    return [{"descriptor": name[a], "forces": name[b]} for a, b in tiles]


def main():
    a = parse()
    if a.impl == "reference":
        return run_reference(a)
    return run_ours(a)


if __name__ == "__main__":
    sys.exit(main())
