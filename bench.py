#!/usr/bin/env python
"""Benchmark of the wavefunction hot path: SCF (CG) iterations per second.

Workload: water32 -- 32 H2O at 1 g/cm^3 in an 18.63 bohr cubic box, PBE,
70 Ry (100^3 grid), 128 doubly occupied bands, GTH pseudopotentials, seeded
positions and a seeded initial wavefunction (synthetic: no dataset exists).
One step = one CG iteration of the reference's wfn_opt loop
(do_opt.f90:80-128): density, potentials, energies, H|psi>, Lambda, PCG,
Cholesky orthonormalisation, all on the GPU through libamdk.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
  python bench.py --impl reference ...   (the CPU restatement on the host cores)

Multi-GPU: the single-system path is not sharded (its only split is the
reference's slab all-to-all, not built); N ranks run N independent replicas
(weak scaling), value = total iterations of all ranks / max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SCF iter/s & MD step/s, 32 H2O: mixed vs FP64 GPU at ΔE≤1e-6 Ha/atom"
UNIT = "SCF iter/s"
WORKLOAD = "water32: 32 H2O, PBE, 70 Ry, 100^3 grid, 128 bands, GTH, Gamma"


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def setup_engine(precision: int, device: int):
    from amdkiit_b200 import configs
    from amdkiit_b200.engine import Engine
    from amdkiit_b200.guess import initial_coefficients
    s = configs.water32()
    e = Engine(s, precision=precision, device=device)
    g = e.gvectors()
    tp = 2.0 * np.pi / s.alat
    c0 = initial_coefficients(g["hg"][: e.ngpw] * tp * tp, e.nstate)
    e.set_wfn(c0)
    e.ortho()
    return s, e


def cpu_reference_iterations(steps: int, warmup: int, nthreads: int):
    """The CPU restatement (oracle) timed on the host cores: one step = one
    CG iteration of the same workload."""
    from amdkiit_b200 import configs
    from amdkiit_b200.guess import initial_coefficients
    from oracle.oracle import Oracle
    s = configs.water32()
    o = Oracle(s, nthreads)
    g = o.gvectors()
    c = initial_coefficients(g["hg"][: o.ngpw] * o.d("tpiba") ** 2, o.nstate)
    o.set_wfn(c)
    o.ortho()
    for i in range(1, warmup + 1):
        o.scf_iteration(i, 1e-6)
    t = time.perf_counter()
    for i in range(warmup + 1, warmup + steps + 1):
        o.scf_iteration(i, 1e-6)
    dt = time.perf_counter() - t
    return steps / dt, dt


def run_reference(args, rank):
    if rank != 0:
        return 0
    nth = os.cpu_count() or 1
    v, dt = cpu_reference_iterations(args.steps, args.warmup, nth)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * dt / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": "fp64", "l2": "working set > L2 (C0,C2,HNM1: 196 MB)"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": nth, "kind": "port",
                         "sample": f"{args.steps} CG iterations of water32 (after {args.warmup} warm-up), "
                                   "CPU restatement of the reference's FP64 path, OpenMP"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--md-steps", type=int, default=3)
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from amdkiit_b200.engine import FP64, MIXED
    prec = MIXED if args.precision == "mixed" else FP64
    s, e = setup_engine(prec, local)
    gcut = 1e-6
    for i in range(1, args.warmup + 1):
        e.scf_iteration(i, gcut)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    clk = ClockSampler(local)
    barrier()
    clk.start()
    e.profile(True)
    n0 = e.launch_count()
    dev_ms = 0.0
    t0 = time.perf_counter()
    for i in range(args.warmup + 1, args.warmup + args.steps + 1):
        en, gm, conv = e.scf_iteration(i, gcut)
        dev_ms += e.last_iteration_ms()
    wall = time.perf_counter() - t0
    launches = e.launch_count() - n0
    clocks = clk.stop()
    barrier()
    kern = {}
    for k, name in e.KERNELS.items():
        n, ms, b = e.profile_get(k)
        kern[name] = (n, ms, b)
    e.profile(False)
    tmax = dev_ms
    if dist:
        t = torch.tensor([dev_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tmax = float(t.item())
    value = world * args.steps / (tmax / 1000.0)

    # end to end through the C-ABI with host buffers: every step uploads C0
    # from pinned host memory, runs the iteration, reads C0 and the energies back
    c_host = torch.empty((e.nstate, e.ngpw), dtype=torch.complex128, pin_memory=True)
    c_np = c_host.numpy()
    e.get_wfn(out=c_np)
    barrier()
    t0 = time.perf_counter()
    ke = max(3, args.steps // 2)
    for i in range(args.warmup + args.steps + 1, args.warmup + args.steps + ke + 1):
        e.set_wfn(c_np)
        en2, gm2, _ = e.scf_iteration(i, gcut)
        e.get_wfn(out=c_np)
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    wfn_bytes = e.nstate * e.ngpw * 16

    # BOMD: velocity-Verlet steps (0.5 fs, 300 K, GRAD_CUTOFF 1e-6), each a
    # full wavefunction optimisation from the previous wavefunction
    md_line = None
    if args.md_steps > 0:
        from amdkiit_b200.md import BOMD
        md = BOMD(e, temperature=300.0, dt_fs=0.5, seed=2024, gcut=1e-6)
        md.start()
        e0 = md.total_energy()
        barrier()
        md_wall = md.run(args.md_steps)
        its = md.scf_iterations[1:]
        if dist:
            t = torch.tensor([md_wall], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            md_wall = float(t.item())
        md_line = {"steps_per_s": world * args.md_steps / md_wall, "unit": "MD step/s", "steps": args.md_steps,
                   "scf_iterations_per_step": float(np.mean(its)), "dt_fs": 0.5, "temperature_K": 300.0,
                   "grad_cutoff": 1e-6, "energy_drift_Ha": md.total_energy() - e0, "timing": "host wall clock"}

    # roofline of the dominant kernel class (CUDA events around its launches)
    dom = max(kern, key=lambda k: kern[k][1])
    n, ms, b = kern[dom]
    peak, src = peaks()
    achieved = (b / n) / ((ms / n) / 1000.0) / 1e9 if n else 0.0
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": tmax / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if prec == FP64 else "f32+f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": args.precision, "parallelism": f"replicas{world}",
                   "l2": "working set > L2 (C0, C2, CG direction: 196 MB resident)",
                   "energy_Ha": en["etotal"], "gemax": gm},
        "e2e": {"value": world * ke / e2e_s, "unit": UNIT, "h2d_bytes_per_step": wfn_bytes,
                "d2h_bytes_per_step": wfn_bytes + 9 * 8 + 8},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": src, "traffic": None,
                     "launches": n, "avg_launch_ms": ms / n if n else None},
        "kernels_ms": {k: round(v[1], 3) for k, v in kern.items()},
        "md": md_line,
        "clocks": clocks,
        "wall_ms_per_step": 1000.0 * wall / args.steps,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nth = os.cpu_count() or 1
        v, dt = cpu_reference_iterations(1, 0, nth)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": nth, "kind": "port",
                                "sample": "1 CG iteration of water32 (first iteration after ortho), CPU restatement, OpenMP"}
    e.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
