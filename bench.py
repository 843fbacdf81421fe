#!/usr/bin/env python
"""Benchmark of the wavefunction hot path: SCF (CG) iterations per second.

Workload: water32 -- 32 H2O at 1 g/cm^3 in an 18.63 bohr cubic box, PBE,
70 Ry (100^3 grid), 128 doubly occupied bands, GTH pseudopotentials, seeded
positions and a seeded initial wavefunction (synthetic: no dataset exists).
One step = one CG iteration of the reference's wfn_opt loop
(do_opt.f90:80-128): density, potentials, energies, H|psi>, Lambda, PCG,
Cholesky orthonormalisation, all on the GPU through libamdk.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision both|fp64|mixed]
  python bench.py --impl reference ...   (the CPU restatement on the host cores)

The default runs both precisions: `value` is the mixed-precision path
(FP32 band-pair FFTs, FP64 elsewhere), `mixed_vs_fp64` holds the FP64 path's
numbers, the speed-ups and the energy/force differences of the two paths at
the converged MD start (the metric's 1e-6 Ha/atom condition).

Multi-GPU: N ranks run N independent replicas of the CG iteration (weak
scaling), value = total iterations of all ranks / max rank time.  The
slab decomposition of the band-pair transforms (the reference's x-ray /
x-plane split with an all-to-all inside each FFT) is measured by
`--slab R,...`: under torchrun every rank holds its own slab and the
all-to-alls are NCCL's; on one GPU the R ranks are emulated in one process
(their launches one after the other, the exchange as copies) and the line
reports the largest rank's kernel time per phase with the bytes each rank
would send over NVLink.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SCF iter/s & MD step/s, 32 H2O: mixed vs FP64 GPU at ΔE≤1e-6 Ha/atom"
UNIT = "SCF iter/s"
WORKLOAD = "water32: 32 H2O, PBE, 70 Ry, 100^3 grid, 128 bands, GTH, Gamma"


# DRAM bytes (read + write) per launch of the dominant kernel classes, from
# one `ncu --set full` capture of each on this workload (one launch inside
# `bench.py --steps 3 --warmup 3 --md-steps 0`); None where none was taken.
PREDICTOR_POINTS = 5  # BOMD wavefunction predictor of the extrapolated MD line (Kolafa K = 3)
TRAFFIC = {("z_vpsi", "mixed"): 146.45e6, ("z_vpsi", "fp64"): 347.35e6, ("z_density", "mixed"): 142.22e6}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks, power and throttle reasons sampled every `period_s` on a
    background thread through NVML (nvidia-smi's own source of these
    figures), from start() to stop(): a bench arm brackets its timed
    iterations, the end-to-end iterations and the MD steps with it."""

    # NVML clocks-event reason bits (nvml.h nvmlClocksEventReason*)
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40}

    def __init__(self, gpu_index: int, period_s: float = 0.02):
        self.idx = gpu_index
        self.period = period_s
        self.samples = []
        self.max_mhz = None
        self._stop = threading.Event()
        self.t = None
        self.err = None

    def _handle(self):
        import pynvml
        pynvml.nvmlInit()
        idx = self.idx
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        parts = [x for x in vis.split(",") if x.strip()]
        if parts and all(x.strip().isdigit() for x in parts) and self.idx < len(parts):
            idx = int(parts[self.idx])
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(idx)

    def start(self):
        try:
            nv, h = self._handle()
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
        except Exception as exc:  # reported in the line, never fatal
            self.err = f"NVML unavailable: {exc}"
            return

        def loop():
            while not self._stop.is_set():
                try:
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                    self.samples.append((float(sm), int(rs), pw))
                except Exception as exc:
                    self.err = str(exc)
                    return
                self._stop.wait(self.period)
        self.t = threading.Thread(target=loop, daemon=True)
        self.t.start()

    def stop(self):
        if self.t is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [self.err or "no samples"], "samples": 0}
        self._stop.set()
        self.t.join(timeout=5)
        sm = [x[0] for x in self.samples]
        reasons = sorted(n for n, bit in self.REASONS.items() if any(x[1] & bit for x in self.samples))
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(sm), "period_ms": 1000.0 * self.period,
                "power_w_max": max((x[2] for x in self.samples), default=None),
                "window": "whole arm: timed, end-to-end and MD iterations"}


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


def cpu_reference_iterations(steps: int, warmup: int, nthreads: int, budget_s: float = 0.0):
    """The CPU restatement (oracle) timed on the host cores: one step = one
    CG iteration of the same workload.  With budget_s > 0 the timed loop stops
    once that much time has passed (at least one iteration)."""
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
    done = 0
    for i in range(warmup + 1, warmup + steps + 1):
        o.scf_iteration(i, 1e-6)
        done += 1
        if budget_s > 0 and time.perf_counter() - t >= budget_s:
            break
    dt = time.perf_counter() - t
    return done / dt, dt, done


# The CPU arm is bounded: one water32 iteration of the restatement takes
# seconds per core count, so it runs at most REF_WARMUP + REF_BUDGET_S worth
# of iterations whatever --steps asks for.
REF_WARMUP = 1
REF_STEPS = 20
REF_BUDGET_S = 30.0


def run_reference(args, rank):
    if rank != 0:
        return 0
    nth = os.cpu_count() or 1
    v, dt, done = cpu_reference_iterations(min(args.steps, REF_STEPS), min(args.warmup, REF_WARMUP), nth,
                                           REF_BUDGET_S)
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": done,
        "warmup": min(args.warmup, REF_WARMUP), "ms_per_step": 1000.0 * dt / done, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": "fp64", "l2": "working set > L2 (C0,C2,HNM1: 196 MB)"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": nth, "kind": "port",
                         "sample": f"{done} CG iterations of water32 (after {min(args.warmup, REF_WARMUP)} warm-up, "
                                   f"bounded at {REF_BUDGET_S:.0f} s of timed work), CPU restatement of the "
                                   "reference's FP64 path, OpenMP on all host threads"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(x: float, dist=None, device: str = "cuda") -> float:
    """Max of a per-rank time over all ranks (every rank takes this step)."""
    if not dist:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_arm(prec, args, local, dist, world):
    """One precision: timed SCF iterations (device time), the same iterations
    end to end through the C-ABI with host buffers, then BOMD steps.  Returns
    the measurements and the converged energy and forces of the MD start."""
    import torch
    from amdkiit_b200.engine import FP64
    s, e = setup_engine(prec, local)
    gcut = 1e-6
    for i in range(1, args.warmup + 1):
        e.scf_iteration(i, gcut)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    def tmax(x):
        return max_over_ranks(x, dist, "cuda")

    clk = ClockSampler(local)
    barrier()
    clk.start()   # stopped after the MD steps: the whole arm under load
    e.profile(True)
    n0 = e.launch_count()
    dev_ms = 0.0
    t0 = time.perf_counter()
    for i in range(args.warmup + 1, args.warmup + args.steps + 1):
        en, gm, conv = e.scf_iteration(i, gcut)
        dev_ms += e.last_iteration_ms()
    wall = time.perf_counter() - t0
    launches = e.launch_count() - n0
    barrier()
    kern = {name: e.profile_get(k) for k, name in e.KERNELS.items()}
    e.profile(False)
    dev_ms = tmax(dev_ms)

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
        e.scf_iteration(i, gcut)
        e.get_wfn(out=c_np)
    e2e_s = tmax(time.perf_counter() - t0)
    wfn_bytes = e.nstate * e.ngpw * 16

    # BOMD: velocity-Verlet steps (0.5 fs, 300 K, GRAD_CUTOFF 1e-6), each a
    # full wavefunction optimisation from the previous wavefunction
    md_line, e_conv, f_conv, eig_conv = None, None, None, None
    if args.md_steps > 0:
        from amdkiit_b200.md import BOMD
        md = BOMD(e, temperature=300.0, dt_fs=0.5, seed=2024, gcut=1e-6)
        md.start()
        e_conv, f_conv = md.energy, np.array(md.force)
        try:  # subspace eigenvalues at the converged start (this arm's precision)
            eig_conv = e.eigenvalues()
        except Exception as exc:  # reported, never fatal to the bench line
            eig_conv = str(exc)
        e0 = md.total_energy()
        etot = [e0]
        barrier()
        md_wall = tmax(md.run(args.md_steps, callback=lambda i, n, ep, et, T: etot.append(et)))
        its = md.scf_iterations[1:]
        md_line = {"steps_per_s": world * args.md_steps / md_wall, "unit": "MD step/s", "steps": args.md_steps,
                   "step_s_median": float(np.median(md.step_wall)), "step_s_mean": float(np.mean(md.step_wall)),
                   "scf_iterations_per_step": float(np.mean(its)), "dt_fs": 0.5, "temperature_K": 300.0,
                   "grad_cutoff": 1e-6, "energy_drift_Ha": md.total_energy() - e0,
                   "energy_fluctuation_Ha": float(np.max(np.abs(np.array(etot) - e0))),
                   "timing": "host wall clock per step (each step ends on a host synchronisation); "
                             "steps_per_s = steps / total"}
        # the same steps with the wavefunction predictor (an option outside
        # the reference's driver): reported beside, not as the MD number
        mdx = BOMD(e, temperature=300.0, dt_fs=0.5, seed=2024, gcut=1e-6, extrapolate=True,
                   predictor_points=PREDICTOR_POINTS)
        mdx.start()
        for _ in range(PREDICTOR_POINTS - 1):  # untimed: the predictor's history fills up
            mdx.step()
        barrier()
        nx = max(args.md_steps, 3)
        x_wall = tmax(mdx.run(nx))
        md_line["extrapolated"] = {"steps_per_s": world * nx / x_wall, "steps": nx,
                                   "step_s_median": float(np.median(mdx.step_wall)),
                                   "scf_iterations_per_step": float(np.mean(mdx.scf_iterations[PREDICTOR_POINTS:])),
                                   "predictor": f"always-stable predictor, {PREDICTOR_POINTS} points: "
                                                "C0(t+dt) = sum_j w_j C0(t-j dt) [C0(t-j dt)^T C0(t)], then ortho"}
    clocks = clk.stop()
    out = {"prec": prec, "nat": s.nat, "na": list(s.na), "value": world * args.steps / (dev_ms / 1000.0),
           "ms_per_step": dev_ms / args.steps, "wall_ms_per_step": 1000.0 * wall / args.steps,
           "launches": launches, "kern": kern, "clocks": clocks, "energy": en["etotal"], "gemax": gm,
           "e2e": {"value": world * ke / e2e_s, "unit": UNIT, "h2d_bytes_per_step": wfn_bytes,
                   "d2h_bytes_per_step": wfn_bytes + 9 * 8 + 8},
           "md": md_line, "e_conv": e_conv, "f_conv": f_conv, "eig_conv": eig_conv, "dtype": "f64" if prec == FP64 else "f32+f64"}
    e.close()
    return out


def config_report(args, local):
    """The other benchmark configurations (one JSON line): SCF iter/s of the
    FP64 and mixed paths, and the converged energy and force differences of
    the two (mixed with its FP64 refinement) from the same start."""
    from amdkiit_b200 import configs
    from amdkiit_b200.engine import FP64, MIXED, Engine
    from amdkiit_b200.guess import initial_coefficients

    def start(e, s):
        g = e.gvectors()
        tp = 2.0 * np.pi / s.alat
        return initial_coefficients(g["hg"][: e.ngpw] * tp * tp, e.nstate)

    def timed(e, n):
        for i in range(1, 4):
            e.scf_iteration(i, 1e-6)
        ms = 0.0
        for i in range(4, 4 + n):
            e.scf_iteration(i, 1e-6)
            ms += e.last_iteration_ms()
        return n / (ms / 1000.0)

    def one(name, s, steps):
        row = {"config": name, "grid": None, "nstate": s.nstate, "atoms": s.nat}
        res = {}
        for pname, prec in (("fp64", FP64), ("mixed", MIXED)):
            e = Engine(s, precision=prec, device=local)
            row["grid"] = list(e.nr)
            row["nstate"] = e.nstate
            c0 = start(e, s)
            e.set_wfn(c0)
            e.ortho()
            row[pname + "_scf_iter_per_s"] = timed(e, steps)
            e.set_wfn(c0)
            e.ortho()
            n, en, gm = e.wfn_opt(4000, 1e-6)
            res[pname] = (en["etotal"], e.get("force") if n > 1 else e.ionic_forces(), n)
            e.close()
        row["scf_speedup"] = row["mixed_scf_iter_per_s"] / row["fp64_scf_iter_per_s"]
        row["dE_Ha_per_atom"] = abs(res["mixed"][0] - res["fp64"][0]) / s.nat
        row["dF_max_Ha_per_bohr"] = float(np.max(np.abs(res["mixed"][1] - res["fp64"][1])))
        row["iterations_to_1e-6"] = {"fp64": res["fp64"][2], "mixed": res["mixed"][2]}
        return row

    rows = [one("cfg0 water1 (64^3, 4 bands)", configs.water1(), args.steps),
            one("cfg1 si64 (72^3, 128 bands)", configs.si64(), args.steps),
            one("cfg4 water128 (160^3, 512 bands)", configs.water128(), max(3, args.steps // 10))]
    # cfg2: 16 independent clusters.  The per-system FP64 loop iterates one
    # system after the other; the ensemble advances all 16 together, each CG
    # segment of all systems one CUDA graph launch (amdk_ensemble_iteration).
    # Device time; value = SCF iterations of all systems / time.
    from amdkiit_b200.engine import Ensemble
    ens = configs.ensemble()

    def engines(prec):
        out = []
        for s in ens:
            e = Engine(s, precision=prec, device=local)
            e.set_wfn(start(e, s))
            e.ortho()
            for i in range(1, 4):
                e.scf_iteration(i, 1e-6)
            out.append(e)
        return out

    ens_row = {"config": "cfg2 ensemble of 16 clusters", "systems": len(ens)}
    es = engines(FP64)
    ens_row["grids"] = sorted({tuple(e.nr) for e in es})
    loop_ms = 0.0
    for e in es:
        for i in range(4, 4 + args.steps):
            e.scf_iteration(i, 1e-6)
            loop_ms += e.last_iteration_ms()
    ens_row["fp64_loop_scf_iter_per_s"] = len(ens) * args.steps / (loop_ms / 1000.0)
    for e in es:
        e.close()
    for pname, prec in (("fp64", FP64), ("mixed", MIXED)):
        es = engines(prec)
        E = Ensemble(es)
        ms = 0.0
        for i in range(4, 4 + args.steps):
            E.iteration([i] * len(es), 1e-6)
            ms += E.last_ms()
        ens_row[pname + "_ensemble_scf_iter_per_s"] = len(ens) * args.steps / (ms / 1000.0)
        E.close()
        for e in es:
            e.close()
    ens_row["ensemble_mixed_vs_fp64_loop"] = ens_row["mixed_ensemble_scf_iter_per_s"] / ens_row["fp64_loop_scf_iter_per_s"]
    ens_row["timing"] = ("device time (CUDA events): the loop sums each system's iterations; the ensemble times "
                         "each iteration of all 16 systems (two graph launches)")
    rows.append(ens_row)
    print(json.dumps({"metric": METRIC, "report": "other configurations", "unit": UNIT, "rows": rows}), flush=True)
    return 0


def relax_report(args, local):
    """cfg4: water128 (160^3, 512 bands, PBE) relaxed by LBFGS from its
    perturbed start (geom_opt_lbfgs, do_opt.f90:197-266) in mixed precision
    (each geometry's CG ends in FP64), GRAD_CUTOFF 1e-6 for the wavefunction
    and 5e-4 Ha/bohr for the geometry.  The reference stops LBFGS on the
    2-norm of the gradient (lbfgs.f); the line reports that and the max
    force component.  One JSON line."""
    from amdkiit_b200 import configs
    from amdkiit_b200.engine import MIXED, Engine
    from amdkiit_b200.geo_opt import GeometryOptimizer
    from amdkiit_b200.guess import initial_coefficients
    s = configs.water128()
    e = Engine(s, precision=MIXED, device=local)
    g = e.gvectors()
    tp = 2.0 * np.pi / s.alat
    e.set_wfn(initial_coefficients(g["hg"][: e.ngpw] * tp * tp, e.nstate))
    e.ortho()
    opt = GeometryOptimizer(e, gcut_wfn=1e-6, gcut_geo=5e-4, max_step=args.relax_steps)
    evaluate = opt.energy_gradient

    def logged(x):  # one progress line per geometry on stderr (energy, max force, SCF iterations)
        out = evaluate(x)
        en, fmax, nscf = opt.evaluations[-1]
        print("relax evaluation %d: E %.8f Ha, max |F| %.3e Ha/bohr, %d SCF iterations, %.1f s"
              % (len(opt.evaluations), en, fmax, nscf, time.perf_counter() - t0), file=sys.stderr, flush=True)
        return out

    opt.energy_gradient = logged
    t0 = time.perf_counter()
    res, atco = opt.run()
    wall = time.perf_counter() - t0
    ev = opt.evaluations
    out = {"metric": "cfg4 LBFGS relaxation", "report": "water128 relaxation", "config": {
        "workload": "water128: 128 H2O, PBE, 70 Ry, 160^3 grid, 512 bands, GTH, perturbed +-0.1 bohr",
        "precision": "mixed (FP64 refinement at the end of each CG)"},
        "converged_2norm": bool(res.converged), "lbfgs_iterations": res.iterations, "evaluations": len(ev),
        "grad_2norm": float(np.linalg.norm(res.g)), "max_force": float(np.max(np.abs(res.g))),
        "max_force_below_5e-4": bool(np.max(np.abs(res.g)) < 5e-4), "energy_Ha": res.f,
        "start": {"energy_Ha": ev[0][0], "max_force": ev[0][1]},
        "scf_iterations_total": int(sum(x[2] for x in ev)), "wall_s": wall,
        "timing": "host wall clock of the whole relaxation"}
    print(json.dumps(out), flush=True)
    e.close()
    return 0


def cufft_compare(args, local):
    """H|psi> of water32's 64 band pairs (V(r)psi: the pair transforms of the
    pencil path with the sphere pack/unpack, kinetic term and nonlocal GEMM,
    through amdk_apply_h) beside cuFFT (torch.fft) doing only the full-grid
    part of the same work: backward 3D FFTs of 64 complex 100^3 grids, the
    multiply by V(r), forward 3D FFTs.  One JSON line; a comparison, not a
    path of the library."""
    import torch
    from amdkiit_b200.engine import FP64, MIXED
    torch.cuda.set_device(local)
    out = {"metric": "V(r)psi of 64 band pairs, water32 100^3 grid", "report": "cuFFT comparison", "unit": "ms"}
    for name, prec, cdt in (("fp64", FP64, torch.complex128), ("mixed", MIXED, torch.complex64)):
        s, e = setup_engine(prec, local)
        e.density()
        e.potential()
        for _ in range(3):
            e.apply_h()
        torch.cuda.synchronize()
        k = 20
        t0 = time.perf_counter()
        for _ in range(k):
            e.apply_h()
        torch.cuda.synchronize()
        ours = 1000.0 * (time.perf_counter() - t0) / k
        n = e.nr[0]
        T = e.nstate // 2
        e.close()
        g = torch.Generator(device="cuda").manual_seed(1)
        x = torch.randn((T, n, n, n), dtype=cdt, device="cuda", generator=g)
        v = torch.rand((n, n, n), dtype=torch.float64 if cdt == torch.complex128 else torch.float32, device="cuda",
                       generator=g)

        def step():
            y = torch.fft.ifftn(x, dim=(1, 2, 3))
            y *= v
            return torch.fft.fftn(y, dim=(1, 2, 3))

        for _ in range(3):
            step()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(k):
            step()
        b.record()
        torch.cuda.synchronize()
        out[name] = {"library_apply_h_ms": ours, "cufft_full_grid_ms": a.elapsed_time(b) / k,
                     "pairs": T, "grid": n}
        del x, v
        torch.cuda.empty_cache()
    print(json.dumps(out))
    return 0


def slab_report(args, local, rank, world):
    """Band-pair transforms of water32 (64 pairs, one pass each of V(r)psi
    and the density) in the slab decomposition: per phase the largest
    rank's device time (CUDA events, median of the timed passes), the
    bytes each rank sends per pass, and the exchange time (NCCL under
    torchrun; on one GPU the emulation's copies, which are not NVLink)."""
    import torch
    from amdkiit_b200.engine import FP64, MIXED
    from amdkiit_b200.slab import LocalExchange, Slab, TorchExchange
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    out = {"metric": "slab-decomposed band-pair transforms, water32 (64 pairs, 100^3)", "unit": "ms per pass",
           "report": "slab decomposition", "mode": "nccl" if world > 1 else "emulated ranks on one GPU",
           "steps": args.steps, "warmup": args.warmup}
    rlist = [world] if world > 1 else [int(x) for x in args.slab.split(",")]
    for name, prec in (("fp64", FP64), ("mixed", MIXED)):
        s, e = setup_engine(prec, local)
        e.density()
        e.potential()
        c0 = e.get_wfn()
        n1 = e.nr[0]
        v = e.get("v_pot").reshape(n1, n1, n1)
        T = (e.nstate + 1) // 2
        res = {}
        for R in rlist:
            mine = [rank] if world > 1 else list(range(R))
            slabs = [Slab(e, R, r) for r in mine]
            ex = TorchExchange() if world > 1 else LocalExchange()
            c0s = [torch.from_numpy(np.ascontiguousarray(c0[:, sl.local_g])).cuda() for sl in slabs]
            vs = [torch.from_numpy(np.ascontiguousarray(v[:, :, sl.plane0:sl.plane0 + sl.nplane])).cuda()
                  for sl in slabs]
            c2s = [torch.zeros_like(c) for c in c0s]
            rhos = [torch.zeros_like(x) for x in vs]
            sends = [sl.new_send(T) for sl in slabs]
            sc = [sl.send_counts(T) for sl in slabs]
            rc = [sl.recv_counts(T) for sl in slabs]
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

            def timed(fn):
                ev[0].record()
                fn()
                ev[1].record()
                torch.cuda.synchronize()
                return ev[0].elapsed_time(ev[1])

            t = {k: [] for k in ("pairs_out", "exchange", "planes_density", "planes_vpsi", "exchange_back",
                                 "pairs_in")}
            for it in range(args.warmup + args.steps):
                if dist is not None:
                    dist.barrier()
                pt = {k: 0.0 for k in t}
                for i, sl in enumerate(slabs):
                    pt["pairs_out"] = max(pt["pairs_out"], timed(lambda: sl.pairs_out(c0s[i], 0, T, sends[i])))
                box = {}
                pt["exchange"] = timed(lambda: box.update(r=ex(sends, sc, rc)))
                recvs = box["r"]
                dens_in = [x.clone() for x in recvs]
                for i, sl in enumerate(slabs):
                    pt["planes_density"] = max(pt["planes_density"],
                                               timed(lambda: sl.planes_density(dens_in[i], 0, T, rhos[i], False)))
                    pt["planes_vpsi"] = max(pt["planes_vpsi"], timed(lambda: sl.planes_vpsi(recvs[i], T, vs[i])))
                pt["exchange_back"] = timed(lambda: box.update(b=ex(recvs, rc, sc)))
                for i, sl in enumerate(slabs):
                    pt["pairs_in"] = max(pt["pairs_in"], timed(lambda: sl.pairs_in(box["b"][i], c0s[i], 0, T, c2s[i])))
                if it >= args.warmup:
                    for k in t:
                        t[k].append(max_over_ranks(pt[k], dist) if dist is not None else pt[k])
            eb = slabs[0].elem_bytes
            send_bytes = max(sum(c for r, c in enumerate(sc[i]) if r != sl.rank) * eb // 2
                             for i, sl in enumerate(slabs))
            res[str(R)] = {k: round(float(np.median(x)), 4) for k, x in t.items()}
            res[str(R)]["nvlink_bytes_per_rank_each_way"] = int(send_bytes)
            res[str(R)]["largest_rank_g"] = max(sl.ngpw_local for sl in slabs)
            res[str(R)]["largest_rank_planes"] = max(sl.nplane for sl in slabs)
            for sl in slabs:
                sl.close()
            del c0s, vs, c2s, rhos, sends
        out[name] = res
        e.close()
        torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()
    return 0


def oracle_fixture():
    """The oracle's converged water32 energy and forces (a committed JSON
    fixture; the oracle itself does not run here), or None."""
    p = os.path.join(ROOT, "tests", "golden", "oracle_water32.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f)


def species_forces(force, na):
    """(nsp, na_max, 3) force array -> (nat, 3) in species order."""
    return np.concatenate([np.asarray(force)[i, :k] for i, k in enumerate(na)])


def compare_arms(f64: dict, mx: dict, fixture: dict | None = None) -> dict:
    """The FP64 arm's numbers beside the mixed arm's line, and, when both ran
    MD, the mixed-vs-FP64 differences at the converged MD start: energy per
    atom, max force component, max subspace eigenvalue; with the oracle's
    converged fixture of the same system, each arm's differences from it."""
    cmp = {"fp64_value": f64["value"], "fp64_ms_per_step": f64["ms_per_step"], "fp64_e2e": f64["e2e"]["value"],
           "fp64_md": f64["md"], "scf_speedup": mx["value"] / f64["value"], "fp64_clocks": f64["clocks"]}
    if f64["md"] and mx["md"]:
        de = abs(mx["e_conv"] - f64["e_conv"]) / f64["nat"]
        df = float(np.max(np.abs(mx["f_conv"] - f64["f_conv"])))
        cmp.update({"md_speedup": mx["md"]["steps_per_s"] / f64["md"]["steps_per_s"],
                    "dE_Ha_per_atom": de, "dF_max_Ha_per_bohr": df,
                    "within_tolerance": bool(de <= 1e-6 and df <= 1e-4),
                    "compared_at": "converged MD start geometry (GRAD_CUTOFF 1e-6)"})
        fx = fixture
        if fx is not None:
            f_ref = np.array(fx["forces"])
            cmp["vs_oracle"] = {
                arm: {"dE_Ha_per_atom": abs(d["e_conv"] - fx["energies"]["etotal"]) / d["nat"],
                      "dF_max_Ha_per_bohr": float(np.max(np.abs(species_forces(d["f_conv"], d["na"]) - f_ref)))}
                for arm, d in (("fp64", f64), ("mixed", mx))}
            cmp["vs_oracle"]["fixture"] = ("tests/golden/oracle_water32.json: the CPU restatement converged to GEMAX "
                                           f"< {fx['gcut']:g} from the seeded start ({fx['iterations']} iterations)")
        ea, eb = mx.get("eig_conv"), f64.get("eig_conv")
        if isinstance(ea, np.ndarray) and isinstance(eb, np.ndarray):
            cmp["dEig_max_Ha"] = float(np.max(np.abs(ea - eb)))
        else:
            cmp["dEig_max_Ha"] = None
            cmp["eigenvalue_error"] = ea if isinstance(ea, str) else eb
    return cmp


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="gpu", choices=["gpu", "reference"])
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "mixed"],
                    help="both: mixed precision is the headline value, FP64 is measured beside it")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--md-steps", type=int, default=20,
                    help="velocity-Verlet steps per arm (200: the 32-water drift run)")
    ap.add_argument("--configs", action="store_true",
                    help="report configurations 0, 1, 2 and 4 instead of the headline line")
    ap.add_argument("--relax", action="store_true",
                    help="cfg4: LBFGS relaxation of water128 (GRAD_CUTOFF 5e-4), one JSON line")
    ap.add_argument("--relax-steps", type=int, default=100)
    ap.add_argument("--slab", default="",
                    help="R,R,...: the slab-decomposed band-pair transforms with R ranks (emulated on one GPU; "
                         "under torchrun the world size, exchanged by NCCL)")
    ap.add_argument("--cufft", action="store_true",
                    help="compare the library's H|psi> with cuFFT full-grid transforms of the same pairs")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.configs:
        return config_report(args, local) if rank == 0 else 0
    if args.cufft:
        return cufft_compare(args, local) if rank == 0 else 0
    if args.slab:
        return slab_report(args, local, rank, world)
    if args.relax:
        return relax_report(args, local) if rank == 0 else 0

    import torch
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from amdkiit_b200.engine import FP64, MIXED
    arms = {}
    if args.precision in ("both", "fp64"):
        arms["fp64"] = run_arm(FP64, args, local, dist, world)
    if args.precision in ("both", "mixed"):
        arms["mixed"] = run_arm(MIXED, args, local, dist, world)
    head = arms["mixed"] if "mixed" in arms else arms["fp64"]

    # roofline of the dominant kernel class (CUDA events around its launches)
    kern = head["kern"]
    dom = max(kern, key=lambda k: kern[k][1])
    n, ms, b = kern[dom]
    peak, src = peaks()
    achieved = (b / n) / ((ms / n) / 1000.0) / 1e9 if n else 0.0
    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": head["dtype"], "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": "mixed" if head is arms.get("mixed") else "fp64",
                   "parallelism": f"replicas{world}",
                   "l2": "working set > L2 (C0, C2, CG direction: 196 MB resident)",
                   "energy_Ha": head["energy"], "gemax": head["gemax"]},
        "e2e": head["e2e"],
        "gpu_launches": head["launches"],
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": src,
                     "traffic": TRAFFIC.get((dom, "mixed" if head is arms.get("mixed") else "fp64")),
                     "launches": n, "avg_launch_ms": ms / n if n else None},
        "kernels_ms": {k: round(v[1], 3) for k, v in kern.items()},
        "md": head["md"],
        "clocks": head["clocks"],
        "wall_ms_per_step": head["wall_ms_per_step"],
    }
    if "fp64" in arms and "mixed" in arms:
        line["mixed_vs_fp64"] = compare_arms(arms["fp64"], arms["mixed"], oracle_fixture())
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        nth = os.cpu_count() or 1
        v, dt, done = cpu_reference_iterations(REF_STEPS, REF_WARMUP, nth, REF_BUDGET_S)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": nth, "kind": "port",
                                "sample": f"{done} CG iterations of water32 (after {REF_WARMUP} warm-up, bounded at "
                                          f"{REF_BUDGET_S:.0f} s of timed work; the reference arm's window), CPU "
                                          "restatement of the reference's FP64 path, OpenMP on all host threads"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
