"""bench.py host logic without a GPU: the max-over-ranks timing reduction on
two gloo ranks, and the reference arm's JSON line (with the CPU restatement
replaced by a stub so the test stays short)."""
import json
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks(1.5 + rank, dist, "cpu")
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(2))
    assert res == {0: 2.5, 1: 2.5}


def test_max_over_ranks_single_process():
    assert bench.max_over_ranks(3.25, None) == 3.25


class _Args:
    steps, warmup, gpus = 5, 3, 1


def test_reference_arm_json(monkeypatch, capsys):
    monkeypatch.setattr(bench, "cpu_reference_iterations", lambda steps, warmup, nth, budget=0.0: (0.5, 4.0, 2))
    assert bench.run_reference(_Args, 0) == 0
    line = json.loads(capsys.readouterr().out.strip())
    assert line["impl"] == "reference" and line["metric"] == bench.METRIC and line["unit"] == bench.UNIT
    assert line["value"] == 0.5 and line["steps"] == 2 and line["higher_is_better"] is True
    assert line["e2e"] == {"value": 0.5, "unit": bench.UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["value"] == 0.5


def test_reference_arm_other_ranks_print_nothing(capsys):
    assert bench.run_reference(_Args, 1) == 0
    assert capsys.readouterr().out == ""


def _arm(value, e, f, eig, md=True):
    return {"value": value, "ms_per_step": 1000.0 / value, "e2e": {"value": value / 2}, "clocks": {},
            "md": {"steps_per_s": value / 100} if md else None, "nat": 3, "na": [1],
            "e_conv": e, "f_conv": np.array(f), "eig_conv": eig}


def test_compare_arms_differences():
    f64 = _arm(400.0, -17.0, [[0.1, 0.0, 0.0]], np.array([-0.9, -0.3]))
    mx = _arm(600.0, -17.0 + 3e-7, [[0.1 + 2e-6, 0.0, 0.0]], np.array([-0.9, -0.3 + 4e-8]))
    c = bench.compare_arms(f64, mx)
    assert abs(c["scf_speedup"] - 1.5) < 1e-12 and abs(c["md_speedup"] - 1.5) < 1e-12
    assert abs(c["dE_Ha_per_atom"] - 1e-7) < 1e-12 and abs(c["dF_max_Ha_per_bohr"] - 2e-6) < 1e-12
    assert abs(c["dEig_max_Ha"] - 4e-8) < 1e-12 and c["within_tolerance"]


def test_compare_arms_reports_eigenvalue_failure_and_no_md():
    f64 = _arm(400.0, -17.0, [[0.0, 0.0, 0.0]], np.array([-0.5]))
    mx = _arm(600.0, -17.0, [[0.0, 0.0, 0.0]], "amdk_apply_h failed (-5): ...")
    c = bench.compare_arms(f64, mx)
    assert c["dEig_max_Ha"] is None and c["eigenvalue_error"].startswith("amdk_apply_h")
    c = bench.compare_arms(_arm(400.0, 0, [[0, 0, 0]], None, md=False), _arm(600.0, 0, [[0, 0, 0]], None, md=False))
    assert "dE_Ha_per_atom" not in c and abs(c["scf_speedup"] - 1.5) < 1e-12


def test_compare_arms_against_the_oracle_fixture():
    f64 = _arm(400.0, -17.0, [[[0.1, 0.0, 0.0]]], None)
    mx = _arm(600.0, -17.0 + 3e-7, [[[0.1 + 2e-6, 0.0, 0.0]]], None)
    fx = {"energies": {"etotal": -17.0 - 6e-7}, "forces": [[0.1 - 1e-6, 0.0, 0.0]], "gcut": 1e-6, "iterations": 9}
    v = bench.compare_arms(f64, mx, fx)["vs_oracle"]
    assert abs(v["fp64"]["dE_Ha_per_atom"] - 2e-7) < 1e-12 and abs(v["mixed"]["dE_Ha_per_atom"] - 3e-7) < 1e-12
    assert abs(v["fp64"]["dF_max_Ha_per_bohr"] - 1e-6) < 1e-12 and abs(v["mixed"]["dF_max_Ha_per_bohr"] - 3e-6) < 1e-12


def test_clock_sampler_without_nvml(monkeypatch):
    """No NVML (no GPU here): the sampler reports why, never raises."""
    cs = bench.ClockSampler(0)
    monkeypatch.setattr(cs, "_handle", lambda: (_ for _ in ()).throw(RuntimeError("no driver")))
    cs.start()
    out = cs.stop()
    assert out["samples"] == 0 and out["sm_mhz"] is None and "no driver" in out["reasons"][0]
