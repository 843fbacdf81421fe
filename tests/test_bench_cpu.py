"""bench.py host logic without a GPU: the max-over-ranks timing reduction on
two gloo ranks, and the reference arm's JSON line (with the CPU restatement
replaced by a stub so the test stays short)."""
import json
import os
import socket

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
