"""Multi-rank logic of bench.py on CPU: two gloo ranks (127.0.0.1).

bench.py runs one independent replica per GPU and times a step by the slowest
rank; these tests run that aggregation over a real two-rank process group, and
check that the reference arm does its work on rank 0 only.
"""

import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    local_ms = [1000.0, 1250.0][rank]  # rank 1 is the slower replica
    m = bench.rank_max(local_ms, dist, "cpu")
    value = bench.replicas_throughput(4096, world, m)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, m, value))


def test_step_time_is_max_over_two_gloo_ranks():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, m, value in res:
        assert m == 1250.0  # every rank sees the slowest replica's time
        assert value == pytest.approx(2 * 4096 / 1.25)


def test_single_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.rank_max(3.5, None, "cpu") == 3.5
    assert bench.replicas_throughput(100, 1, 500.0) == pytest.approx(200.0)


def test_reference_arm_runs_on_rank_zero_only(capsys):
    sys.path.insert(0, ROOT)
    import argparse

    import bench

    args = argparse.Namespace(warmup=3, steps=1, cpu_spots_per_thread=1, spots=4096, seed=7)
    assert bench.run_reference(args, rank=1, world=2) is None
    assert capsys.readouterr().out == ""


def test_reference_arm_prints_contract_line(capsys):
    """Rank 0 of the reference arm times the oracle port on the host cores and
    prints one JSON line with the contract's keys, its cpu_baseline and an e2e
    equal to its own value (no device copies)."""
    sys.path.insert(0, ROOT)
    import argparse
    import json

    import bench

    args = argparse.Namespace(warmup=1, steps=1, cpu_spots_per_thread=1, spots=64, seed=7)
    bench.run_reference(args, rank=0, world=1)
    lines = [ln for ln in capsys.readouterr().out.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
