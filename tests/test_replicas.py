"""The N > 1 replica path of bench.py on CPU: gloo, world size 2.

bench.py runs one independent replica per GPU; its only collectives are a
barrier, the max over ranks of the timed region and sums of per-rank counts.
These tests run those helpers across two real processes.
"""
import json
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, str(ROOT))
    import bench

    dist = bench.init_dist(world, backend="gloo")
    try:
        dist.barrier()
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, device="cpu")
        solves = bench.sum_over_ranks(1.0 + rank, dist, device="cpu")
        value = bench.replica_throughput(1000, 20, ms, world)
        Path(out_dir, f"r{rank}.json").write_text(json.dumps({"ms": ms, "solves": solves, "value": value}))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time_and_sum_counts(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [json.loads((tmp_path / f"r{r}.json").read_text()) for r in range(world)]
    for r in res:
        assert r["ms"] == 15.0                      # the slower rank's time
        assert r["solves"] == 3.0                   # 1 + 2
        assert r["value"] == pytest.approx(2 * 1000 * 20 / 15e-3 / 1e6)


def test_single_process_needs_no_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.init_dist(1) is None
    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.sum_over_ranks(2.0, None) == 2.0
    assert bench.replica_throughput(5_170_176, 1000, 157.7, 1) == pytest.approx(5_170_176 * 1000 / 0.1577 / 1e6)


def test_reference_arm_prints_only_on_rank_zero(monkeypatch, capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")

    class Args:
        gpus, steps, warmup = 2, 3, 3

    assert bench.run_reference_arm(Args()) is None
    assert capsys.readouterr().out == ""
