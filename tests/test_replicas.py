"""Replica path of bench.py on CPU: two gloo ranks, no GPU.

Windows are independent, so N GPUs run N replicas with their own windows
(seeded per rank) and no data-path collective; the only collectives are the
timing barrier and the max-over-ranks reduction of the device time.
"""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(Path(__file__).resolve().parent.parent))  # bench.py at the repository root

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from cgmli_slam_b200 import synth

        windows = synth.make_windows("c4", 2, seed=bench.rank_seed(7, rank))
        local_ms = 100.0 + 50.0 * rank  # rank 1 is the slow replica
        dist.barrier()
        slowest = bench.max_over_ranks(local_ms, dist, device="cpu")
        value = bench.aggregate_rate(world, 2, 3, slowest)
        out.put((rank, slowest, value, windows[0].state_vector()[:7].tolist(), windows[0].L))
    finally:
        dist.destroy_process_group()


def test_two_gloo_replicas_take_the_max_and_shard_windows():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    # both ranks see the slowest replica's time and report the same job rate
    assert [r[1] for r in results] == [150.0, 150.0]
    assert results[0][2] == pytest.approx(2 * 2 * 3 / 0.150)
    assert results[0][2] == results[1][2]
    # each replica solves different windows
    assert not np.allclose(results[0][3], results[1][3]) or results[0][4] != results[1][4]


def test_single_process_helpers():
    import bench

    assert bench.max_over_ranks(3.5, None) == 3.5
    assert bench.rank_seed(11, 0) == 11 and bench.rank_seed(11, 2) == 200011
    assert bench.aggregate_rate(1, 512, 5, 1000.0) == pytest.approx(2560.0)
