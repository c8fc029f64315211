"""The multi-rank host logic of independent replicas, run as two gloo ranks on
the CPU (no GPU): start partition, per-rank seeds, the slowest rank's time and
the best start over all ranks."""

import math
import os
import socket

import pytest

from qoraphasecu_b200 import replicas


def test_rank_starts_partition_every_start_once():
    for starts in (0, 1, 7, 32, 33):
        for world in (1, 2, 3, 8):
            seen = []
            for rank in range(world):
                first, count = replicas.rank_starts(starts, world, rank)
                seen.extend(range(first, first + count))
            assert seen == list(range(starts))
    with pytest.raises(ValueError):
        replicas.rank_starts(4, 2, 2)


def test_single_process_needs_no_group():
    assert replicas.max_over_ranks(1.5) == 1.5
    assert replicas.best_over_ranks([0.3, float("nan"), 0.1]) == (0, 2, 0.1)
    rank, index, error = replicas.best_over_ranks([float("nan")])
    assert (rank, index) == (0, 0) and math.isnan(error)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        slowest = replicas.max_over_ranks(10.0 + rank)
        # rank 0's best is 0.5 at index 1; rank 1 holds the global best 0.25 at index 2
        errors = [[0.9, 0.5, float("nan")], [0.7, 0.6, 0.25]][rank]
        best = replicas.best_over_ranks(errors)
        tie = replicas.best_over_ranks([0.4, 0.4])
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(repr((slowest, best, tie, replicas.rank_seed(7, rank))))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    results = [eval((tmp_path / f"rank{r}.txt").read_text()) for r in range(2)]
    for rank, (slowest, best, tie, seed) in enumerate(results):
        assert slowest == 11.0
        assert best == (1, 2, 0.25)
        assert tie == (0, 0, 0.4)
        assert seed == 7 + rank
