"""Independent replicas across the ranks of a process group (one GPU per rank).

Starts never interact: each has its own iterate, support and error history
(src/cuda/cuda_solver.cu:98-102 of the reference), so N GPUs run N independent
solvers with no data exchange. The only cross-rank steps are bookkeeping: the
best start over all ranks (an argmin over one float per start, the reference's
best_index at src/core/solver.cpp:95-103 taken across ranks) and the slowest
rank's time for a benchmark. Both go through the default process group of
``torch.distributed``, whatever its backend (NCCL on GPUs, gloo on CPUs).
"""

from __future__ import annotations

import math


def _dist():
    import torch.distributed as dist

    return dist


def _tensor(values, dtype):
    import torch

    dist = _dist()
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    return torch.tensor(values, dtype=dtype, device=device)


def rank_starts(starts: int, world: int, rank: int) -> tuple[int, int]:
    """(first, count) of the starts rank `rank` runs when `starts` are split as
    evenly as possible over `world` ranks (the first `starts % world` ranks run
    one more)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    if starts < 0:
        raise ValueError("starts must be >= 0")
    base, extra = divmod(starts, world)
    count = base + (1 if rank < extra else 0)
    first = rank * base + min(rank, extra)
    return first, count


def rank_seed(seed: int, rank: int) -> int:
    """Seed of a rank's random starts: replicas draw distinct starts."""
    return int(seed) + int(rank)


def max_over_ranks(value: float) -> float:
    """The largest `value` over all ranks (the slowest rank's time)."""
    dist = _dist()
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = _tensor([float(value)], _float64())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def best_over_ranks(errors) -> tuple[int, int, float]:
    """(rank, index, error) of the start with the lowest final error over all
    ranks; `errors` are this rank's final errors. A NaN never displaces a
    finite error; ties go to the lowest rank, then the lowest index."""
    errors = [float(e) for e in errors]
    local = (math.inf, -1)
    for i, e in enumerate(errors):
        if not math.isnan(e) and e < local[0]:
            local = (e, i)
    dist = _dist()
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return 0, max(local[1], 0), local[0] if local[1] >= 0 else math.nan
    world = dist.get_world_size()
    mine = _tensor([local[0], float(local[1])], _float64())
    gathered = [_tensor([0.0, 0.0], _float64()) for _ in range(world)]
    dist.all_gather(gathered, mine)
    best = (math.inf, -1, -1)
    for r, t in enumerate(gathered):
        e, i = float(t[0].item()), int(t[1].item())
        if i >= 0 and e < best[0]:
            best = (e, r, i)
    if best[1] < 0:
        return 0, 0, math.nan
    return best[1], best[2], best[0]


def _float64():
    import torch

    return torch.float64
