"""Host-side sharding of independent frames over ranks (one process per GPU).

Frames are independent units (no exchange step between them), so the path
scales with no data-path collective:
  - weak scaling: every rank compresses its own frames, drawn from a
    rank-specific seed (`frame_seeds`);
  - a fixed set of inputs (strong scaling) is split by greedy
    longest-processing-time first over the ranks (`lpt_partition`), so the
    byte loads differ by at most the largest input;
  - a step's time is the maximum over ranks (`max_over_ranks`), one
    all-reduce of one float outside the timed region.
"""
from __future__ import annotations

import heapq

BASE_SEED = 0x50525A4D  # "PRZM"


def rank_seed(rank: int, config: int = 2) -> int:
    return BASE_SEED + config + 1000003 * rank


def frame_seeds(rank: int, count: int, config: int = 2) -> list[int]:
    """Seeds of a rank's frames; no two (rank, frame) pairs share a seed
    for count < 1000003 // 7919."""
    s = rank_seed(rank, config)
    return [s + 7919 * i for i in range(count)]


def lpt_partition(sizes, world: int) -> list[list[int]]:
    """Indices of `sizes` per rank: largest first onto the least-loaded rank
    (ties: lower rank).  Every index appears exactly once; within a rank the
    indices are ascending."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(p) for p in parts]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The maximum of `value` over all ranks of the default process group
    (the value itself without one)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
