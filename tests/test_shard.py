"""Multi-rank host logic on CPU: two gloo ranks shard frames the way
bench.py does under torchrun (weak scaling, no data-path collective, step
time = max over ranks), and split a fixed uneven input set by LPT."""
from __future__ import annotations

import ast
import hashlib
import os
import socket

import numpy as np
import pytest

from przm_b200 import shard
from przm_b200 import workloads as W


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        from oracle import oracle as O

        # weak scaling: each rank compresses its own frames
        frames = [W.mixture(s, 20_000)[0] for s in shard.frame_seeds(rank, 3)]
        digests = [hashlib.sha256(O.compress_p1(a)).hexdigest() for a in frames]
        for a in frames:  # every frame decodes back where the reference decoder is built
            if O.ref_decoder_available():
                assert O.ref_decompress(O.compress_p1(a), len(a)) == a.tobytes()
        gathered = [None] * world
        dist.all_gather_object(gathered, digests)
        # a fake per-rank step time; every rank must see the maximum
        step_ms = 10.0 + 5.0 * rank
        m = shard.max_over_ranks(step_ms, dist)
        # strong scaling split of one uneven input set
        sizes = W.config3_sizes(64)
        parts = shard.lpt_partition(sizes, world)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{m}\n{gathered}\n{parts[rank]}\n")
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_frames(tmp_path):
    import torch.multiprocessing as mp

    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0 = (tmp_path / "rank0.txt").read_text().splitlines()
    r1 = (tmp_path / "rank1.txt").read_text().splitlines()
    assert float(r0[0]) == float(r1[0]) == 15.0
    assert r0[1] == r1[1]
    g = ast.literal_eval(r0[1])  # per-rank digest lists written by the ranks
    assert len(g) == 2 and not set(g[0]) & set(g[1])  # disjoint frames
    p0, p1 = ast.literal_eval(r0[2]), ast.literal_eval(r1[2])
    assert sorted(p0 + p1) == list(range(64))


def test_lpt_partition_balance():
    sizes = W.config3_sizes(4096)
    for world in (1, 2, 3, 8):
        parts = shard.lpt_partition(sizes, world)
        assert sorted(i for p in parts for i in p) == list(range(len(sizes)))
        loads = [int(np.sum(sizes[p])) for p in parts]
        assert max(loads) - min(loads) <= int(np.max(sizes))


def test_frame_seeds_distinct_over_ranks():
    seen = set()
    for r in range(8):
        s = shard.frame_seeds(r, 256)
        assert len(set(s)) == 256
        assert not seen & set(s)
        seen |= set(s)
    assert shard.frame_seeds(0, 2)[0] == shard.rank_seed(0)


def test_max_over_ranks_without_group():
    assert shard.max_over_ranks(3.5) == 3.5


@pytest.mark.parametrize("world", [0, -1])
def test_lpt_rejects_empty_world(world):
    with pytest.raises(ValueError):
        shard.lpt_partition([1, 2], world)
