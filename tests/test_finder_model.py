"""CPU pinning of the canonical tile-finder semantics.

The reference tile finder (przm_search_matches_kernel, gpu/kernel/
przm_lz77.cu:221-360) updates a bucket with a plain read of the old value
followed by atomicMax (:350-355), so when two positions of one 256-position
step hit the same bucket the low half (the second candidate) depends on
timing.  On inputs where no bucket is hit twice in a step the update has one
outcome: high half = p + 1, low half = the previous high half.  Here a
pure-Python model that follows the kernel line by line under that condition
is compared with the oracle's canonical finder (tile_find) on such inputs;
the GPU test runs the reference kernel itself on the same inputs."""
from __future__ import annotations

import numpy as np
import pytest

from tests.inputs import STEP, TILE, hash4, race_free_tile, steps_race_free, words4


def _lcp(t: np.ndarray, a: int, b: int, limit: int) -> int:
    """przm_gpu_lcp_shared (przm_lz77.cu:63-85): exact common prefix, capped."""
    if limit <= 0:
        return 0
    ne = np.flatnonzero(t[a:a + limit] != t[b:b + limit])
    return int(ne[0]) if len(ne) else limit


def reference_tile_model(a: np.ndarray) -> np.ndarray:
    """przm_lz77.cu:221-360 for one block of 256 threads, every step's queries
    against the bucket table as it stood after the previous step."""
    n = len(a)
    out = np.zeros(n, np.uint32)
    for t0 in range(0, n, TILE):
        tl = min(TILE, n - t0)
        t = a[t0:t0 + tl]
        w = words4(t)
        h = hash4(w)
        head = np.zeros(2048, np.uint32)
        for s0 in range(0, tl, STEP):
            upd = []
            for p in range(s0, min(s0 + STEP, tl)):
                if p + 4 > tl:
                    continue
                lane = p & 31
                lim = min(tl - p, 4095)
                best_len = best_off = 0
                for d in range(1, 5):  # __shfl_up_sync within the 32-lane warp
                    if lane >= d and w[p - d] == w[p]:
                        L = _lcp(t, p, p - d, lim)
                        if L > best_len:
                            best_len, best_off = L, d
                bv = int(head[h[p]])
                c0, c1 = bv >> 16, bv & 0xFFFF
                for c, need in ((c0, False), (c1, True)):
                    if c == 0 or (need and best_len >= 258):
                        continue
                    cand = c - 1
                    if cand < p and w[cand] == w[p]:
                        L = _lcp(t, p, cand, lim)
                        if L > best_len:
                            best_len, best_off = L, p - cand
                if best_len >= 4:
                    out[t0 + p] = (min(best_len, 4095) << 20) | best_off
                upd.append(p)
            for p in upd:  # one hit per bucket per step: the atomicMax has one outcome
                old = int(head[h[p]])
                head[h[p]] = max(old, ((p + 1) << 16) | (old >> 16))
    return out


@pytest.mark.parametrize("n,seed", [(3000, 1), (32768, 2), (40000, 3), (65536, 4)])
def test_race_free_inputs_have_the_property(n, seed):
    a = race_free_tile(n, seed)
    assert steps_race_free(a)
    # and they are not trivial: most positions inside a copy find a match
    assert np.count_nonzero(hash4(words4(a))) > 0


@pytest.mark.parametrize("n,seed", [(3000, 5), (20000, 6), (40000, 7)])
def test_canonical_tile_finder_is_the_reference_rule_on_race_free_inputs(oracle, n, seed):
    a = race_free_tile(n, seed)
    want = reference_tile_model(a)
    got = oracle.tile_find(a)
    assert np.count_nonzero(want) > n // 4  # the copies give matches
    assert np.array_equal(got, want)
