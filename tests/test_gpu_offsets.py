"""Section 3 distance coding on the device (przmg_package_offsets_batch)
against the oracle's PackageOffsetsSection, byte for byte: the reference
tests' container modes, the flat fallback, out-of-range distances, empty
arrays, random distance sets, the adaptive code-stream case and the offsets
of real frames, all sections of one call together, two calls in a row."""
from __future__ import annotations

import numpy as np
import pytest

from przm_b200 import gpu
from przm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def distance_sets(oracle) -> list[np.ndarray]:
    rng = np.random.default_rng(11)
    sets = [np.full(n, 1000) for n in (70, 200, 1000, 70_000)]          # 0x0B, 0x0A, 0x0A, 0x06
    sets += [np.array([(i % 4) + 1 for i in range(10)])]                 # 0x09 fallback
    sets += [np.array([], np.int64), np.array([5, 0, 7]), np.array([9, 16777217])]  # empty, out of range
    sets += [rng.choice([3, 300_123], 500)]                              # adaptive code stream
    for n in (1, 17, 64, 255, 256, 4000, 120_000):
        sets += [rng.integers(1, 9, n), np.exp(rng.uniform(0, np.log(1 << 20), n)).astype(np.int64) + 1,
                 rng.integers(16_000_000, 16_777_217, n)]
    for kind in ("markov", "records", "table"):                          # offsets of real frames
        _, off, _ = oracle.tokenize(W.gen(kind, 77, 1 << 20))
        sets += [np.array(leb_values(off), np.int64)]
    return [s.astype(np.uint32) for s in sets]


def leb_values(b: bytes) -> list[int]:
    out, v, sh = [], 0, 0
    for x in b:
        v |= (x & 0x7F) << sh
        sh += 7
        if not x & 0x80:
            out.append(v)
            v, sh = 0, 0
    return out


def run(comp, sets):
    from przm_b200 import devmem
    counts = np.array([len(s) for s in sets], np.uint32)
    dist_offs = np.concatenate([[0], np.cumsum(counts)[:-1]]).astype(np.uint64)
    caps = (1 + 5 * counts.astype(np.uint64)).astype(np.uint64)
    out_offs = np.concatenate([[0], np.cumsum(caps + 16)[:-1]]).astype(np.uint64)
    d_dist = devmem.upload(np.concatenate(sets + [np.zeros(4, np.uint32)]).view(np.uint8))
    d_out = devmem.alloc(int(out_offs[-1] + caps[-1]) + 64)
    lens = comp.PackageOffsetsBatch(d_dist.ptr, dist_offs, counts, d_out.ptr, out_offs, caps)
    return [devmem.download(d_out.ptr + int(o), int(n)) if n else b"" for o, n in zip(out_offs, lens)]


def test_sections_match_oracle_twice(comp, oracle):
    sets = distance_sets(oracle)
    want = [oracle.package_offsets(s) for s in sets]
    assert [w[0] for w in want[:5]] == [0x0B, 0x0A, 0x0A, 0x06, 0x09]
    for _ in range(2):  # the second call reuses the context's scratch
        got = run(comp, sets)
        for i, (g, w) in enumerate(zip(got, want)):
            assert g == w, f"set {i}: {len(sets[i])} distances, got {len(g)} bytes, want {len(w)}"


def test_capacity_and_limits(comp):
    from przm_b200 import devmem
    d = devmem.upload(np.full(300, 1000, np.uint32).view(np.uint8))
    out = devmem.alloc(4096)
    with pytest.raises(gpu.GPUError):  # the section needs more than 8 bytes
        comp.PackageOffsetsBatch(d.ptr, [0], [300], out.ptr, [0], [8])
    with pytest.raises(gpu.GPUError):  # above the reference's 2^21 distances per section
        comp.PackageOffsetsBatch(d.ptr, [0], [(1 << 21) + 1], out.ptr, [0], [1 << 24])
