"""Seeded inputs shared by the parity tests: every content kind of the
workload mixture plus the edge cases the reference's own tests exercise
(empty and sub-minimum inputs, gpu/gpu_test.go:188-208; 32 KiB tile and
64 KiB finder boundaries, max match length 4095 and long runs,
tests/e2e/gpu_tier2_boundaries_test.go:20-334; cross-tile periodic data,
gpu/gpu_test.go:241-285)."""
from __future__ import annotations

import numpy as np

from przm_b200 import workloads as W

EDGE_SIZES = [1, 2, 3, 4, 7, 8, 9, 11, 12, 13, 15, 16, 17, 31, 32, 33, 255, 256, 257, 4095, 4096, 4097,
              32767, 32768, 32769, 65535, 65536, 65537, 65543, 98304, 131072 + 5]


def periodic(n: int) -> np.ndarray:
    """gpu/gpu_test.go:248-257: byte ((i*73 + (i/4096)*17) & 0xFF) with a
    pattern pasted every 256 KiB."""
    i = np.arange(n, dtype=np.int64)
    a = ((i * 73 + (i // 4096) * 17) & 0xFF).astype(np.uint8)
    pat = np.frombuffer(b"RADIX_STRIKE_LONG_DISTANCE_CROSS_TILE_MATCH_VERIFICATION_PAYLOAD_1234567890!", np.uint8)
    for off in range(0, n - len(pat) + 1, 256 * 1024):
        a[off:off + len(pat)] = pat
    return a


def runs(n: int, seed: int) -> np.ndarray:
    """Runs of repeated bytes of random lengths (RLE opcodes, long matches)."""
    rng = np.random.default_rng(seed)
    out = np.empty(n, np.uint8)
    i = 0
    while i < n:
        L = int(rng.integers(1, 5000)) if rng.random() < 0.3 else int(rng.integers(1, 40))
        out[i:i + L] = rng.integers(0, 256)
        i += L
    return out


def repeats(n: int, seed: int, period: int) -> np.ndarray:
    """A random block repeated: every position matches at distance `period`."""
    rng = np.random.default_rng(seed)
    blk = rng.integers(0, 256, period, dtype=np.uint8)
    return np.resize(blk, n)


def kinds(n: int, seed: int) -> dict[str, np.ndarray]:
    return {
        "markov": W.gen("markov", seed, n),
        "table": W.gen("table", seed + 1, n),
        "records": W.gen("records", seed + 2, n),
        "uniform": W.gen("uniform", seed + 3, n),
        "zeros": np.zeros(n, np.uint8),
        "runs": runs(n, seed + 4),
        "rep7": repeats(n, seed + 5, 7),
        "rep4096": repeats(n, seed + 6, 4096),
        "rep5000": repeats(n, seed + 7, 5000),
        "periodic": periodic(n),
    }


def parity_cases(max_n: int = 1 << 20, seed: int = 11) -> list[tuple[str, np.ndarray]]:
    cases = []
    for n in EDGE_SIZES:
        for k, a in kinds(n, seed + n).items():
            cases.append((f"{k}-{n}", a))
    for n in (200_000, max_n):
        for k, a in kinds(n, seed + n).items():
            cases.append((f"{k}-{n}", a))
    return cases
