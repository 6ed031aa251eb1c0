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


TILE = 32768
STEP = 256  # positions the reference tile finder queries between two bucket updates


def hash4(words: np.ndarray) -> np.ndarray:
    """przm_gpu_hash4 (przm_lz77.cu:55-57) of little-endian u32 words."""
    w = words.astype(np.uint64)
    return (((w * 0x1E35A7BD) & 0xFFFFFFFF) >> 21) & 2047


def words4(a: np.ndarray) -> np.ndarray:
    """Little-endian u32 word at every position p with p + 4 <= len(a)."""
    b = a.astype(np.uint32)
    n = len(a) - 3
    return b[:n] | (b[1:n + 1] << 8) | (b[2:n + 2] << 16) | (b[3:n + 3] << 24) if n > 0 else np.zeros(0, np.uint32)


def kmer_hash(a: np.ndarray) -> np.ndarray:
    """Radix-strike hash (przm_lz77.cu:171-174) of the k-mer at every 8-aligned p with p + 8 <= len(a)."""
    c = len(a) // 8 if len(a) >= 8 else 0
    k = np.frombuffer(np.ascontiguousarray(a[:8 * c]).tobytes(), "<u8")
    with np.errstate(over="ignore"):
        return ((k * np.uint64(0x9E3779B97F4A7C15)) >> np.uint64(43)) & np.uint64((1 << 19) - 1)


def race_free_tile(n: int, seed: int, copy_rate: float = 0.9) -> np.ndarray:
    """Bytes on which the reference tile finder is deterministic: inside every
    256-position step of every 32 KiB tile, no two valid positions share a
    hash bucket, so each bucket takes at most one update per step and the
    read-then-atomicMax of przm_lz77.cu:350-355 has one outcome.  Most bytes
    continue a copy of earlier data (offsets of one step or more, so that
    copied words sit in other steps), which gives plenty of matches; a byte
    whose completed word would hit a bucket already used in its step is
    replaced by another value until it does not."""
    rng = np.random.default_rng(seed)
    a = np.zeros(n, np.uint8)
    used: set[int] = set()
    cur = -1
    src = -1  # copy source of the next byte, -1 = random
    for i in range(n):
        if src < 0 and i >= 2 * STEP and rng.random() < copy_rate:
            local = i % TILE
            if local >= 2 * STEP:
                off = int(rng.integers(STEP + 4, min(local, 8 * 1024) + 1))
                src = i - off
        b = int(a[src]) if src >= 0 else int(rng.integers(0, 256))
        if src >= 0:
            src += 1
            if rng.random() < 1 / 24:  # copy runs of mean length 24
                src = -1
        p = i - 3
        if p >= 0 and p // TILE == i // TILE:
            step = p // STEP  # steps never straddle tiles (TILE is a multiple of STEP)
            if step != cur:
                cur, used = step, set()
            base = int(a[p]) | (int(a[p + 1]) << 8) | (int(a[p + 2]) << 16)
            h = ((((base | (b << 24)) * 0x1E35A7BD) & 0xFFFFFFFF) >> 21) & 2047
            while h in used:
                b = int(rng.integers(0, 256))
                src = -1
                h = ((((base | (b << 24)) * 0x1E35A7BD) & 0xFFFFFFFF) >> 21) & 2047
            used.add(h)
        a[i] = b
    return a


def steps_race_free(a: np.ndarray) -> bool:
    """No hash bucket hit twice by the valid positions of one step."""
    n = len(a)
    for t0 in range(0, n, TILE):
        tl = min(TILE, n - t0)
        h = hash4(words4(a[t0:t0 + tl]))
        for s0 in range(0, len(h), STEP):
            hs = h[s0:s0 + STEP]
            if len(np.unique(hs)) != len(hs):
                return False
    return True


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


def ident_text(n: int, seed: int) -> np.ndarray:
    """Lower-case identifiers, each followed by one syntax byte (the order-2
    foliation, mode 3, codes it best)."""
    rng = np.random.default_rng(seed)
    alpha = np.frombuffer(b"abcdefghijklmnopqrstuvwxyz_", np.uint8)
    punct = np.frombuffer(b"(){};,.=+ ", np.uint8)
    out, size = [], 0
    while size < n:
        w = alpha[rng.integers(0, len(alpha), int(rng.integers(2, 9)))]
        out += [w, punct[rng.integers(0, len(punct), 1)]]
        size += len(w) + 1
    return np.concatenate(out)[:n].copy()


def tagged_numbers(n: int, seed: int) -> np.ndarray:
    """An upper-case letter, a decimal number and a separator, repeated (the
    two-way foliation, mode 2, codes it best)."""
    rng = np.random.default_rng(seed)
    parts, size = [], 0
    while size < n:
        s = b"%c%d%c" % (65 + int(rng.integers(0, 26)), int(rng.integers(0, 10 ** 6)), b" ,;"[int(rng.integers(0, 3))])
        parts.append(s)
        size += len(s)
    return np.frombuffer(b"".join(parts)[:n], np.uint8).copy()
