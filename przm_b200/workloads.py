"""Seeded synthetic workloads of the five benchmark configurations.

No corpus exists for this path; every input is generated from the published
xoshiro256** / splitmix64 generators in csrc/przm_gen.c, so the same seed gives
the same bytes everywhere.  Seed of configuration k: 0x50525A4D ("PRZM") + k.
"""
from __future__ import annotations

import numpy as np

from . import _lib

SEED = 0x50525A4D
MiB = 1 << 20
KIND = {0: "markov", 1: "table", 2: "records", 3: "uniform"}


def gen(kind: str, seed: int, n: int) -> np.ndarray:
    a = np.zeros(max(n, 1), np.uint8)
    getattr(_lib.gen(), f"przm_gen_{kind}")(seed, a.ctypes.data, n)
    return a[:n]


def zipf(seed: int, n: int, s: float = 1.1) -> np.ndarray:
    a = np.zeros(max(n, 1), np.uint8)
    _lib.gen().przm_gen_zipf(seed, s, a.ctypes.data, n)
    return a[:n]


def mixture(seed: int, n: int) -> tuple[np.ndarray, str]:
    a = np.zeros(max(n, 1), np.uint8)
    k = _lib.gen().przm_gen_mixture(seed, a.ctypes.data, n)
    return a[:n], KIND[k]


def config0() -> np.ndarray:
    """One 4 MiB order-1 Markov input with ~30% copies (one frame)."""
    return gen("markov", SEED + 0, 4 * MiB)


def config1(count: int = 64, size: int = MiB) -> list[np.ndarray]:
    """64 x 1 MiB Zipf(1.1) streams for histogram + V-ANS in isolation."""
    z = zipf(SEED + 1, count * size)
    return [z[i * size:(i + 1) * size] for i in range(count)]


def config2(count: int = 256, size: int = MiB) -> list[np.ndarray]:
    """256 x 1 MiB segments of the mixture (one frame per segment)."""
    return [mixture(SEED + 2 + 7919 * i, size)[0] for i in range(count)]


def config3_sizes(count: int = 4096) -> np.ndarray:
    rng = np.random.default_rng(SEED + 3)
    return np.floor(np.exp(rng.uniform(np.log(1024), np.log(4 * MiB), count))).astype(np.int64)


def config3(count: int = 4096) -> list[np.ndarray]:
    """4096 inputs, sizes log-uniform in [1 KiB, 4 MiB], mixture content."""
    return [mixture(SEED + 3 + 104729 * i, int(n))[0] for i, n in enumerate(config3_sizes(count))]


def config4_sizes(count: int) -> np.ndarray:
    rng = np.random.default_rng(SEED + 4)
    s = np.floor(np.exp(rng.normal(np.log(65536), 1.5, count))).astype(np.int64)
    return np.clip(s, 1, 16 * MiB - 1)


def config4(count: int) -> list[np.ndarray]:
    """Serving jobs: log-normal sizes (median 64 KiB, sigma 1.5, < 16 MiB)."""
    return [mixture(SEED + 4 + 15485863 * i, int(n))[0] for i, n in enumerate(config4_sizes(count))]
