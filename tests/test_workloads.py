"""The synthetic workloads are deterministic and have the configured shapes."""
import hashlib

import numpy as np

from przm_b200 import workloads as W


def test_deterministic():
    a = W.gen("markov", 5, 100000)
    b = W.gen("markov", 5, 100000)
    assert np.array_equal(a, b)
    assert not np.array_equal(a, W.gen("markov", 6, 100000))


def test_markov_alphabet_and_copies():
    a = W.gen("markov", 1, 1 << 20)
    assert a.min() >= 0x20 and a.max() <= 0x5F


def test_zipf_skew():
    z = W.zipf(3, 1 << 20)
    c = np.sort(np.bincount(z, minlength=256))[::-1]
    assert c[0] > 10 * c[50] > 0


def test_table_columns_walk():
    t = W.gen("table", 2, 64 * 1000).view("<i4").reshape(-1, 16)
    d = np.diff(t.astype(np.int64), axis=0)
    assert np.all(np.abs(d) <= 8)


def test_config_sizes():
    s = W.config3_sizes()
    assert len(s) == 4096 and s.min() >= 1024 and s.max() < 4 << 20
    s4 = W.config4_sizes(1000)
    assert s4.max() < 16 << 20 and 30000 < np.median(s4) < 140000


def test_mixture_kinds():
    kinds = [W.mixture(i, 4096)[1] for i in range(400)]
    frac = {k: kinds.count(k) / 400 for k in set(kinds)}
    assert abs(frac["markov"] - 0.4) < 0.08 and abs(frac["uniform"] - 0.1) < 0.06
