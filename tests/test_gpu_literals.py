"""Section 4 selection on the device (przmg_package_literals_batch) against
the oracle's PackageLiteralsSection, byte for byte with the flag nibble:
text on which a sheaf foliation wins, Markov text, records, uniform bytes
that stay raw, one byte, an empty stream and the literal streams of real
frames, all in one call, twice."""
from __future__ import annotations

import numpy as np
import pytest

from przm_b200 import gpu
from przm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def json_lines(seed: int, n: int) -> bytes:
    rng = np.random.default_rng(seed)
    words = ["alpha", "beta_x", "gamma", "delta_id", "eps", "zeta", "user_name", "count"]
    out = bytearray()
    while len(out) < n:
        k = words[int(rng.integers(len(words)))]
        out += f'{{"{k}": {int(rng.integers(0, 100_000))}, "ts": "{float(rng.uniform(0, 1000)):.3f}"}}\n'.encode()
    return bytes(out[:n])


def streams(oracle) -> list[bytes]:
    s = [json_lines(1, 300_000), json_lines(2, 5000), W.gen("markov", 3, 200_000).tobytes(),
         W.gen("records", 4, 100_000).tobytes(), W.gen("uniform", 5, 40_000).tobytes(), b"A", b""]
    for kind in ("markov", "table", "records"):
        _, _, lits = oracle.tokenize(W.gen(kind, 9, 1 << 20))
        s.append(bytes(lits))
    return s


def run(comp, ss):
    from przm_b200 import devmem
    lens = np.array([len(x) for x in ss], np.uint32)
    in_offs = np.concatenate([[0], np.cumsum(lens.astype(np.uint64) + 16)[:-1]]).astype(np.uint64)
    host = np.zeros(int(in_offs[-1]) + int(lens[-1]) + 64, np.uint8)
    for x, o in zip(ss, in_offs):
        host[int(o):int(o) + len(x)] = np.frombuffer(x, np.uint8)
    caps = np.maximum(lens.astype(np.uint64), 1)
    out_offs = np.concatenate([[0], np.cumsum(caps + 16)[:-1]]).astype(np.uint64)
    d_in = devmem.upload(host)
    d_out = devmem.alloc(int(out_offs[-1] + caps[-1]) + 64)
    ol, nb = comp.PackageLiteralsBatch(d_in.ptr, in_offs, lens, d_out.ptr, out_offs, caps)
    return [(devmem.download(d_out.ptr + int(o), int(n)) if n else b"", int(f)) for o, n, f in zip(out_offs, ol, nb)]


def test_sections_match_oracle_twice(comp, oracle):
    ss = streams(oracle)
    want = [oracle.package_literals(x) for x in ss]
    assert want[0][0][3] & 0x04  # a foliation wins on the JSON-like text
    assert want[4][1] == 0       # uniform bytes stay raw
    for _ in range(2):
        got = run(comp, ss)
        for i, (g, w) in enumerate(zip(got, want)):
            assert g == w, f"stream {i}: {len(ss[i])} bytes, got {len(g[0])}/{g[1]:#x}, want {len(w[0])}/{w[1]:#x}"


def test_stream_limit(comp):
    with pytest.raises(gpu.GPUError):
        comp.PackageLiteralsBatch(0, [0], [(4 << 20) + 1], 0, [0], [8 << 20])


def test_many_small_streams(comp, oracle):
    """4000 streams in one call (68 000 V-ANS tasks, more than one grid row
    of tasks), at every byte offset: JSON-like text, Markov text, empty and
    one-byte streams."""
    ss = []
    for i in range(4000):
        n = (i * 37) % 1500
        ss.append(json_lines(i, n) if i % 3 == 0 else b"" if i % 97 == 0 else W.gen("markov", 50 + i, max(n, 1)).tobytes())
    want = [oracle.package_literals(x) for x in ss]
    assert any(w[1] and w[0][3] & 0x04 for w in want)
    got = run(comp, ss)
    bad = [i for i, (g, w) in enumerate(zip(got, want)) if g != w]
    assert not bad, f"{len(bad)} streams differ, first {bad[0]}"


def test_capacity_too_small(comp, oracle):
    """A section above its capacity fails the call (BUFFER_TOO_SMALL); the
    context stays usable."""
    from przm_b200 import devmem
    x = W.gen("uniform", 7, 10_000)
    d_in = devmem.upload(np.concatenate([x, np.zeros(64, np.uint8)]))
    d_out = devmem.alloc(20_000)
    with pytest.raises(gpu.GPUError):
        comp.PackageLiteralsBatch(d_in.ptr, [0], [len(x)], d_out.ptr, [0], [len(x) - 1])
    ss = [json_lines(3, 50_000)]
    assert run(comp, ss) == [oracle.package_literals(ss[0])]
