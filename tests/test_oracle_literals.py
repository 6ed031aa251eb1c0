"""Section 4 selection in the oracle (core/literals/literals.go:600-693,
sheaf.go), pinned by the reference's C99 decoder: its own fiber classes
(przm_context_classify, przm_context_classify_order2) for every context, its
fiber reconstitution (przm_reconstitute_fibers), and whole P3 frames through
przm_decompress.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from przm_b200 import workloads as W

needs_dec = pytest.mark.skipif(not O.ref_decoder_available(), reason="reference decoder not built")


def json_lines(seed: int, n: int) -> np.ndarray:
    """Seeded JSON-like log lines (identifiers, digits, quotes and colons)."""
    rng = np.random.default_rng(seed)
    words = ["alpha", "beta_x", "gamma", "delta_id", "eps", "zeta", "user_name", "count"]
    out = bytearray()
    while len(out) < n:
        k = words[int(rng.integers(len(words)))]
        v = int(rng.integers(0, 100_000))
        f = float(rng.uniform(0, 1000))
        out += f'{{"{k}": {v}, "ts": "{f:.3f}", "tag": "{words[int(rng.integers(len(words)))]}"}}\n'.encode()
    return np.frombuffer(bytes(out[:n]), np.uint8)


def inputs():
    return {
        "json": json_lines(1, 200_000),
        "markov": W.gen("markov", 3, 200_000),
        "records": W.gen("records", 4, 100_000),
        "uniform": W.gen("uniform", 5, 30_000),
        "one": np.frombuffer(b"A", np.uint8),
    }


@needs_dec
def test_fiber_classes_match_reference_decoder():
    for mode in range(3):
        for p1 in range(256):
            assert O.sheaf_class(0, p1, mode) == O.ref_context_classify(0, p1, mode), (mode, p1)
    for p2 in range(256):
        for p1 in range(256):
            assert O.sheaf_class(p2, p1, 3) == O.ref_context_classify(p2, p1, 3), (p2, p1)


@needs_dec
@pytest.mark.parametrize("mode", [0, 1, 2, 3])
@pytest.mark.parametrize("name", ["json", "markov", "records", "uniform", "one"])
def test_fibers_reconstitute_with_reference(name, mode):
    a = inputs()[name].tobytes()
    fibers = O.decompose_fibers(a, mode)
    assert sum(len(f) for f in fibers) == len(a)
    if mode == 2:
        assert fibers[2] == b"" and fibers[3] == b""
    assert O.ref_reconstitute_fibers(fibers, mode) == a


@pytest.mark.parametrize("name", ["json", "markov", "records", "uniform", "one"])
def test_package_literals_picks_the_smallest(name):
    a = inputs()[name].tobytes()
    sec, nib = O.package_literals(a)
    cands = [O.adaptive_vans(a)] + [O.pack_sheaf(a, m) for m in range(4)]
    best = min(len(c) for c in cands)
    if best < len(a):
        assert nib == 0x80 and len(sec) == best
        first = next(c for c in cands if len(c) == best)  # ties keep the earlier candidate
        assert sec == first
    else:
        assert nib == 0 and sec == a


def test_sheaf_container_layout():
    a = json_lines(2, 50_000).tobytes()
    for mode in range(4):
        c = O.pack_sheaf(a, mode)
        assert c[:3] == b"VA\x01" and c[3] == (0x01 | 0x04 | (mode << 4))
        assert int.from_bytes(c[4:8], "little") == len(a)
        l = [int.from_bytes(c[8 + 4 * k:12 + 4 * k], "little") for k in range(4)]
        e = [int.from_bytes(c[24 + 4 * k:28 + 4 * k], "little") for k in range(4)]
        assert sum(l) == len(a) and len(c) == 40 + sum(e)
        assert all(ek <= lk and (lk or not ek) for ek, lk in zip(e, l))


@needs_dec
@pytest.mark.parametrize("name", ["json", "markov", "records", "uniform", "one"])
def test_p3_frames_decode(name):
    a = inputs()[name]
    p2, p3 = O.compress_p2(a), O.compress_p3(a)
    assert O.ref_decompress(p3, len(a)) == a.tobytes()
    assert len(p3) <= len(p2)


@needs_dec
def test_p3_json_frame_carries_a_foliation():
    a = json_lines(7, 300_000)
    f = O.compress_p3(a)
    assert O.ref_decompress(f, len(a)) == a.tobytes()
    _, off, lits = O.tokenize(a)
    sec, nib = O.package_literals(lits)
    assert nib == 0x80 and sec[3] & 0x04  # a sheaf container wins on this text
    assert f.endswith(sec) and f[4] & 0x80


def test_p3_section4_forms_of_the_test_inputs():
    # the Section 4 forms tests/test_gpu_coded_sections.py expects the device
    # to reproduce: raw, the adaptive container and every foliation
    from tests import inputs as I
    from tests.frames import section4_form
    xs = [a for n in (4096, 20_000, 200_000) for a in I.kinds(n, 5 + n).values()]
    xs += [I.ident_text(200_000, 7), I.tagged_numbers(20_000, 7)]
    forms = {section4_form(O.compress_p3(a)) for a in xs}
    assert {"raw", "AD", "SH0", "SH1", "SH2", "SH3"} <= forms, forms
