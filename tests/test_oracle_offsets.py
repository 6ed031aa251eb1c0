"""Section 3 distance coding in the oracle (core/distance/distance.go), pinned
by the reference: its Go tests' known answers (modes of PackageOffsetsSection,
the flat fallback) and its C99 decoder (oracle/_ref/libprzm_dec.so): the
decoder's own distance coder, its Mode 12 decoder, its distance-prefix
decoder, and whole P2 frames through przm_decompress.  CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from przm_b200 import workloads as W

needs_dec = pytest.mark.skipif(not O.ref_decoder_available(), reason="reference decoder not built")


def leb128(ds) -> bytes:
    out = bytearray()
    for v in ds:
        v = int(v)
        while v >= 0x80:
            out.append((v & 0x7F) | 0x80)
            v >>= 7
        out.append(v)
    return bytes(out)


def parse_leb128(b: bytes) -> list[int]:
    out, v, sh = [], 0, 0
    for x in b:
        v |= (x & 0x7F) << sh
        sh += 7
        if not x & 0x80:
            out.append(v)
            v, sh = 0, 0
    return out


def header_size(mode: int) -> int:
    return {0x0B: 4, 0x0A: 7, 0x06: 13}[mode]


def check_section(ds, sec: bytes) -> None:
    """sec decodes to ds (reference decoder) and is no larger than 0x09 + varints."""
    raw = leb128(ds)
    assert len(sec) <= 1 + len(raw)
    if sec[0] == 0x09:
        assert sec[1:] == raw
    else:
        assert sec[0] in (0x06, 0x0A, 0x0B)
        assert O.ref_distance_prefix_decode(sec, len(raw)) == raw


@needs_dec
def test_distance_to_code_matches_reference_coder():
    ds = set(range(1, 70))
    for c in range(49):  # every bracket's first and last distance
        base = O.ref_code_to_distance(c, 0)
        ds.update({base, base - 1, base + 1})
    ds.update({16777216, 16777217, 16777218, 33554432})
    rng = np.random.default_rng(7)
    ds.update(int(x) for x in np.exp(rng.uniform(0, np.log(33554432), 20000)).astype(np.uint64) + 1)
    for d in sorted(x for x in ds if 1 <= x <= 33554432):
        assert O.distance_to_code(d) == O.ref_distance_to_code(d), d
        c, ex, nb = O.distance_to_code(d)
        assert ex < (1 << nb) or nb == 0 and ex == 0
        assert O.ref_code_to_distance(c, ex) == d


@needs_dec
@pytest.mark.parametrize("n", [1, 2, 5, 63, 64, 1000, 50_000])
def test_mode12_stream_decodes(n):
    rng = np.random.default_rng(n)
    codes = np.minimum(rng.geometric(0.08, n) + 4, 48).astype(np.uint8)
    s = O.dist_mode12(codes)
    assert s[0] == 0x0C
    assert O.ref_decode_dist4(s, n) == codes.tobytes()


def test_mode12_empty_stream():
    assert O.dist_mode12(b"") == b"\x0c" + (65536).to_bytes(4, "little")


@needs_dec
@pytest.mark.parametrize("n,mode", [(70, 0x0B), (200, 0x0A), (1000, 0x0A), (70_000, 0x06)])
def test_package_offsets_modes_of_reference_tests(n, mode):
    # distance_test.go:404-477: n matches of distance 1000 pick these containers
    ds = [1000] * n
    sec = O.package_offsets(ds)
    assert sec[0] == mode
    check_section(ds, sec)


def test_package_offsets_flat_fallback():
    # distance_test.go:479-495: ten small alternating distances stay flat
    ds = [(i % 4) + 1 for i in range(10)]
    sec = O.package_offsets(ds)
    assert sec == b"\x09" + leb128(ds)


def test_package_offsets_empty():
    assert O.package_offsets([]) == b""


def test_pack_distance_prefix_rejects_out_of_range():
    assert O.pack_distance_prefix([5, 0, 7]) is None
    assert O.pack_distance_prefix([5, 16777217]) is None
    assert O.package_offsets([5, 0, 7])[0] == 0x09  # the fallback keeps the varints


@needs_dec
@pytest.mark.parametrize("kind", ["small", "loguniform", "equal", "two_brackets", "near_max"])
@pytest.mark.parametrize("n", [1, 17, 64, 255, 256, 4000, 120_000])
def test_package_offsets_roundtrip(kind, n):
    rng = np.random.default_rng(n * 31 + len(kind))
    if kind == "small":
        ds = rng.integers(1, 9, n)
    elif kind == "loguniform":
        ds = np.exp(rng.uniform(0, np.log(1 << 20), n)).astype(np.uint64) + 1
    elif kind == "equal":
        ds = np.full(n, 4096)
    elif kind == "two_brackets":
        ds = rng.choice([3, 300_000], n)
    else:
        ds = rng.integers(16_000_000, 16_777_217, n)
    ds = [int(x) for x in ds]
    check_section(ds, O.package_offsets(ds))


@needs_dec
def test_adaptive_code_stream_is_chosen_and_decodes():
    # two code values only: the adaptive V-ANS of the codes beats the static model
    rng = np.random.default_rng(3)
    ds = [int(x) for x in rng.choice([3, 300_123], 500)]
    sec = O.package_offsets(ds)
    h = header_size(sec[0])
    assert sec[h:h + 3] == b"VA\x01"
    check_section(ds, sec)


def frame_sections(frame: bytes):
    """(l2, l3, section 3 bytes) of a compressed (not stored) PRZM frame."""
    flags = frame[4]
    assert not flags & 0x04
    if flags & 0x08:
        l2 = int.from_bytes(frame[8:11], "little")
        l3 = int.from_bytes(frame[11:14], "little")
        o = 14 + 8
    else:
        l2 = int.from_bytes(frame[8:10], "little")
        l3 = int.from_bytes(frame[10:12], "little")
        o = 12 + 8
    return l2, l3, frame[o + l2:o + l2 + l3]


@needs_dec
@pytest.mark.parametrize("kind,n", [("markov", 100_000), ("markov", 1 << 20), ("table", 300_000),
                                    ("records", 1 << 20), ("records", 70_000), ("uniform", 50_000)])
def test_p2_frames_decode_and_carry_package_offsets(kind, n):
    a = W.gen(kind, 4242 + n, n)
    p1, p2 = O.compress_p1(a), O.compress_p2(a)
    assert O.ref_decompress(p2, n) == a.tobytes()
    assert len(p2) <= len(p1)
    if p2[4] & 0x04:  # stored: P1 is stored too
        assert p1 == p2
        return
    _, off, _ = O.tokenize(a)
    ds = parse_leb128(off)
    _, l3, s3 = frame_sections(p2)
    assert s3 == O.package_offsets(ds)
    assert l3 == len(s3) and (l3 == 0) == (len(ds) == 0)


def de_bruijn(k: int, n: int) -> list[int]:
    """Every length-n word over k symbols exactly once (cyclically)."""
    a, seq = [0] * k * n, []

    def db(t: int, p: int) -> None:
        if t > n:
            if n % p == 0:
                seq.extend(a[1:p + 1])
        else:
            a[t] = a[t - p]
            db(t + 1, p)
            for j in range(a[t - p] + 1, k):
                a[t] = j
                db(t + 1, t)

    db(1, 1)
    return seq


@needs_dec
def test_p2_frame_without_matches_has_empty_section3():
    # four symbols, no 4-byte word twice: no match, yet the literals shrink
    a = np.array([0x41 + s for s in de_bruijn(4, 4)], np.uint8)
    _, off, _ = O.tokenize(a)
    assert off == b""
    f = O.compress_p2(a)
    assert not f[4] & 0x04
    l2, l3, s3 = frame_sections(f)
    assert l3 == 0 and s3 == b""
    assert O.ref_decompress(f, len(a)) == a.tobytes()


def test_p2_section3_forms_of_the_parity_kinds():
    # the forms tests/test_gpu_p2.py expects the device to reproduce, on the
    # inputs it uses (the smaller half; 0x06 needs multi-MiB frames)
    from tests import inputs as I
    from tests.frames import section3_form
    forms = set()
    for n in (4096, 20_000, 200_000):
        for a in I.kinds(n, 5 + n).values():
            forms.add(section3_form(O.compress_p2(a)))
    assert {"empty", "09", "0B-M12", "0A-M12", "0A-AD"} <= forms, forms
