"""CPU tests of the oracle (the checker of the CUDA path).

The oracle restates the reference's GPU path in C.  It is pinned here by:
  - the known-answer properties the reference's own tests state;
  - byte-exact round trips through the reference's own C99 decoder
    (src/przm_dec.c, built from its sources into oracle/_ref/);
  - a second, independent pure-Python restatement of the finders and the
    tokenizer on small inputs;
  - the committed golden fixtures (tests/golden/).
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np
import pytest

from tests import inputs as I
from tests import pyref

HERE = os.path.dirname(os.path.abspath(__file__))


def test_pack_match32_kat(oracle):
    # gpu/gpu_test.go:210-241
    for length, off in [(4, 1), (10, 50), (258, 65535), (4095, 1048575)]:
        d = oracle.pack_match32(length, off)
        assert d >> 20 == length and d & 0xFFFFF == off
    assert oracle.pack_match32(3, 10) == 0
    assert oracle.pack_match32(10, 0) == 0
    assert oracle.pack_match32(5000, 7) >> 20 == 4095


@pytest.mark.parametrize("n", [0, 1, 3])
def test_match_edge_cases(oracle, n):
    # gpu/gpu_test.go:188-208: empty and sub-minimum inputs have no matches
    pos, dsc = oracle.match_lz77(bytes(range(n)))
    assert len(pos) == 0


def _valid_table(a: np.ndarray, desc: np.ndarray, exact: bool):
    n = len(a)
    for p in np.nonzero(desc)[0]:
        L, d = int(desc[p] >> 20), int(desc[p] & 0xFFFFF)
        assert 4 <= L <= 4095 and 0 < d <= p and p + L <= n
        assert bytes(a[p:p + L]) == bytes(a[p - d:p - d + L])
        if exact and L < 4095 and p + L < n:
            assert a[p + L] != a[p - d + L]


@pytest.mark.parametrize("name,a", [c for c in I.parity_cases(300_000) if len(c[1]) <= 300_000][::7])
def test_match_table_valid(oracle, name, a):
    """Every descriptor is a real match and its length the exact common
    prefix (capped at 4095, the tile end or the input end)."""
    desc = oracle.match_table(a)
    if len(a) <= 65536:
        # tile finder: lengths are capped at the 32 KiB tile end
        for p in np.nonzero(desc)[0]:
            L, d = int(desc[p] >> 20), int(desc[p] & 0xFFFFF)
            te = (p // 32768 + 1) * 32768
            assert 0 < d <= p % 32768 and bytes(a[p:p + L]) == bytes(a[p - d:p - d + L])
            if L < 4095 and p + L < min(te, len(a)):
                assert a[p + L] != a[p - d + L]
    else:
        assert not np.any(desc[np.arange(len(a)) % 8 != 0])
        _valid_table(a, desc, exact=True)


@pytest.mark.parametrize("n", [5, 40, 300, 700, 2100, 9000])
@pytest.mark.parametrize("kind", ["markov", "runs", "rep7", "records", "table"])
def test_finders_match_python_restatement(oracle, n, kind):
    a = I.kinds(n, 3 + n)[kind]
    assert np.array_equal(oracle.tile_find(a), pyref.tile_find(a))
    assert np.array_equal(oracle.radix_find(a), pyref.radix_find(a))


@pytest.mark.parametrize("n", [5, 40, 300, 2100, 9000, 40000])
@pytest.mark.parametrize("kind", ["markov", "runs", "rep7", "records", "zeros"])
def test_tokenizer_matches_python_restatement(oracle, n, kind):
    a = I.kinds(n, 5 + n)[kind]
    desc = oracle.match_table(a)
    assert oracle.tokenize_with(a, desc) == pyref.tokenize(a, desc)


@pytest.mark.parametrize("name,a", I.parity_cases(1 << 20)[::3])
def test_frames_round_trip_reference_decoder(oracle, name, a):
    if not oracle.ref_decoder_available():
        pytest.skip("reference decoder not built (needs the reference checkout)")
    n = len(a)
    for fr in (oracle.compress_p0(a), oracle.compress_p1(a)):
        if n == 0:
            assert fr == b""
            continue
        if fr[4] & 0x04 == 0 and fr[4] & 0x08 == 0 and n > 65535:
            pytest.fail("large frame without the extended directory")
        # P0 raw literals may be misread by both decoders (reference behaviour)
        if fr is not None and not (fr[4] & 0x80) and oracle.raw_literals_misparse(oracle.tokenize(a)[2]):
            continue
        assert oracle.ref_decompress(fr, n) == bytes(a), name


def test_p1_never_misparses(oracle):
    # raw literals starting with 'VA\x01' force the V-ANS container (or the
    # uncompressed frame) in the entropy-coded profile
    a = np.frombuffer(b"VA\x01" + bytes(range(200)) * 3, np.uint8)
    fr = oracle.compress_p1(a)
    assert oracle.ref_decompress(fr, len(a)) == bytes(a)


def test_split_commands_matches_reference_c(oracle):
    import ctypes as C
    if not oracle.ref_decoder_available():
        pytest.skip("reference decoder not built")
    D = oracle.dec()
    for name, a in I.parity_cases(200_000)[::11]:
        cmd = oracle.tokenize(a)[0]
        if not cmd:
            continue
        op, meta, var = oracle.split_commands(cmd)
        n = len(cmd)
        bo, bm, bv = (np.zeros(n + 8, np.uint8) for _ in range(3))
        lo, lm, lv = C.c_size_t(), C.c_size_t(), C.c_size_t()
        c = np.frombuffer(cmd, np.uint8)
        r = D.przm_split_commands(c.ctypes.data_as(C.POINTER(C.c_uint8)), n,
                                  bo.ctypes.data_as(C.POINTER(C.c_uint8)), n + 8, C.byref(lo),
                                  bm.ctypes.data_as(C.POINTER(C.c_uint8)), n + 8, C.byref(lm),
                                  bv.ctypes.data_as(C.POINTER(C.c_uint8)), n + 8, C.byref(lv))
        assert r == 0
        assert (bytes(bo[:lo.value]), bytes(bm[:lm.value]), bytes(bv[:lv.value])) == (op, meta, var), name


def test_mode8_activation_kat(oracle):
    # core/commands/commands_test.go:649-695
    s = oracle.package_commands(bytes([0x06]) * 500)
    assert s[0] == 0x08 and len(s) < 500
    assert oracle.package_commands(bytes([1, 2, 3])) == bytes([0x09, 1, 2, 3])


def test_cross_decode_kat(oracle):
    # core/commands/commands_test.go:697-779: a hand-built Mode 8 frame with
    # explicit matches decodes to "PRZM_EXPLICIT_TEST_" * 3
    if not oracle.ref_decoder_available():
        pytest.skip("reference decoder not built")
    lit = b"PRZM_EXPLICIT_TEST_"
    expected = lit * 3
    cmds = bytes([0xF0, 19, 0x8F, 0x00, 0x8F, 0x00])
    op, meta, var = oracle.split_commands(cmds)
    assert (op, meta, var) == (bytes([0xF0, 0x8F, 0x8F]), b"", bytes([19, 0, 0]))
    pk = oracle.package_commands(cmds)
    # PackCommandsMode8 directly (PackageCommandsSection would choose 0x09 here)
    s2 = bytes([0x08]) + len(cmds).to_bytes(4, "little") + (1 + len(op)).to_bytes(4, "little") + (1).to_bytes(4, "little")
    s2 += bytes([0x09]) + op + bytes([0x09]) + bytes([0x09]) + var
    assert pk[0] in (0x08, 0x09)
    s3 = bytes([19, 19])
    frame = b"PRZM" + bytes([0]) + len(expected).to_bytes(3, "little") + len(s2).to_bytes(2, "little")
    frame += len(s3).to_bytes(2, "little") + bytes([0, 16, 0, 0, 0, 0, 0, 0]) + s2 + s3 + lit
    assert oracle.ref_decompress(frame, len(expected)) == expected


@pytest.mark.parametrize("seed", range(6))
def test_vans_round_trip_reference_decoder(oracle, seed):
    # core/literals/literals_test.go:139-175 (V-ANS round trip, seed 42 style)
    if not oracle.ref_decoder_available():
        pytest.skip("reference decoder not built")
    rng = np.random.default_rng(42 + seed)
    for n in (1, 2, 3, 4, 5, 17, 1000, 65537):
        a = rng.integers(0, 1 + 15 * seed, n, dtype=np.uint8) if seed else np.full(n, 7, np.uint8)
        for c in (oracle.adaptive_vans(a), oracle.vans_encode_host(a)):
            assert c[:3] == b"VA\x01"
            assert oracle.ref_decode_vans_literals(c) == bytes(a)
        m8 = oracle.encode_meta8(a)
        assert oracle.ref_decode_meta8(m8, n) == bytes(a)


def test_vans_header_kat(oracle):
    # gpu/gpu_test.go:648-677: 'V','A',01,01 then LE32 length
    a = np.frombuffer(b"hello gpu v-ans encoder " * 40, np.uint8)
    c = oracle.vans_encode_host(a)
    assert c[:4] == b"VA\x01\x01" and int.from_bytes(c[4:8], "little") == len(a)
    assert oracle.adaptive_vans(a)[:4] == b"VA\x01\x00"


def test_normalisers(oracle):
    rng = np.random.default_rng(3)
    for t in range(200):
        k = int(rng.integers(1, 257))
        counts = np.zeros(256, np.uint32)
        idx = rng.choice(256, k, replace=False)
        counts[idx] = rng.integers(1, [2, 50, 100000][t % 3], k)
        for f in (oracle.normalize_frequencies(counts), oracle.normalize_freq(counts)):
            assert int(f.sum()) == 4096
            assert np.all((f > 0) == (counts > 0))
        # NormalizeFrequencies gives the shortfall to the largest counts first
        f = oracle.normalize_frequencies(counts)
        base = 1 + (counts.astype(np.int64) * (4096 - k)) // counts.sum()
        bumped = np.nonzero((f.astype(np.int64) - np.where(counts > 0, base, 0)) == 1)[0]
        if len(bumped):
            order = sorted(np.nonzero(counts)[0], key=lambda s: (-int(counts[s]), s))
            assert set(bumped) == set(order[:len(bumped)])


def test_normalize_freq_ties_follow_go_sort(oracle):
    """When no equal remainders straddle the +1 cutoff the Go sort's tie order
    cannot matter and the result equals a plain descending-remainder pick."""
    rng = np.random.default_rng(9)
    checked = 0
    for _ in range(300):
        counts = rng.integers(0, 5000, 256).astype(np.uint32)
        if oracle.normalize_freq_tie_straddles(counts):
            continue
        tot, act = int(counts.sum()), int((counts > 0).sum())
        rt = 4096 - act
        f = np.where(counts > 0, 1 + counts.astype(np.int64) * rt // tot, 0)
        rem = counts.astype(np.int64) * rt % tot
        diff = 4096 - int(f.sum())
        order = sorted(np.nonzero(counts)[0], key=lambda s: -int(rem[s]))
        for s in order[:diff]:
            f[s] += 1
        assert np.array_equal(f, oracle.normalize_freq(counts))
        checked += 1
    assert checked > 100


def test_serialize_matrix_layout(oracle):
    f = np.zeros(256, np.uint16)
    f[0x41], f[0x42], f[0xF3] = 4000, 95, 1
    m = oracle.serialize_matrix(f)
    # rowMask rows 4 and 15; row 4 colMask {1,2}: 4000 -> two bytes, 95 -> one
    assert m == bytes([0x10, 0x80, 0x06, 0x00, 0x8F, 0xA0, 95, 0x08, 0x00, 1])


def _digest(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def test_golden_fixtures(oracle):
    """Oracle outputs on the committed fixtures (tests/golden/make_golden.py)."""
    path = os.path.join(HERE, "golden", "oracle_golden.json")
    g = json.load(open(path))
    from przm_b200 import workloads as W
    for case in g["cases"]:
        a = W.gen(case["kind"], case["seed"], case["n"])
        assert _digest(a.tobytes()) == case["input_sha256"], case["name"]
        assert _digest(oracle.match_table(a).tobytes()) == case["match_table_sha256"], case["name"]
        c, o, l = oracle.tokenize(a)
        assert _digest(c + b"|" + o + b"|" + l) == case["tokens_sha256"], case["name"]
        assert _digest(oracle.compress_p0(a)) == case["p0_sha256"], case["name"]
        assert _digest(oracle.compress_p1(a)) == case["p1_sha256"], case["name"]
        assert _digest(oracle.vans_encode_host(a)) == case["vans_host_sha256"], case["name"]
