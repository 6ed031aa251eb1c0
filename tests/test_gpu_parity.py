"""GPU parity: the CUDA path against the oracle, byte for byte, through the
C ABI (przm_b200.gpu binds include/przmgpu.h).  Integer path: the bar is
bit-exact equality."""
from __future__ import annotations

import numpy as np
import pytest

from tests import inputs as I

pytestmark = pytest.mark.gpu

CASES = I.parity_cases(1 << 20)


def _ids(cases):
    return [c[0] for c in cases]


@pytest.mark.parametrize("name,a", CASES, ids=_ids(CASES))
def test_match_table(comp, oracle, name, a):
    assert np.array_equal(comp.MatchTable(a), oracle.match_table(a)), name


@pytest.mark.parametrize("name,a", CASES, ids=_ids(CASES))
def test_tokenize(comp, oracle, name, a):
    c, o, l, prof = comp.Tokenize(a)
    assert (c, o, l) == oracle.tokenize(a), name
    assert prof.CmdBytes == len(c) and prof.LiteralBytes == len(l)


@pytest.mark.parametrize("name,a", CASES, ids=_ids(CASES))
def test_compress_d2d(comp, oracle, name, a):
    fr, prof = comp.CompressD2D(a)
    assert fr == oracle.compress_p0(a), name


@pytest.mark.parametrize("name,a", CASES, ids=_ids(CASES))
def test_compress_entropy_frame(comp, oracle, name, a):
    fr, _ = comp.Compress(a)
    ref = oracle.compress_p1(a)
    assert fr == ref, name
    if len(a) and oracle.ref_decoder_available():
        assert oracle.ref_decompress(fr, len(a)) == bytes(a)


@pytest.mark.parametrize("name,a", CASES[::4], ids=_ids(CASES[::4]))
def test_match_lz77(comp, oracle, name, a):
    pos, off, ln, _ = comp.MatchLZ77Arrays(a)
    opos, odsc = oracle.match_lz77(a)
    assert np.array_equal(pos, opos)
    assert np.array_equal(off, odsc & 0xFFFFF)
    assert np.array_equal(ln, odsc >> 20)


def test_match_lz77_streaming_chunks(comp, oracle):
    a = I.periodic(3 << 20)
    for chunk in (1 << 20, 1536 * 1024):
        pos, off, ln, prof = comp.MatchLZ77Arrays(a, chunk)
        opos, odsc = oracle.match_lz77(a, oracle.streaming_chunk(len(a), chunk))
        assert np.array_equal(pos, opos) and np.array_equal(off, odsc & 0xFFFFF) and np.array_equal(ln, odsc >> 20)
        assert prof.PipelinedChunks == (len(a) + chunk - 1) // chunk
    # matches never cross chunk boundaries (gpu/bridge.go:1494-1496)
    pos, off, ln, _ = comp.MatchLZ77Arrays(a, 1 << 20)
    assert np.all((pos // (1 << 20)) == ((pos - off) // (1 << 20)))


def test_match_lz77_cross_tile_and_valid(comp):
    # gpu/gpu_test.go:241-360: long-distance matches exist and every match verifies
    a = I.periodic(4 << 20)
    pos, off, ln, _ = comp.MatchLZ77Arrays(a)
    assert len(pos) > 0 and np.any(off > 32768)
    assert np.all(np.diff(pos.astype(np.int64)) > 0)
    b = a.tobytes()
    for p, o, l in list(zip(pos, off, ln))[:: max(1, len(pos) // 2000)]:
        assert 4 <= l and 0 < o <= p and b[p:p + l] == b[p - o:p - o + l]


@pytest.mark.parametrize("n", [1, 3, 1000, 65536, 1 << 20, (4 << 20) + 3])
def test_histogram(comp, oracle, n):
    a = np.random.default_rng(n).integers(0, 256, n, dtype=np.uint8)
    counts, _ = comp.ComputeHistogramHost(a)
    assert np.array_equal(counts, np.bincount(a, minlength=256))


@pytest.mark.parametrize("name,a", CASES[::5], ids=_ids(CASES[::5]))
def test_vans_encode_host(comp, oracle, name, a):
    c, _ = comp.VANSEncode4xHost(a)
    assert c == oracle.vans_encode_host(a), name


def test_pack_stream_flat(comp):
    # gpu/gpu_test.go:620-646
    a = np.arange(100000, dtype=np.uint32).view(np.uint8)
    out, _ = comp.PackStreamFlatHost(a)
    assert out[0] == 0 and int.from_bytes(out[1:5], "little") == len(a) and out[5:] == a.tobytes()
    assert comp.PackStreamFlatHost(b"")[0] == bytes(5)


def test_tokenize_device_zero_copy(comp):
    # gpu/tokenizer_test.go:269-364: device streams equal the host Tokenize
    a = I.kinds(700_000, 77)["records"]
    c, o, l, _ = comp.Tokenize(a)
    st, _ = comp.TokenizeDevice(a)
    assert (st.CmdLen, st.OffLen, st.LitLen) == (len(c), len(o), len(l))
    assert comp.DownloadDeviceBytes(st.DFinalCmds, st.CmdLen) == c
    assert comp.DownloadDeviceBytes(st.DFinalOffs, st.OffLen) == o
    assert comp.DownloadDeviceBytes(st.DFinalLits, st.LitLen) == l
    tot = np.frombuffer(comp.DownloadDeviceBytes(st.DTotals, 12), np.uint32)
    assert list(tot) == [len(c), len(o), len(l)]


def test_encode_d2d_matches_compress_d2d(comp, oracle):
    a = I.kinds(300_000, 5)["markov"]
    st, _ = comp.TokenizeDevice(a)
    fr, _ = comp.EncodeD2D(st, len(a), 0)
    assert fr == oracle.compress_p0(a)


def test_empty_inputs(comp):
    assert comp.CompressD2D(b"")[0] == b""
    assert comp.Compress(b"")[0] == b""
    assert comp.Tokenize(b"")[:3] == (b"", b"", b"")
    assert comp.MatchLZ77(b"")[0] == []
    assert comp.VANSEncode4xHost(b"")[0] == b""
