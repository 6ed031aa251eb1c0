"""Full-size parity on the five workload shapes the measurements use:
  c0  one 4 MiB order-1 Markov input with copies, one frame;
  c1  64 x 1 MiB Zipf(1.1) streams, histogram + V-ANS with both normalisers;
  c2  256 x 1 MiB segments of the mixture as one device-resident batch;
  c3  4096 inputs log-uniform in [1 KiB, 4 MiB] as one batch;
  c4  serving sizes (log-normal, median 64 KiB, below 16 MiB), largest included.
Bytes are compared with the oracle on every frame or on a fixed sample, and
frames are decoded by the reference's C decoder (oracle/_ref/libprzm_dec.so).
Sizes are those of the measurements, so this file takes the longest."""
from __future__ import annotations

import numpy as np
import pytest

from przm_b200 import devmem, gpu
from przm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _decodes(oracle, frame: bytes, a: np.ndarray) -> bool:
    return not oracle.ref_decoder_available() or oracle.ref_decompress(frame, len(a)) == a.tobytes()


def test_c0_one_4mib_frame(comp, oracle):
    a = W.config0()
    assert len(a) == 4 << 20
    assert np.array_equal(comp.MatchTable(a), oracle.match_table(a))
    cmd, off, lit, _ = comp.Tokenize(a)
    assert (cmd, off, lit) == oracle.tokenize(a)
    counts, _ = comp.ComputeHistogramHost(lit)
    assert np.array_equal(counts, np.bincount(np.frombuffer(lit, np.uint8), minlength=256))
    for profile, want in ((gpu.PROFILE_D2D, oracle.compress_p0(a)), (gpu.PROFILE_ANS, oracle.compress_p1(a))):
        f = comp.Compress(a, profile)[0]
        assert f == want
        assert _decodes(oracle, f, a)


@pytest.mark.parametrize("norm", [gpu.NORM_GO, gpu.NORM_CPU])
def test_c1_64_streams(comp, oracle, norm):
    streams = W.config1()
    assert len(streams) == 64 and all(len(s) == 1 << 20 for s in streams)
    host = np.concatenate(streams)
    d_in = devmem.upload(host)
    lens = np.array([len(s) for s in streams], np.uint32)
    in_offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64)
    slot = 2 * (1 << 20) + 1024
    out_offs = np.arange(len(streams), dtype=np.uint64) * slot
    d_out = devmem.alloc(slot * len(streams))
    ol = comp.VANSEncodeBatch(d_in.ptr, in_offs, lens, norm, d_out.ptr, out_offs)
    for i, s in enumerate(streams):
        got = devmem.download(d_out.ptr + int(out_offs[i]), int(ol[i]))
        want = oracle.vans_encode_host(s) if norm == gpu.NORM_GO else oracle.adaptive_vans(s)
        assert got == want, i
        if i % 16 == 0 and oracle.ref_decoder_available():
            assert oracle.ref_decode_vans_literals(got) == s.tobytes()
        counts, _, _ = comp.ComputeHistogramGPU(d_in.ptr + int(in_offs[i]), len(s))
        assert np.array_equal(counts, np.bincount(s, minlength=256))


def _batch_frames(comp, xs):
    b = gpu.DeviceBatch(comp, [len(a) for a in xs], gpu.PROFILE_ANS)
    try:
        b.upload(np.concatenate(xs))
        b.enqueue(graph=True)
        sizes = b.frame_sizes()
        out = [devmem.download(b.d_out + int(o), int(s)) for o, s in zip(b.out_offs, sizes)]
    finally:
        b.close()
    return out


def test_c2_256_frames(comp, oracle):
    xs = W.config2()
    frames = _batch_frames(comp, xs)
    for i in range(0, len(xs), 8):
        assert frames[i] == oracle.compress_p1(xs[i]), i
    for f, a in zip(frames, xs):  # every frame decodes
        assert _decodes(oracle, f, a)


def test_c3_4096_uneven_inputs(comp, oracle):
    xs = W.config3()
    frames = _batch_frames(comp, xs)
    sample = range(0, len(xs), 16)
    for i in sample:
        assert frames[i] == oracle.compress_p1(xs[i]), i
        assert _decodes(oracle, frames[i], xs[i])


def test_c4_request_sizes_up_to_the_cap(comp, oracle):
    sizes = W.config4_sizes(20000)
    picks = [int(sizes.max()), int(np.percentile(sizes, 99)), int(np.median(sizes)), int(sizes.min())]
    assert picks[0] < 16 << 20
    for k, n in enumerate(picks):
        a = W.mixture(0x50525A4D + 4 + k, n)[0]
        f = comp.Compress(a)[0]
        assert f == oracle.compress_p1(a), n
        assert _decodes(oracle, f, a)
