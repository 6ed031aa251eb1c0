"""GPU: batched and device-resident runs give the same bytes as one call per
input; the stream-batch V-ANS matches the oracle with both normalisers."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from przm_b200 import gpu
from przm_b200 import workloads as W
from tests import inputs as I

pytestmark = pytest.mark.gpu


def _uneven(count: int, seed: int) -> list[np.ndarray]:
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(1), np.log(2 << 20), count))).astype(int)
    sizes[:4] = [0, 1, 65536, 65537]
    return [W.mixture(seed + i, int(n))[0] for i, n in enumerate(sizes)]


@pytest.mark.parametrize("profile", [gpu.PROFILE_D2D, gpu.PROFILE_ANS])
def test_batch_equals_single_calls(comp, oracle, profile):
    xs = _uneven(40, 1234)
    fb, st, _ = comp.CompressBatch(xs, profile, batched=True)
    fp, sp, _ = comp.CompressBatch(xs, profile, batched=False)
    assert all(s == 0 for s in st) and all(s == 0 for s in sp)
    ref = oracle.compress_p1 if profile == gpu.PROFILE_ANS else oracle.compress_p0
    for x, a, b in zip(xs, fb, fp):
        assert a == b == ref(x)


def test_device_batch_graph_replay(comp, oracle):
    from przm_b200 import devmem
    xs = _uneven(24, 99)
    sizes = [len(x) for x in xs]
    b = gpu.DeviceBatch(comp, sizes, gpu.PROFILE_ANS)
    try:
        host = np.zeros(int(b.in_offs[-1]) + max(sizes[-1], 1) + 64, np.uint8)
        for x, o in zip(xs, b.in_offs):
            host[int(o):int(o) + len(x)] = x
        devmem.upload_to(b.d_in, host)
        for graph in (False, True, True):
            b.enqueue(graph=graph)
            fs = b.frame_sizes()
            for x, o, s in zip(xs, b.out_offs, fs):
                assert devmem.download(b.d_out + int(o), int(s)) == oracle.compress_p1(x)
        assert b.launches() >= 6
    finally:
        b.close()


@pytest.mark.parametrize("profile", [gpu.PROFILE_D2D, gpu.PROFILE_ANS])
def test_plain_per_input_launches_equal_the_batched_launch(comp, oracle, profile):
    from przm_b200 import devmem
    xs = _uneven(30, 321)
    sizes = [len(x) for x in xs]
    b = gpu.DeviceBatch(comp, sizes, profile)
    try:
        host = np.zeros(int(b.in_offs[-1]) + max(sizes[-1], 1) + 64, np.uint8)
        for x, o in zip(xs, b.in_offs):
            host[int(o):int(o) + len(x)] = x
        devmem.upload_to(b.d_in, host)
        b.enqueue(graph=True)
        fs = b.frame_sizes().copy()
        batched = [devmem.download(b.d_out + int(o), int(s)) for o, s in zip(b.out_offs, fs)]
        devmem.upload_to(b.d_out, np.zeros(int(b.out_offs[-1]) + 64, np.uint8))
        launches = b.enqueue_plain()
        assert launches > b.launches()  # one launch sequence per non-empty input
        fp = b.frame_sizes()
        assert np.array_equal(fs, fp)
        ref = oracle.compress_p1 if profile == gpu.PROFILE_ANS else oracle.compress_p0
        for x, o, s, want in zip(xs, b.out_offs, fp, batched):
            got = devmem.download(b.d_out + int(o), int(s))
            assert got == want == ref(x)
    finally:
        b.close()


@pytest.mark.parametrize("norm", [gpu.NORM_GO, gpu.NORM_CPU])
def test_vans_batch_config1_shapes(comp, oracle, norm):
    streams = W.config1(count=8, size=1 << 18)
    from przm_b200 import devmem
    host = np.concatenate(streams)
    d_in = devmem.upload(host)
    lens = np.array([len(s) for s in streams], np.uint32)
    in_offs = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.uint64)
    out_offs = np.array([i * (2 * (1 << 18) + 1024) for i in range(len(streams))], np.uint64)
    d_out = devmem.alloc(int(out_offs[-1]) + 2 * (1 << 18) + 1024)
    ol = comp.VANSEncodeBatch(d_in.ptr, in_offs, lens, norm, d_out.ptr, out_offs)
    for s, o, n in zip(streams, out_offs, ol):
        got = devmem.download(d_out.ptr + int(o), int(n))
        if norm == gpu.NORM_GO:
            assert got == oracle.vans_encode_host(s)
        else:
            assert got == oracle.adaptive_vans(s)


def test_vans_encode4x_gpu_given_tables(comp, oracle):
    from przm_b200 import devmem
    a = W.zipf(5, 300_000)
    counts = np.bincount(a, minlength=256).astype(np.uint32)
    freq = gpu.NormalizeFreq(counts)
    cdf = gpu.BuildCDF(freq)
    mat = gpu.SerializeMatrix(freq)
    d_in = devmem.upload(a)
    d_out = devmem.alloc(2 * len(a) + 1024)
    n, ms, gb = comp.VANSEncode4xGPU(d_in.ptr, d_out.ptr, len(a), freq, cdf, mat)
    assert devmem.download(d_out.ptr, n) == oracle.vans_encode(a, freq, 0x01)
    assert np.array_equal(freq, oracle.normalize_freq(counts))
