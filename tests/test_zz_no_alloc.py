"""przmg_vans_encode_noalloc: the allocation-free single-stream V-ANS entry
point (static device scratch).  It must give the same container bytes as
przmg_vans_encode_batch with one stream and as the oracle's encoder on
consecutive calls, allocate no device memory, and refuse sizes beyond its
fixed scratch.  The file name sorts last, so in a full run it also goes
after every other GPU test of the process."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from przm_b200 import _lib, devmem, gpu
from przm_b200 import workloads as W

pytestmark = pytest.mark.gpu

MAXN = _lib.NOALLOC_MAX_N


def _noalloc(d_in: int, n: int, norm: int, d_out: int, cap: int, d_len: int) -> int:
    return _lib.lib().przmg_vans_encode_noalloc(d_in, n, norm, d_out, cap, d_len, 0)


def _encode_noalloc(d_in: int, n: int, norm: int, d_out: int, d_len: int) -> bytes:
    rc = _noalloc(d_in, n, norm, d_out, 1024 + 2 * MAXN, d_len)
    assert rc == 0, _lib.lib().przmg_last_error()
    devmem.rt().cudaDeviceSynchronize()
    size = int(np.frombuffer(devmem.download(d_len, 4), np.uint32)[0])
    return devmem.download(d_out, size)


def _encode_batch(comp, d_in: int, n: int, norm: int, d_out: int) -> bytes:
    ol = comp.VANSEncodeBatch(d_in, [0], [n], norm, d_out, [0])
    return devmem.download(d_out, int(ol[0]))


def _encode_oracle(oracle, a: np.ndarray, norm: int) -> bytes:
    # VANSEncode4xHost (NormalizeFreq, flag 0x01) or EncodeAdaptiveVANS4x
    # (NormalizeFrequencies, flag 0x00) restated on the CPU
    return oracle.vans_encode_host(a) if norm == gpu.NORM_GO else oracle.adaptive_vans(a)


def _free_device_bytes() -> int:
    free, total = C.c_size_t(), C.c_size_t()
    rt = devmem.rt()
    rt.cudaMemGetInfo.argtypes = [C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
    assert rt.cudaMemGetInfo(C.byref(free), C.byref(total)) == 0
    return free.value


@pytest.mark.parametrize("norm", [gpu.NORM_GO, gpu.NORM_CPU])
def test_noalloc_matches_batch_on_consecutive_calls(oracle, norm):
    # inputs of different size and statistics back to back: a call that saw
    # the previous call's histogram, table or lane records would differ
    inputs = [W.zipf(101, MAXN), W.gen("markov", 102, 300_001), W.gen("uniform", 103, 65_537)]
    d_in = devmem.alloc(MAXN + 64)
    d_out = devmem.alloc(1024 + 2 * MAXN)
    d_ref = devmem.alloc(1024 + 2 * MAXN)
    d_len = devmem.alloc(16)
    got = []
    for a in inputs:  # the allocation-free calls come first, before any context exists in a lone run
        devmem.upload_to(d_in.ptr, a)
        got.append(_encode_noalloc(d_in.ptr, len(a), norm, d_out.ptr, d_len.ptr))
    comp = gpu.GetGlobalCompressor()
    for a, g in zip(inputs, got):
        devmem.upload_to(d_in.ptr, a)
        want = _encode_batch(comp, d_in.ptr, len(a), norm, d_ref.ptr)
        assert len(g) == len(want) and g == want
        assert g == _encode_oracle(oracle, a, norm)
    # and the same input twice in a row gives the same bytes
    devmem.upload_to(d_in.ptr, inputs[1])
    again = [_encode_noalloc(d_in.ptr, len(inputs[1]), norm, d_out.ptr, d_len.ptr) for _ in range(2)]
    assert again[0] == again[1] == got[1]


def test_noalloc_small_and_empty_streams(oracle):
    comp = gpu.GetGlobalCompressor()
    d_in = devmem.alloc(4096)
    d_out = devmem.alloc(1024 + 2 * MAXN)
    d_ref = devmem.alloc(1024 + 2 * MAXN)
    d_len = devmem.alloc(16)
    for n in (0, 1, 3, 4, 63, 64, 65, 1000):
        a = W.zipf(200 + n, max(n, 1))[:n]
        if n:
            devmem.upload_to(d_in.ptr, a)
        got = _encode_noalloc(d_in.ptr, n, gpu.NORM_CPU, d_out.ptr, d_len.ptr)
        want = _encode_batch(comp, d_in.ptr, n, gpu.NORM_CPU, d_ref.ptr)
        assert got == want, n
        if n:
            assert got == _encode_oracle(oracle, a, gpu.NORM_CPU), n


def test_noalloc_allocates_no_device_memory():
    # buffers first, then one call (the first call on a device may load the
    # module), then the free device memory must not move over more calls
    d_in = devmem.alloc(MAXN + 64)
    d_out = devmem.alloc(1024 + 2 * MAXN)
    d_len = devmem.alloc(16)
    a = W.gen("markov", 301, MAXN)
    devmem.upload_to(d_in.ptr, a)
    first = _encode_noalloc(d_in.ptr, MAXN, gpu.NORM_GO, d_out.ptr, d_len.ptr)
    before = _free_device_bytes()
    for norm in (gpu.NORM_GO, gpu.NORM_CPU, gpu.NORM_GO):
        _encode_noalloc(d_in.ptr, MAXN, norm, d_out.ptr, d_len.ptr)
    assert _free_device_bytes() == before
    assert _encode_noalloc(d_in.ptr, MAXN, gpu.NORM_GO, d_out.ptr, d_len.ptr) == first


def test_noalloc_rejects_what_does_not_fit():
    L = _lib.lib()
    d_buf = devmem.alloc(64)
    # beyond the static scratch: refused before anything is launched
    assert _noalloc(d_buf.ptr, MAXN + 1, gpu.NORM_GO, d_buf.ptr, 1 << 40, d_buf.ptr) == -5
    assert b"PRZMG_NOALLOC_MAX_N" in L.przmg_last_error()
    # output capacity below 1024 + 2n
    assert _noalloc(d_buf.ptr, 1000, gpu.NORM_GO, d_buf.ptr, 1024 + 2000 - 1, d_buf.ptr) == -4
    # unknown normaliser, null addresses
    assert _noalloc(d_buf.ptr, 10, 7, d_buf.ptr, 1 << 20, d_buf.ptr) == -1
    assert _noalloc(d_buf.ptr, 10, gpu.NORM_GO, 0, 1 << 20, d_buf.ptr) == -1
    assert _noalloc(d_buf.ptr, 10, gpu.NORM_GO, d_buf.ptr, 1 << 20, 0) == -1
    assert _noalloc(0, 10, gpu.NORM_GO, d_buf.ptr, 1 << 20, d_buf.ptr) == -1
    # the length is stored as a u32: its address must be 4-byte aligned
    assert _noalloc(d_buf.ptr, 10, gpu.NORM_GO, d_buf.ptr, 1 << 20, d_buf.ptr + 2) == -1
    assert b"aligned" in L.przmg_last_error()
