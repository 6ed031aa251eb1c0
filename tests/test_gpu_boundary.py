"""The tokenizer-only and pinned-memory entry points of the boundary:
TokenizeDeviceOnly / TokenizePointersDeviceOnly (gpu/bridge.go:1915,2163),
GetPinned (gpu/bridge.go:452) and PinnedBufferPool (gpu/memory.go:98-165).

Written after the reference's own tests: the device-only tokenizer must give
the streams of the Tokenize call that staged its input
(gpu/tokenizer_test.go:195-225,353-362); a pool hands back the buffer it was
given (gpu/gpu_test.go:155-185) and survives concurrent Get/Put
(tests/e2e/gpu_tier3_interactions_test.go:325-380)."""
from __future__ import annotations

import threading

import numpy as np
import pytest

from przm_b200 import gpu
from przm_b200 import workloads as W

pytestmark = pytest.mark.gpu

INPUTS = [("markov-70001", W.gen("markov", 41, 70001)), ("records-40000", W.gen("records", 42, 40000)),
          ("table-1MiB", W.gen("table", 43, 1 << 20))]


@pytest.mark.parametrize("name,a", INPUTS, ids=[n for n, _ in INPUTS])
def test_tokenize_device_only_repeats_the_staged_input(comp, oracle, name, a):
    cmd, off, lit, _ = comp.Tokenize(a)
    assert (cmd, off, lit) == tuple(oracle.tokenize(a))
    for _ in range(2):  # the staged input and match table stay valid across runs
        c2, o2, l2, prof = comp.TokenizeDeviceOnly(len(a))
        assert (c2, o2, l2) == (cmd, off, lit)
        assert prof.KernelTimeMs >= 0 and prof.LiteralBytes == len(lit)
    st, _ = comp.TokenizePointersDeviceOnly(len(a))
    assert (st.CmdLen, st.OffLen, st.LitLen) == (len(cmd), len(off), len(lit))
    assert comp.DownloadDeviceBytes(st.DFinalCmds, st.CmdLen) == cmd
    assert comp.DownloadDeviceBytes(st.DFinalOffs, st.OffLen) == off
    assert comp.DownloadDeviceBytes(st.DFinalLits, st.LitLen) == lit


def test_tokenize_device_only_needs_a_staged_input(comp):
    a = W.gen("markov", 44, 5000)
    comp.Tokenize(a)
    with pytest.raises(gpu.GPUError) as e:
        comp.TokenizeDeviceOnly(len(a) + 1)
    assert e.value.code == -1
    # a many-input call replaces the staged single input
    comp.CompressBatch([a, a], gpu.PROFILE_D2D)
    with pytest.raises(gpu.GPUError):
        comp.TokenizePointersDeviceOnly(len(a))
    assert comp.TokenizeDeviceOnly(0)[:3] == (b"", b"", b"")


def test_pinned_pool_reuses_its_buffers():
    pool = gpu.PinnedBufferPool(64 * 1024, 4)
    try:
        assert pool.Pooled() == 4
        buf = pool.Get()
        assert len(buf.Bytes) == 64 * 1024 and buf.Ptr != 0
        buf.Bytes[0] = 0xAA
        buf.Bytes[-1] = 0x55
        pool.Put(buf)
        buf2 = pool.Get()
        assert buf2.Ptr == buf.Ptr and buf2.Bytes[0] == 0xAA and buf2.Bytes[-1] == 0x55
        pool.Put(buf2)
        # a buffer of another length is ignored by Put, as in the reference
        pool.Put(gpu.PinnedBuffer(buf2.Bytes[:10], buf2.Ptr))
        assert pool.Pooled() == 4
        # beyond max(initialCap, 8) buffers a Put frees instead of keeping
        many = [pool.Get() for _ in range(12)]
        for b in many:
            pool.Put(b)
        assert pool.Pooled() == 8
    finally:
        pool.Close()


def test_pinned_pool_concurrent_get_put():
    pool = gpu.PinnedBufferPool(64 * 1024, 4)
    errors: list[str] = []

    def worker(wid: int) -> None:
        fill = wid + 1
        for _ in range(30):
            b = pool.Get()
            if len(b.Bytes) != 64 * 1024 or b.Ptr == 0:
                errors.append(f"worker {wid}: bad buffer")
                return
            b.Bytes[:] = fill
            if not np.all(b.Bytes == fill):  # nobody else holds this buffer
                errors.append(f"worker {wid}: buffer shared")
            pool.Put(b)

    threads = [threading.Thread(target=worker, args=(w,)) for w in range(16)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    pool.Close()
    assert not errors, errors


def test_get_pinned_pools_by_power_of_two(comp):
    b1, p1 = comp.GetPinned(100_000)
    assert len(b1.Bytes) == 100_000 and p1.bufSize == 131072
    b1.Bytes[:] = 7
    # the lease is sliced to 100000 bytes, so Put keeps it only when it is
    # handed back with the pool's buffer size (Put checks the length)
    p1.Put(b1)
    assert p1.Pooled() == 0
    p1.Put(gpu.PinnedBuffer(np.empty(p1.bufSize, np.uint8), b1.Ptr))
    assert p1.Pooled() == 1
    b2, p2 = comp.GetPinned(131072)
    assert p2.bufSize == 131072 and b2.Ptr == b1.Ptr  # the same pool, the same buffer back
    p2.Put(b2)
    b3, p3 = comp.GetPinned(131073)
    assert p3.bufSize == 262144 and b3.Ptr != b1.Ptr
    p3.Put(b3)
