"""bench.py's Section 3 and Section 4 legs on CPU: their host logic (layout of
the device buffers, timing loop, the fields of their JSON objects) driven
through a stand-in for device memory and a compressor whose two entry points
are the oracle's section encoders.  No device is touched."""
from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class _Mem:
    """Host arrays addressed like device pointers (base << 40 + offset)."""

    def __init__(self):
        self.bufs = {}

    def _buf(self, a):
        class B:
            pass
        b = B()
        b.a = a
        b.ptr = (len(self.bufs) + 1) << 40
        self.bufs[b.ptr] = b
        return b

    def upload(self, a):
        return self._buf(np.array(a, np.uint8).copy())

    def alloc(self, n):
        return self._buf(np.zeros(n, np.uint8))

    def find(self, ptr):
        b = self.bufs[ptr >> 40 << 40]
        return b.a, ptr - b.ptr

    def download(self, ptr, n):
        a, o = self.find(ptr)
        return bytes(a[o:o + n])


class _Comp:
    def __init__(self, mem, oracle):
        self.mem, self.O = mem, oracle

    def PackageOffsetsBatch(self, dDist, distOffs, counts, dOut, outOffs, outCaps, stream=0):
        a, o = self.mem.find(dDist)
        dist = a[o:].view(np.uint32)
        out, oo = self.mem.find(dOut)
        lens = []
        for off, n, dst, cap in zip(distOffs, counts, outOffs, outCaps):
            s = self.O.package_offsets(dist[int(off):int(off) + int(n)])
            assert len(s) <= cap
            out[oo + int(dst):oo + int(dst) + len(s)] = np.frombuffer(s, np.uint8)
            lens.append(len(s))
        return np.array(lens, np.uint64)

    def PackageLiteralsBatch(self, dIn, inOffs, lens, dOut, outOffs, outCaps, stream=0):
        a, o = self.mem.find(dIn)
        out, oo = self.mem.find(dOut)
        ls, nb = [], []
        for off, n, dst, cap in zip(inOffs, lens, outOffs, outCaps):
            s, f = self.O.package_literals(a[o + int(off):o + int(off) + int(n)])
            assert len(s) <= cap
            out[oo + int(dst):oo + int(dst) + len(s)] = np.frombuffer(s, np.uint8)
            ls.append(len(s))
            nb.append(f)
        return np.array(ls, np.uint64), np.array(nb, np.uint8)


@pytest.fixture()
def legs(monkeypatch, oracle):
    sys.path.insert(0, ROOT)
    import bench
    from przm_b200 import devmem
    mem = _Mem()
    for name in ("upload", "alloc", "download"):
        monkeypatch.setattr(devmem, name, getattr(mem, name))
    return bench, _Comp(mem, oracle)


def test_section3_leg(legs):
    bench, comp = legs
    r = bench.section3_measure(comp, 4, per=3000, calls=2)
    assert r["sections"] == 4 and r["distances"] == 12_000
    assert 0 < r["section_bytes"] < r["varint_bytes"] + 4
    assert sum(r["modes"].values()) == 4 and r["ms_per_call"] > 0


def test_section4_leg(legs):
    bench, comp = legs
    r = bench.section4_measure(comp, 3, size=20_000, calls=2)
    assert r["streams"] == 3 and r["bytes"] == 60_000
    assert 0 < r["section_bytes"] <= r["bytes"] and r["ratio"] <= 1
    assert sum(r["forms"].values()) == 3 and r["gbps"] > 0
