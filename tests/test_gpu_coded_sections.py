"""GPU: frames with the CPU compressor's coded sections from the batch
pipeline against the oracle, byte for byte, and through the reference
decoder.  P2 (PROFILE_ANS_DIST): Section 3 as PackageOffsetsSection
(core/distance/distance.go:825-849), against or_compress_p2.  P3
(PROFILE_ANS_SHEAF): also Section 4 as PackageLiteralsSection
(core/literals/literals.go:664-693), against or_compress_p3.  Every parity
case one call at a time, batches reaching every Section 3 form (empty, 0x09
varints, 0x0B / 0x0A / 0x06 containers with Mode 12 and adaptive code
streams) and every Section 4 form (raw, adaptive container, each of the four
foliations), device batches (one launch sequence, graph replay, per-input
launches) and the serving engine."""
from __future__ import annotations

import numpy as np
import pytest

from przm_b200 import gpu
from przm_b200 import workloads as W
from tests import inputs as I
from tests.frames import section3_form, section4_form

pytestmark = pytest.mark.gpu

CASES = I.parity_cases(1 << 20)


def _ids(cases):
    return [c[0] for c in cases]


PROFILES = [gpu.PROFILE_ANS_DIST, gpu.PROFILE_ANS_SHEAF]


def _want(oracle, profile, a) -> bytes:
    return oracle.compress_p2(a) if profile == gpu.PROFILE_ANS_DIST else oracle.compress_p3(a)


def _check(oracle, profile, a, fr):
    assert fr == _want(oracle, profile, a)
    if len(a) and oracle.ref_decoder_available():
        assert oracle.ref_decompress(fr, len(a)) == bytes(a)


@pytest.mark.parametrize("profile", PROFILES)
@pytest.mark.parametrize("name,a", CASES, ids=_ids(CASES))
def test_frame(comp, oracle, name, a, profile):
    fr, _ = comp.Compress(a, profile)
    _check(oracle, profile, a, fr)


def form_inputs() -> list[np.ndarray]:
    xs = []
    for n in (4096, 20_000, 200_000):
        xs += list(I.kinds(n, 5 + n).values())
    xs += [W.gen("table", 3, 4 << 20), W.gen("records", 3, 4 << 20)]
    xs += [I.ident_text(200_000, 7), I.tagged_numbers(20_000, 7)]
    return xs


@pytest.mark.parametrize("profile", PROFILES)
def test_section_forms(comp, oracle, profile):
    xs = form_inputs()
    frames, st, _ = comp.CompressBatch(xs, profile)
    assert all(s == 0 for s in st)
    for a, fr in zip(xs, frames):
        _check(oracle, profile, a, fr)
    forms = {section3_form(fr) for fr in frames}
    assert {"empty", "09", "0B-M12", "0A-M12", "0A-AD", "06-AD"} <= forms, forms
    if profile == gpu.PROFILE_ANS_SHEAF:
        forms4 = {section4_form(fr) for fr in frames}
        assert {"raw", "AD", "SH0", "SH1", "SH2", "SH3"} <= forms4, forms4


def _uneven(count: int, seed: int) -> list[np.ndarray]:
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(1), np.log(2 << 20), count))).astype(int)
    sizes[:4] = [0, 1, 65536, 65537]
    return [W.mixture(seed + i, int(n))[0] for i, n in enumerate(sizes)]


@pytest.mark.parametrize("profile", PROFILES)
def test_device_batch(comp, oracle, profile):
    from przm_b200 import devmem
    xs = _uneven(30, 2718)
    sizes = [len(x) for x in xs]
    want = [_want(oracle, profile, x) for x in xs]
    b = gpu.DeviceBatch(comp, sizes, profile)
    try:
        host = np.zeros(int(b.in_offs[-1]) + max(sizes[-1], 1) + 64, np.uint8)
        for x, o in zip(xs, b.in_offs):
            host[int(o):int(o) + len(x)] = x
        devmem.upload_to(b.d_in, host)
        for run in ("batched", "graph", "graph", "plain"):
            if run == "plain":
                assert b.enqueue_plain() > 0
            else:
                b.enqueue(graph=run == "graph")
            fs = b.frame_sizes()
            for w, o, s in zip(want, b.out_offs, fs):
                assert devmem.download(b.d_out + int(o), int(s)) == w, run
        st = b.stats()
        assert st["frame_bytes"] == sum(len(w) for w in want)
    finally:
        b.close()


@pytest.mark.parametrize("profile", PROFILES)
def test_serving(comp, oracle, profile):
    xs = _uneven(12, 99)
    srv = gpu.Server(comp, profile, mem_budget=16 << 30, max_inflight=2)
    try:
        ids = [srv.submit(x) for x in xs]
        got = [srv.poll(r, 2 * len(x) + 4096)[0] for r, x in zip(ids, xs)]
    finally:
        srv.close()
    for a, fr in zip(xs, got):
        _check(oracle, profile, a, fr)
