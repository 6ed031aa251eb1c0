"""GPU: P2 frames (PROFILE_ANS_DIST, the entropy-coded frame with Section 3
as PackageOffsetsSection, core/distance/distance.go:825-849, as the
reference's CPU compressor writes it) from the batch pipeline against the
oracle's or_compress_p2, byte for byte, and through the reference decoder:
every parity case one call at a time, a batch reaching every Section 3 form
the frames produce (empty, 0x09 varints, 0x0B / 0x0A / 0x06 containers with
Mode 12 and adaptive code streams), device batches (one launch sequence,
graph replay, per-input launches) and the serving engine."""
from __future__ import annotations

import numpy as np
import pytest

from przm_b200 import gpu
from przm_b200 import workloads as W
from tests import inputs as I
from tests.frames import section3_form

pytestmark = pytest.mark.gpu

CASES = I.parity_cases(1 << 20)


def _ids(cases):
    return [c[0] for c in cases]


def _check(oracle, a, fr):
    assert fr == oracle.compress_p2(a)
    if len(a) and oracle.ref_decoder_available():
        assert oracle.ref_decompress(fr, len(a)) == bytes(a)


@pytest.mark.parametrize("name,a", CASES, ids=_ids(CASES))
def test_p2_frame(comp, oracle, name, a):
    fr, _ = comp.Compress(a, gpu.PROFILE_ANS_DIST)
    _check(oracle, a, fr)


def form_inputs() -> list[np.ndarray]:
    xs = []
    for n in (4096, 20_000, 200_000):
        xs += list(I.kinds(n, 5 + n).values())
    xs += [W.gen("table", 3, 4 << 20), W.gen("records", 3, 4 << 20)]
    return xs


def test_p2_section3_forms(comp, oracle):
    xs = form_inputs()
    frames, st, _ = comp.CompressBatch(xs, gpu.PROFILE_ANS_DIST)
    assert all(s == 0 for s in st)
    for a, fr in zip(xs, frames):
        _check(oracle, a, fr)
    forms = {section3_form(fr) for fr in frames}
    assert {"empty", "09", "0B-M12", "0A-M12", "0A-AD", "06-AD"} <= forms, forms


def _uneven(count: int, seed: int) -> list[np.ndarray]:
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(1), np.log(2 << 20), count))).astype(int)
    sizes[:4] = [0, 1, 65536, 65537]
    return [W.mixture(seed + i, int(n))[0] for i, n in enumerate(sizes)]


def test_p2_device_batch(comp, oracle):
    from przm_b200 import devmem
    xs = _uneven(30, 2718)
    sizes = [len(x) for x in xs]
    want = [oracle.compress_p2(x) for x in xs]
    b = gpu.DeviceBatch(comp, sizes, gpu.PROFILE_ANS_DIST)
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


def test_p2_serving(comp, oracle):
    xs = _uneven(12, 99)
    srv = gpu.Server(comp, gpu.PROFILE_ANS_DIST, mem_budget=16 << 30, max_inflight=2)
    try:
        ids = [srv.submit(x) for x in xs]
        got = [srv.poll(r, 2 * len(x) + 4096)[0] for r, x in zip(ids, xs)]
    finally:
        srv.close()
    for a, fr in zip(xs, got):
        _check(oracle, a, fr)
