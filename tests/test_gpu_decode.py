"""GPU decoder (przmg_decompress, przmg_decompress_batch_device,
przmg_batch_verify) against the reference decoder (src/przm_dec.c, built
from the reference's sources): frames of every profile (P0-P3, written by
the oracle) decode to their inputs; the batch pipeline's frames of every
profile verify on the device; truncated and bit-flipped frames fail where
the reference decoder fails and decode to its bytes where it succeeds."""
from __future__ import annotations

import numpy as np
import pytest

from przm_b200 import gpu
from przm_b200 import workloads as W
from tests import inputs as I

pytestmark = pytest.mark.gpu

CASES = I.parity_cases(1 << 20)[::2]


def _ids(cases):
    return [c[0] for c in cases]


def _frame(oracle, profile, a) -> bytes:
    return (oracle.compress_p0, oracle.compress_p1, oracle.compress_p2, oracle.compress_p3)[profile](a)


def _p0_misread(oracle, a) -> bool:
    """A P0 frame (CompressD2D) stores raw literals without the decodability
    guard of the entropy-coded profiles: literals whose first eight bytes
    look like a container or nibble planes are misread by the reference
    decoder too (reference behaviour); the device decoder answers
    PRZMG_ERR_UNSUPPORTED_MODE for the nibble-plane form."""
    return oracle.raw_literals_misparse(oracle.tokenize(a)[2])


@pytest.mark.parametrize("profile", [0, 1, 2, 3])
@pytest.mark.parametrize("name,a", CASES, ids=_ids(CASES))
def test_decode_oracle_frames(comp, oracle, name, a, profile):
    fr = _frame(oracle, profile, a)
    if profile == 0 and len(a) and _p0_misread(oracle, a):
        try:
            got = comp.Decompress(fr)
        except gpu.GPUError:
            return
        ok, ref = _ref(oracle, fr)  # decoded anyway: as the reference decoder reads it
        assert ok and got == ref
        return
    assert comp.Decompress(fr) == bytes(a)


def _uneven(count: int, seed: int) -> list[np.ndarray]:
    rng = np.random.default_rng(seed)
    sizes = np.floor(np.exp(rng.uniform(np.log(1), np.log(2 << 20), count))).astype(int)
    sizes[:4] = [0, 1, 65536, 65537]
    return [W.mixture(seed + i, int(n))[0] for i, n in enumerate(sizes)]


@pytest.mark.parametrize("profile", [0, 1, 2, 3])
def test_batch_frames_verify_on_device(comp, oracle, profile):
    from przm_b200 import devmem
    xs = _uneven(40, 4242) + [I.ident_text(100_000, 3), I.tagged_numbers(50_000, 3), np.zeros(70_000, np.uint8)]
    want_bad = sum(1 for x in xs if len(x) and _p0_misread(oracle, x)) if profile == 0 else 0
    sizes = [len(x) for x in xs]
    b = gpu.DeviceBatch(comp, sizes, profile)
    try:
        host = np.zeros(int(b.in_offs[-1]) + max(sizes[-1], 1) + 64, np.uint8)
        for x, o in zip(xs, b.in_offs):
            host[int(o):int(o) + len(x)] = x
        devmem.upload_to(b.d_in, host)
        b.enqueue()
        assert b.verify() == want_bad
    finally:
        b.close()


def _device_decode(comp, frames, caps):
    """All frames in one device call: (statuses, decoded bytes)."""
    from przm_b200 import devmem
    so = np.zeros(len(frames), np.uint64)
    do = np.zeros(len(frames), np.uint64)
    o = d = 0
    for i, (f, c) in enumerate(zip(frames, caps)):
        so[i], do[i] = o, d
        o += (len(f) + 15) // 16 * 16 + 16
        d += (c + 15) // 16 * 16 + 16
    src = np.zeros(o + 64, np.uint8)
    for f, x in zip(frames, so):
        src[int(x):int(x) + len(f)] = np.frombuffer(f, np.uint8)
    b_src, b_dst = devmem.alloc(len(src)), devmem.alloc(d + 64)
    try:
        devmem.upload_to(b_src.ptr, src)
        st, ln = comp.DecompressBatchDevice(b_src.ptr, so, [len(f) for f in frames], b_dst.ptr, do, caps)
        outs = [devmem.download(b_dst.ptr + int(x), int(n)) for x, n in zip(do, ln)]
    finally:
        b_src.free()
        b_dst.free()
    return st, outs


def test_batch_device_decode(comp, oracle):
    xs = [W.gen(k, 9, n) for k in ("markov", "table", "records") for n in (5000, 300_000)]
    frames = [_frame(oracle, p, a) for p in range(4) for a in xs]
    want = [bytes(a) for p in range(4) for a in xs]
    st, outs = _device_decode(comp, frames, [max(len(w), 1) for w in want])
    assert list(st) == [0] * len(frames)
    assert outs == want


def _ref(oracle, fr: bytes):
    usize = int.from_bytes(fr[5:8], "little") if len(fr) >= 8 else 0
    try:
        return True, oracle.ref_decompress(fr, usize)
    except ValueError:
        return False, None


def test_corrupted_frames_fail_like_the_reference(comp, oracle):
    if not oracle.ref_decoder_available():
        pytest.skip("reference decoder not built")
    rng = np.random.default_rng(31)
    base = []
    for p in (1, 2, 3):
        for a in (W.gen("markov", 5, 20_000), W.gen("records", 6, 60_000), I.ident_text(30_000, 4)):
            base.append(_frame(oracle, p, a))
    variants = []
    for fr in base:
        variants += [fr[:len(fr) - 1], fr[:len(fr) // 2], fr[:8], b"PRZN" + fr[4:]]
        for _ in range(40):
            b = bytearray(fr)
            i = int(rng.integers(8, len(b)))
            b[i] ^= 1 << int(rng.integers(0, 8))
            variants.append(bytes(b))
    caps = [max(int.from_bytes(v[5:8], "little"), 1) for v in variants]
    st, outs = _device_decode(comp, variants, caps)
    agree = 0
    for v, s, o in zip(variants, st, outs):
        ok, ref = _ref(oracle, v)
        if v[:4] != b"PRZM":
            assert s == -2
            continue
        assert (s == 0) == ok, (s, ok)
        if ok:
            assert o == ref
        agree += 1
    assert agree > 300


def test_batch_device_decode_many_frames(comp, oracle):
    """More than 512 frames in one call: the adaptive bodies decode eight per
    warp (the other tests' calls decode them one per warp).  640 frames of
    every entropy-coded profile, sizes from 1 byte to 40 000, several
    workloads, each equal to its input."""
    kinds = ("markov", "table", "records", "uniform")
    xs = [W.gen(kinds[i % 4], 300 + i, 1 + (i * 7919) % 40_000) for i in range(640)]
    frames = [_frame(oracle, 1 + i % 3, a) for i, a in enumerate(xs)]
    want = [bytes(a) for a in xs]
    st, outs = _device_decode(comp, frames, [max(len(w), 1) for w in want])
    assert list(st) == [0] * len(frames)
    bad = [i for i, (o, w) in enumerate(zip(outs, want)) if o != w]
    assert not bad, f"{len(bad)} frames differ, first {bad[0]}"
