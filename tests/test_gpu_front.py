"""GPU: the persistent front end (one launch running the match finders,
tokenizer and gather of a whole batch from a device work queue) gives the
same frames as one kernel per stage, for every tuning it can be given; and
its bounded waits fail cleanly: a wait that nothing ends makes the call
return PRZMG_ERR_DEVICE without hanging, and the context keeps working."""
from __future__ import annotations

import numpy as np
import pytest

from przm_b200 import devmem, gpu
from przm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _inputs(kind: str, seed: int) -> list[np.ndarray]:
    rng = np.random.default_rng(seed)
    if kind == "small":
        sizes = np.floor(np.exp(rng.uniform(np.log(1), np.log(64 << 10), 60))).astype(int)
        sizes[:3] = [0, 1, 65536]
    elif kind == "uneven":
        sizes = np.floor(np.exp(rng.uniform(np.log(1 << 10), np.log(3 << 20), 40))).astype(int)
        sizes[:4] = [0, 7, 65536, 65537]
    else:  # "large": 1 MiB frames and one 4 MiB frame
        sizes = np.array([1 << 20] * 6 + [4 << 20])
    return [W.mixture(seed + 17 * i, int(n))[0] for i, n in enumerate(sizes)]


def _run(comp, xs, profile=gpu.PROFILE_ANS, graph=True):
    sizes = [len(x) for x in xs]
    b = gpu.DeviceBatch(comp, sizes, profile)
    try:
        host = np.zeros(int(b.in_offs[-1]) + max(sizes[-1], 1) + 64, np.uint8)
        for x, o in zip(xs, b.in_offs):
            host[int(o):int(o) + len(x)] = x
        devmem.upload_to(b.d_in, host)
        b.enqueue(graph=graph)
        fs = b.frame_sizes().copy()
        frames = [devmem.download(b.d_out + int(o), int(s)) for o, s in zip(b.out_offs, fs)]
        return frames, b.info()
    finally:
        b.close()


@pytest.fixture
def tuning(comp):
    saved = [comp.GetTuning(k) for k in range(4)]
    yield
    for k, t in enumerate(saved):
        comp.SetTuning(k, t["front"], t["ctas_per_sm"], t["verify_chunk"])


@pytest.mark.parametrize("kind", ["small", "uneven", "large"])
@pytest.mark.parametrize("ctas,chunk", [(2, 2048), (3, 256), (1, 4096)])
def test_front_equals_stage_kernels(comp, oracle, tuning, kind, ctas, chunk):
    xs = _inputs(kind, {"small": 11, "uneven": 12, "large": 13}[kind])
    for k in range(4):
        comp.SetTuning(k, 0, 2, 2048)
    want, info0 = _run(comp, xs)
    assert info0["front"] == 0
    for k in range(4):
        comp.SetTuning(k, 1, ctas, chunk)
    for graph in (False, True):
        got, info1 = _run(comp, xs, graph=graph)
        assert info1["front"] == 1 and info1["ctas_per_sm"] == ctas and info1["verify_chunk"] == chunk
        assert got == want
    for x, f in list(zip(xs, want))[:6]:
        assert f == oracle.compress_p1(x)


def test_front_d2d_profile_and_one_input_calls(comp, oracle, tuning):
    for k in range(4):
        comp.SetTuning(k, 1, 2, 2048)
    xs = _inputs("uneven", 21)[:12]
    got, info = _run(comp, xs, profile=gpu.PROFILE_D2D)
    assert info["front"] == 1
    assert got == [oracle.compress_p0(x) for x in xs]
    a = W.gen("markov", 22, 300_000)
    fr, _ = comp.Compress(a, gpu.PROFILE_ANS)  # the one-input path lays out a one-input batch
    assert fr == oracle.compress_p1(a)
    cmd, off, lit, _ = comp.Tokenize(a)
    assert (cmd, off, lit) == tuple(oracle.tokenize(a))


def test_front_wait_limit_fails_cleanly(comp, oracle, tuning):
    for k in range(4):
        comp.SetTuning(k, 1, 2, 2048)
    xs = _inputs("uneven", 31)[:10]
    comp.SetFrontWait(2_000_000, addUnreachableWait=True)  # 2 ms, and one wait nothing ends
    try:
        with pytest.raises(gpu.GPUError) as e:
            _run(comp, xs)
        assert e.value.code == -13 and "wait" in str(e.value)
    finally:
        comp.SetFrontWait(1_000_000_000, addUnreachableWait=False)
    got, info = _run(comp, xs)  # the context still works
    assert info["front"] == 1
    assert got == [oracle.compress_p1(x) for x in xs]
