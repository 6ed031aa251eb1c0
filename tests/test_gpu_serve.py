"""Serving engine (przmg_serve_*): continuous batching with several batches
in flight.  Each frame must be the same alone and in the mix (here: byte for
byte, the tolerance of an integer path), under concurrent submitters and an
open-loop Poisson arrival process."""
from __future__ import annotations

import threading

import numpy as np
import pytest

from przm_b200 import gpu, serving
from przm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _mix(count: int, seed: int = 11):
    sizes = np.minimum(W.config4_sizes(count), 3 << 20)  # keep the suite fast
    return [W.mixture(seed + i, int(s))[0] for i, s in enumerate(sizes)]


@pytest.mark.parametrize("profile", [gpu.PROFILE_ANS, gpu.PROFILE_D2D])
def test_same_alone_and_in_the_mix(comp, oracle, profile):
    inputs = _mix(60) + [np.zeros(0, np.uint8), W.gen("uniform", 3, 1), W.gen("records", 4, (1 << 20) + 5)]
    alone = [comp.Compress(a, profile)[0] for a in inputs]
    srv = gpu.Server(comp, profile, mem_budget=48 << 30, max_inflight=3)
    try:
        res = serving.run_open_loop(srv, inputs, rate_hz=2000.0)
        st = srv.stats()
    finally:
        srv.close()
    for a, f, g in zip(inputs, res["frames"], alone):
        assert f == g
    for a, f in list(zip(inputs, res["frames"]))[:6]:  # and against the oracle / reference decoder
        want = oracle.compress_p1(a) if profile == gpu.PROFILE_ANS else oracle.compress_p0(a)
        assert f == want
        if oracle.ref_decoder_available() and len(a):
            assert oracle.ref_decompress(f, len(a)) == a.tobytes()
    assert st["done"] == len(inputs) and st["pending"] == 0 and st["live"] == 0
    assert st["batches"] >= 2


def test_concurrent_submitters_and_saturation(comp):
    inputs = _mix(90, seed=500)
    alone = [comp.Compress(a)[0] for a in inputs]
    srv = gpu.Server(comp, gpu.PROFILE_ANS, mem_budget=48 << 30, max_inflight=4)
    out = [None] * len(inputs)
    try:
        def worker(k):
            for i in range(k, len(inputs), 3):
                rid = srv.submit(inputs[i])
                out[i] = srv.poll(rid, 2 * len(inputs[i]) + 4096)[0]
        th = [threading.Thread(target=worker, args=(k,)) for k in range(3)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        res = serving.run_open_loop(srv, inputs, rate_hz=None)  # everything at once
        st = srv.stats()
    finally:
        srv.close()
    assert out == alone
    assert res["frames"] == alone
    assert st["max_batch"] > 1  # requests were batched


def test_errors(comp):
    srv = gpu.Server(comp, gpu.PROFILE_ANS, mem_budget=48 << 30, max_inflight=2)
    try:
        with pytest.raises(gpu.GPUError) as e:
            srv.submit(np.zeros(16 << 20, np.uint8))
        assert e.value.code == -5
        with pytest.raises(gpu.GPUError) as e:
            srv.poll(123456, 10)
        assert e.value.code == -14
        a = W.gen("markov", 9, 100_000)
        rid = srv.submit(a)
        with pytest.raises(gpu.GPUError) as e:
            srv.poll(rid, 10)  # too small: the request stays pollable
        assert e.value.code == -4
        f = srv.poll(rid, 2 * len(a) + 4096)[0]
        assert f == comp.Compress(a)[0]
    finally:
        srv.close()
    with pytest.raises(gpu.GPUError):
        gpu.Server(comp, gpu.PROFILE_ANS, mem_budget=1 << 20, max_inflight=2)
