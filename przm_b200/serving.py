"""Open-loop load generation for the serving engine (gpu.Server): requests
arrive as a Poisson process and are submitted at their arrival times; the
frames are collected afterwards.  Latencies come from the engine's own
submit / complete stamps (steady clock, frame on the host), so collecting
late does not change them, and one thread keeps the submission schedule
free of interpreter-lock contention."""
from __future__ import annotations

import time

import numpy as np


def run_open_loop(server, inputs, rate_hz: float | None, seed: int = 7, cap_of=None) -> dict:
    """rate_hz None submits everything at once (saturation).  Returns the
    frames (in input order), per-request latencies in ms, and throughput."""
    n = len(inputs)
    rng = np.random.default_rng(seed)
    gaps = np.zeros(n) if rate_hz is None else rng.exponential(1.0 / rate_hz, n)
    arrive = np.cumsum(gaps)
    ids = []
    t0 = time.perf_counter()
    for i in range(n):
        d = t0 + arrive[i] - time.perf_counter()
        if d > 0:
            time.sleep(d)
        ids.append(server.submit(inputs[i]))
    frames = [None] * n
    t_sub = np.zeros(n, np.int64)
    t_done = np.zeros(n, np.int64)
    for i in range(n):
        cap = cap_of(len(inputs[i])) if cap_of else 2 * len(inputs[i]) + 4096
        frames[i], t_sub[i], t_done[i] = server.poll(ids[i], cap, wait=True)
    lat = (t_done - t_sub) / 1e6
    span = (t_done.max() - t_sub.min()) / 1e9
    nbytes = int(sum(len(a) for a in inputs))
    offered = None if rate_hz is None else nbytes / max(arrive[-1], 1e-9) / 1e9
    return {"frames": frames, "lat_ms": lat, "gbps": nbytes / span / 1e9, "offered_gbps": offered,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "requests": n, "bytes": nbytes, "span_s": span}
