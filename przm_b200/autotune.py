"""Autotuner of the launch geometry per size class.

For each size class of batches (mean input size: <= 64 KiB, <= 768 KiB,
<= 2 MiB, above) it builds a seeded batch of that class from the workload
mixture, runs the whole pipeline under every candidate geometry -- one kernel
per front-end stage, or the persistent front end with 1-3 resident blocks
per SM and 1024-4096 radix candidates per verify item -- and keeps the
fastest.  Every candidate must give byte-identical frames (checked: frame
sizes and a digest of all frames), since the geometry never changes an
output byte.  The result goes to przm_b200/tuning.json, which
GPUCompressor applies at start-up.

    python -m przm_b200.autotune            # all classes, writes tuning.json
    python -m przm_b200.autotune --dry-run  # measure and print only
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
TUNING_PATH = os.path.join(HERE, "tuning.json")

# (front, ctas_per_sm, verify_chunk); the first is the per-stage kernel path
CANDIDATES = [(0, 2, 2048)] + [(1, c, v) for c in (2, 3) for v in (1024, 2048, 4096)]


def class_sizes(cls: int, seed: int) -> np.ndarray:
    """Input sizes of the representative batch of a size class."""
    rng = np.random.default_rng(seed + cls)
    if cls == 0:   # many small inputs (the serving median is 64 KiB)
        return np.floor(np.exp(rng.uniform(np.log(1 << 10), np.log(64 << 10), 4096))).astype(np.int64)
    if cls == 1:   # the uneven batch: log-uniform in [1 KiB, 4 MiB]
        return np.floor(np.exp(rng.uniform(np.log(1 << 10), np.log(4 << 20), 4096))).astype(np.int64)
    if cls == 2:   # 1 MiB frames
        return np.full(256, 1 << 20, np.int64)
    return np.full(32, 4 << 20, np.int64)  # large frames


def choose(results: dict) -> dict:
    """results: {class: [{"candidate": (front, ctas, chunk), "ms": t, "digest": d}, ...]}
    -> {class: best entry}.  Candidates whose frames differ from the first
    candidate's are rejected (never chosen); ties keep the earlier one."""
    best = {}
    for cls, rows in results.items():
        ref = rows[0]["digest"]
        ok = [r for r in rows if r["digest"] == ref]
        best[cls] = min(ok, key=lambda r: r["ms"])
    return best


def table(best: dict, results: dict, device: str) -> dict:
    return {
        "device": device,
        "note": "launch geometry per size class; written by przm_b200/autotune.py",
        "classes": {str(k): {"front": v["candidate"][0], "ctas_per_sm": v["candidate"][1],
                             "verify_chunk": v["candidate"][2], "ms": round(v["ms"], 3)} for k, v in best.items()},
        "measured": {str(k): [{"front": r["candidate"][0], "ctas_per_sm": r["candidate"][1],
                               "verify_chunk": r["candidate"][2], "ms": round(r["ms"], 3)} for r in rows]
                     for k, rows in results.items()},
    }


def measure(comp, sizes: np.ndarray, seed: int, reps: int = 5) -> list[dict]:
    import torch
    from . import devmem, gpu
    from . import workloads as W
    xs = [W.mixture(seed + 104729 * i, int(n))[0] for i, n in enumerate(sizes)]
    host = np.concatenate(xs)
    rows = []
    saved = [comp.GetTuning(k) for k in range(4)]
    try:
        for cand in CANDIDATES:
            for k in range(4):
                comp.SetTuning(k, *cand)
            b = gpu.DeviceBatch(comp, [len(x) for x in xs], gpu.PROFILE_ANS)
            try:
                b.upload(host)
                st = torch.cuda.Stream()
                for _ in range(2):
                    b.enqueue(st.cuda_stream, graph=True)
                torch.cuda.synchronize()
                times = []
                for _ in range(reps):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(st)
                    b.enqueue(st.cuda_stream, graph=True)
                    e1.record(st)
                    e1.synchronize()
                    times.append(e0.elapsed_time(e1))
                fs = b.frame_sizes()
                h = hashlib.sha256(fs.tobytes())
                region = devmem.download(b.d_out, int(b.out_offs[-1]) + int(fs[-1]))
                for o, s in zip(b.out_offs, fs):  # the frames only (the gaps between them are not written)
                    h.update(region[int(o):int(o) + int(s)])
                rows.append({"candidate": cand, "ms": sorted(times)[len(times) // 2], "digest": h.hexdigest(),
                             "front_used": b.info()["front"]})
            finally:
                b.close()
    finally:
        for k, t in enumerate(saved):
            comp.SetTuning(k, t["front"], t["ctas_per_sm"], t["verify_chunk"])
    return rows


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--dry-run", action="store_true")
    ap.add_argument("--classes", default="0,1,2,3")
    ap.add_argument("--seed", type=int, default=0x50525A4D + 5)
    ap.add_argument("--out", default=TUNING_PATH, help="where the table goes (default: przm_b200/tuning.json)")
    args = ap.parse_args()
    from . import gpu
    comp = gpu.GPUCompressor(0)
    results = {}
    for cls in (int(c) for c in args.classes.split(",")):
        t0 = time.time()
        results[cls] = measure(comp, class_sizes(cls, args.seed), args.seed + 1000 * cls)
        print(json.dumps({"class": cls, "rows": [{k: (v if k != "digest" else v[:12]) for k, v in r.items()}
                                                  for r in results[cls]], "s": round(time.time() - t0, 1)}), flush=True)
    best = choose(results)
    out = table(best, results, comp.DeviceName)
    print(json.dumps(out["classes"]), flush=True)
    if not args.dry_run:
        with open(args.out, "w") as f:
            json.dump(out, f, indent=1)
            f.write("\n")


if __name__ == "__main__":
    main()
