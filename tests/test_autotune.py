"""CPU checks of the launch-geometry tuning: size classes, the autotuner's
choice (fastest candidate among those whose frames match the per-stage
kernel path), the committed table's shape, and the representative batches."""
from __future__ import annotations

import json
import os

import numpy as np

from przm_b200 import autotune as A
from przm_b200 import gpu


def test_size_classes():
    assert [gpu.SizeClass(x) for x in (0, 1, 65536, 65537, 768 << 10, (768 << 10) + 1, 2 << 20, (2 << 20) + 1)] == \
        [0, 0, 0, 1, 1, 2, 2, 3]


def test_choose_fastest_with_identical_frames():
    rows = [{"candidate": (0, 2, 2048), "ms": 10.0, "digest": "a"},
            {"candidate": (1, 2, 1024), "ms": 7.0, "digest": "b"},   # wrong bytes: never chosen
            {"candidate": (1, 3, 2048), "ms": 8.0, "digest": "a"},
            {"candidate": (1, 2, 4096), "ms": 8.0, "digest": "a"}]
    best = A.choose({1: rows})
    assert best[1]["candidate"] == (1, 3, 2048)
    t = A.table(best, {1: rows}, "B200")
    assert t["classes"]["1"] == {"front": 1, "ctas_per_sm": 3, "verify_chunk": 2048, "ms": 8.0}
    assert len(t["measured"]["1"]) == 4


def test_class_batches_fall_in_their_class():
    for cls in range(4):
        sizes = A.class_sizes(cls, 7)
        assert gpu.SizeClass(int(sizes.mean())) == cls


def test_committed_table_is_valid():
    if not os.path.exists(A.TUNING_PATH):
        return
    t = json.load(open(A.TUNING_PATH))
    assert set(t["classes"]) <= {"0", "1", "2", "3"}
    for v in t["classes"].values():
        assert v["front"] in (0, 1) and 1 <= v["ctas_per_sm"] <= 3
        assert v["verify_chunk"] % 256 == 0 and 256 <= v["verify_chunk"] <= 65536
    for cls, rows in t["measured"].items():
        # the chosen geometry is one of the measured candidates
        chosen = t["classes"][cls]
        assert any((r["front"], r["ctas_per_sm"], r["verify_chunk"], r["ms"]) ==
                   (chosen["front"], chosen["ctas_per_sm"], chosen["verify_chunk"], chosen["ms"]) for r in rows)
