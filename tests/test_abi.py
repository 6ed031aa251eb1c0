"""CPU checks of the C ABI: the library loads, exports every function that
include/przmgpu.h declares, and its host-only helpers agree with the oracle.
No device is touched."""
from __future__ import annotations

import os
import re

import numpy as np
import pytest

from przm_b200 import _lib, gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions() -> list[str]:
    txt = open(os.path.join(ROOT, "include", "przmgpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(przmg_[a-z0-9_]+)\s*\(", txt)))


def test_header_and_bindings_agree():
    assert header_functions() == sorted(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    for name in header_functions():
        assert hasattr(L, name), name


def test_no_device_here_reports_unavailable():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    assert not gpu.IsAvailable()
    with pytest.raises(gpu.GPUError) as e:
        gpu.GPUCompressor(0)
    assert e.value.code == -11


def test_mock_unavailable_switch():
    gpu.SetMockUnavailableForTest(True)
    try:
        assert not gpu.IsAvailable()
    finally:
        gpu.SetMockUnavailableForTest(False)


def test_host_helpers_match_oracle(oracle):
    rng = np.random.default_rng(1)
    for t in range(100):
        counts = np.zeros(256, np.uint32)
        k = int(rng.integers(1, 257))
        counts[rng.choice(256, k, replace=False)] = rng.integers(1, [3, 40, 1 << 20][t % 3], k)
        f = gpu.NormalizeFreq(counts)
        assert np.array_equal(f, oracle.normalize_freq(counts))
        assert np.array_equal(gpu.NormalizeFrequencies(counts), oracle.normalize_frequencies(counts))
        assert np.array_equal(gpu.BuildCDF(f), oracle.build_cdf(f))
        assert gpu.SerializeMatrix(f) == oracle.serialize_matrix(f)


def test_pack_match_helpers():
    assert gpu.PackMatch32(4, 1) == (4 << 20) | 1
    assert gpu.PackMatch32(3, 1) == 0 and gpu.PackMatch32(9, 0) == 0
    assert gpu.UnpackMatch32(gpu.PackMatch32(4095, 1048575)) == (4095, 1048575)
    assert gpu.IsMatch32(gpu.PackMatch32(5, 5)) and not gpu.IsMatch32(0)


def test_frame_bound_covers_oracle_frames(oracle):
    from tests import inputs as I
    for name, a in I.parity_cases(200_000)[::9]:
        assert len(oracle.compress_p0(a)) <= gpu.FrameBound(len(a))
        assert len(oracle.compress_p1(a)) <= gpu.FrameBound(len(a))
