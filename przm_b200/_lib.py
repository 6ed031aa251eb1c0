"""Loader and ctypes signatures of libprzmgpu.so (include/przmgpu.h).

The library is built in place (przm_b200/build.py); importing this module
never compiles anything.  A missing library raises instead of falling back.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libprzmgpu.so")
GEN_PATH = os.path.join(HERE, "libprzm_gen.so")

vp = C.c_void_p
i32 = C.c_int32
u32 = C.c_uint32
u64 = C.c_uint64
i64 = C.c_int64
dbl = C.c_double


class Profile(C.Structure):
    _fields_ = [("ingress_dma_bytes", u64), ("ingress_dma_time_ms", dbl), ("ingress_dma_bandwidth_gbps", dbl),
                ("kernel_time_ms", dbl), ("internal_vram_bandwidth_gbps", dbl), ("egress_dma_bytes", u64),
                ("egress_dma_time_ms", dbl), ("egress_dma_bandwidth_gbps", dbl), ("total_round_trip_ms", dbl),
                ("end_to_end_bandwidth_gbps", dbl), ("pcie_overhead_percent", dbl), ("device_name", C.c_char * 128),
                ("sm_count", i32), ("pipelined_chunks", i32), ("total_vram_bytes", u64)]


class TokProfile(C.Structure):
    _fields_ = [("kernel_time_ms", dbl), ("pass1_ms", dbl), ("pass2_ms", dbl), ("pass3_ms", dbl),
                ("total_round_trip_ms", dbl), ("throughput_gbps", dbl), ("cmd_bytes", i64), ("offset_bytes", i64),
                ("literal_bytes", i64), ("num_chunks", i64)]


class DevStreams(C.Structure):
    _fields_ = [("d_final_cmds", u64), ("d_final_offs", u64), ("d_final_lits", u64), ("d_totals", u64),
                ("cmd_len", u32), ("off_len", u32), ("lit_len", u32), ("num_chunks", u32), ("stream", u64)]


class Job(C.Structure):
    _fields_ = [("src", vp), ("n", u64), ("dst", vp), ("cap", u64), ("out_len", u64), ("status", i32),
                ("reserved", i32)]


NOALLOC_MAX_N = 1 << 20  # PRZMG_NOALLOC_MAX_N

MATCH_DTYPE = np.dtype([("position", "<u4"), ("offset", "<u4"), ("length", "<u2"), ("literal", "u1"),
                        ("reserved", "u1")])

# name -> (restype, argtypes); the same list drives the export check in tests
SIGNATURES: dict[str, tuple] = {
    "przmg_is_available": (i32, []),
    "przmg_init": (i32, [i32, vp]),
    "przmg_get_global": (i32, [vp]),
    "przmg_reset_global_for_test": (None, []),
    "przmg_close": (i32, [vp]),
    "przmg_set_mock_unavailable": (None, [i32]),
    "przmg_set_mock_match_error": (None, [i32]),
    "przmg_device_info": (i32, [vp, vp, vp, C.c_char_p, C.c_size_t, vp, vp]),
    "przmg_last_error": (C.c_char_p, []),
    "przmg_match_lz77": (i32, [vp, vp, u64, vp, u64, vp, vp]),
    "przmg_match_table": (i32, [vp, vp, u64, vp]),
    "przmg_match_lz77_streaming": (i32, [vp, vp, u64, i64, vp, u64, vp, vp]),
    "przmg_tokenize": (i32, [vp, vp, u64, vp, u64, vp, u64, vp, u64, vp, vp]),
    "przmg_tokenize_device": (i32, [vp, vp, u64, vp, vp]),
    "przmg_tokenize_device_only": (i32, [vp, u64, vp, u64, vp, u64, vp, u64, vp, vp]),
    "przmg_tokenize_pointers_device_only": (i32, [vp, u64, vp, vp]),
    "przmg_download_device_bytes": (i32, [vp, u64, u64, vp]),
    "przmg_frame_bound": (u64, [u64]),
    "przmg_encode_d2d": (i32, [vp, vp, u32, i32, vp, u64, vp, vp]),
    "przmg_compress_d2d": (i32, [vp, vp, u64, vp, u64, vp, vp]),
    "przmg_compress": (i32, [vp, vp, u64, i32, vp, u64, vp, vp]),
    "przmg_compress_batch": (i32, [vp, vp, u64, i32, i32, vp]),
    "przmg_batch_create": (i32, [vp, vp, u64, i32, vp]),
    "przmg_batch_inputs": (i32, [vp, vp, vp]),
    "przmg_batch_outputs": (i32, [vp, vp, vp]),
    "przmg_batch_enqueue": (i32, [vp, u64, i32]),
    "przmg_batch_sizes": (i32, [vp, vp]),
    "przmg_batch_launch_count": (i32, [vp]),
    "przmg_batch_enqueue_plain": (i32, [vp, u64, vp]),
    "przmg_size_class": (i32, [u64]),
    "przmg_set_tuning": (i32, [vp, i32, i32, i32, i32]),
    "przmg_get_tuning": (i32, [vp, i32, vp, vp, vp]),
    "przmg_batch_info": (i32, [vp, vp]),
    "przmg_set_front_wait": (i32, [vp, u64, i32]),
    "przmg_batch_destroy": (i32, [vp]),
    "przmg_batch_upload": (i32, [vp, vp, u64]),
    "przmg_batch_download": (i32, [vp, vp, u64, vp, vp, u64]),
    "przmg_batch_stage_times": (i32, [vp, vp, i32, vp]),
    "przmg_stage_name": (C.c_char_p, [i32]),
    "przmg_batch_stats": (i32, [vp, vp]),
    "przmg_batch_stream_lens": (i32, [vp, vp, u64]),
    "przmg_compress_packed": (i32, [vp, vp, vp, u64, i32, vp, u64, vp, vp]),
    "przmg_compute_histogram_gpu": (i32, [vp, u64, u64, u64, vp, vp, vp]),
    "przmg_compute_histogram_host": (i32, [vp, vp, u64, vp, vp]),
    "przmg_pack_stream_flat_gpu": (i32, [vp, u64, u64, u64, u64, vp, vp, vp]),
    "przmg_pack_stream_flat_host": (i32, [vp, vp, u64, vp, u64, vp, vp]),
    "przmg_vans_encode4x_gpu": (i32, [vp, u64, u64, u64, vp, vp, vp, u32, u64, vp, vp, vp]),
    "przmg_vans_encode4x_host": (i32, [vp, vp, u64, vp, u64, vp, vp]),
    "przmg_vans_encode_batch": (i32, [vp, u64, vp, vp, u64, i32, u64, vp, vp, u64]),
    "przmg_package_offsets_batch": (i32, [vp, u64, vp, vp, u64, u64, vp, vp, vp, u64]),
    "przmg_package_literals_batch": (i32, [vp, u64, vp, vp, u64, u64, vp, vp, vp, vp, u64]),
    "przmg_vans_encode_noalloc": (i32, [u64, u32, i32, u64, u64, u64, u64]),
    "przmg_serve_create": (i32, [vp, i32, u64, i32, u64, vp]),
    "przmg_serve_submit": (i32, [vp, vp, u64, vp]),
    "przmg_serve_poll": (i32, [vp, u64, i32, vp, u64, vp, vp, vp]),
    "przmg_serve_stats": (i32, [vp, vp]),
    "przmg_serve_timing": (i32, [vp, vp]),
    "przmg_serve_destroy": (i32, [vp]),
    "przmg_normalize_freq": (None, [vp, u32, vp]),
    "przmg_normalize_frequencies": (None, [vp, vp]),
    "przmg_build_cdf": (None, [vp, vp]),
    "przmg_serialize_matrix": (u32, [vp, vp]),
    "przmg_benchmark_vram_bandwidth": (i32, [vp, i32, i32, vp]),
    "przmg_benchmark_d2d_entropy": (i32, [vp, i32, i32, vp]),
    "przmg_benchmark_entropy_vram": (i32, [vp, i32, i32, vp]),
    "przmg_alloc_pinned_host": (i32, [u64, vp]),
    "przmg_free_pinned_host": (i32, [vp]),
    "przmg_pinned_pool_create": (i32, [u64, i32, vp]),
    "przmg_pinned_pool_get": (i32, [vp, vp]),
    "przmg_pinned_pool_put": (None, [vp, vp, u64]),
    "przmg_pinned_pool_close": (i32, [vp]),
    "przmg_pinned_pool_buf_size": (u64, [vp]),
    "przmg_pinned_pool_pooled": (u64, [vp]),
    "przmg_get_pinned": (i32, [vp, u64, vp, vp]),
    "przmg_decompress": (i32, [vp, vp, u64, vp, u64, vp]),
    "przmg_decompress_batch_device": (i32, [vp, u64, vp, vp, u64, u64, vp, vp, vp, vp, u64]),
    "przmg_batch_verify": (i32, [vp, vp]),
}

_LIB: C.CDLL | None = None


def lib() -> C.CDLL:
    """The loaded libprzmgpu.so; raises if it was not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python przm_b200/build.py` "
                              "(the CUDA path has no fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


_GEN: C.CDLL | None = None


def gen() -> C.CDLL:
    global _GEN
    if _GEN is None:
        if not os.path.exists(GEN_PATH):
            raise ImportError(f"{GEN_PATH} is missing: build it with `python przm_b200/build.py`")
        G = C.CDLL(GEN_PATH)
        for f in ("przm_gen_markov", "przm_gen_table", "przm_gen_records", "przm_gen_uniform"):
            getattr(G, f).argtypes = [u64, vp, u64]
            getattr(G, f).restype = None
        G.przm_gen_zipf.argtypes = [u64, dbl, vp, u64]
        G.przm_gen_zipf.restype = None
        G.przm_gen_mixture.argtypes = [u64, vp, u64]
        G.przm_gen_mixture.restype = i32
        _GEN = G
    return _GEN
