"""ctypes bindings to the test-only checkers built by oracle/Makefile.

TEST INFRASTRUCTURE ONLY: the CPU restatement (liboracle.so) and the
reference's own C99 decoder and CUDA kernels (_ref/).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may import this
module; the product package never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_DEC = None

u8p = C.POINTER(C.c_uint8)
u16p = C.POINTER(C.c_uint16)
u32p = C.POINTER(C.c_uint32)
u64p = C.POINTER(C.c_uint64)


def build() -> None:
    """Build liboracle.so (and _ref/ when a reference checkout is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib() -> C.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.or_pack_match32.restype = C.c_uint32
        L.or_pack_match32.argtypes = [C.c_uint32, C.c_uint32]
        L.or_tile_find.argtypes = [u8p, C.c_uint64, C.c_uint32, u32p]
        L.or_radix_find.argtypes = [u8p, C.c_uint64, C.c_uint32, u32p]
        L.or_match_table.argtypes = [u8p, C.c_uint64, u32p]
        L.or_match_lz77.restype = C.c_uint64
        L.or_match_lz77.argtypes = [u8p, C.c_uint64, u32p, u32p]
        L.or_match_lz77_chunked.restype = C.c_uint64
        L.or_match_lz77_chunked.argtypes = [u8p, C.c_uint64, C.c_uint64, u32p, u32p]
        L.or_streaming_chunk.restype = C.c_uint64
        L.or_streaming_chunk.argtypes = [C.c_uint64, C.c_int64]
        L.or_tokenize.argtypes = [u8p, C.c_uint64, u32p, u8p, u64p, u8p, u64p, u8p, u64p]
        L.or_tokenize_tiles.argtypes = [u8p, C.c_uint64, u32p, u32p]
        L.or_split_commands.restype = C.c_int
        L.or_split_commands.argtypes = [u8p, C.c_uint64, u8p, u64p, u8p, u64p, u8p, u64p]
        L.or_normalize_frequencies.argtypes = [u32p, u16p]
        L.or_normalize_freq.argtypes = [u32p, C.c_uint32, u16p]
        L.or_normalize_freq_tie_straddles.restype = C.c_int
        L.or_normalize_freq_tie_straddles.argtypes = [u32p, C.c_uint32]
        L.or_build_cdf.argtypes = [u16p, u16p]
        L.or_serialize_matrix.restype = C.c_uint32
        L.or_serialize_matrix.argtypes = [u16p, u8p]
        L.or_vans_encode.restype = C.c_uint64
        L.or_vans_encode.argtypes = [u8p, C.c_uint64, u16p, C.c_uint8, u8p]
        L.or_histogram.argtypes = [u8p, C.c_uint64, u32p]
        L.or_adaptive_vans.restype = C.c_uint64
        L.or_adaptive_vans.argtypes = [u8p, C.c_uint64, u8p]
        L.or_vans_encode_host.restype = C.c_uint64
        L.or_vans_encode_host.argtypes = [u8p, C.c_uint64, u8p]
        L.or_encode_meta8.restype = C.c_uint64
        L.or_encode_meta8.argtypes = [u8p, C.c_uint64, u8p]
        L.or_package_commands.restype = C.c_uint64
        L.or_package_commands.argtypes = [u8p, C.c_uint64, u8p]
        L.or_compress_p0.restype = C.c_uint64
        L.or_compress_p0.argtypes = [u8p, C.c_uint64, u8p]
        L.or_compress_p1.restype = C.c_uint64
        L.or_compress_p1.argtypes = [u8p, C.c_uint64, u8p]
        L.or_frame_bound.restype = C.c_uint64
        L.or_frame_bound.argtypes = [C.c_uint64]
        L.or_raw_literals_misparse.restype = C.c_int
        L.or_raw_literals_misparse.argtypes = [u8p, C.c_uint64]
        L.or_tokenize_input.argtypes = [u8p, C.c_uint64, u8p, u64p, u8p, u64p, u8p, u64p]
        L.or_distance_to_code.restype = C.c_uint8
        L.or_distance_to_code.argtypes = [C.c_uint32, u32p, u32p]
        L.or_dist_mode12.restype = C.c_uint64
        L.or_dist_mode12.argtypes = [u8p, C.c_uint64, u8p, C.c_uint64]
        L.or_pack_distance_prefix.restype = C.c_uint64
        L.or_pack_distance_prefix.argtypes = [u32p, C.c_uint64, u8p, C.c_uint64]
        L.or_package_offsets.restype = C.c_uint64
        L.or_package_offsets.argtypes = [u32p, C.c_uint64, u8p]
        L.or_compress_p2.restype = C.c_uint64
        L.or_compress_p2.argtypes = [u8p, C.c_uint64, u8p]
        L.or_compress_p3.restype = C.c_uint64
        L.or_compress_p3.argtypes = [u8p, C.c_uint64, u8p]
        L.or_sheaf_class.restype = C.c_uint8
        L.or_sheaf_class.argtypes = [C.c_uint8, C.c_uint8, C.c_int]
        L.or_decompose_fibers.argtypes = [u8p, C.c_uint64, C.c_int, C.POINTER(u8p), u64p]
        L.or_pack_sheaf.restype = C.c_uint64
        L.or_pack_sheaf.argtypes = [u8p, C.c_uint64, C.c_int, u8p]
        L.or_package_literals.restype = C.c_uint64
        L.or_package_literals.argtypes = [u8p, C.c_uint64, u8p, u8p]
        _LIB = L
    return _LIB


def _p(a: np.ndarray, t=u8p):
    return a.ctypes.data_as(t)


def _u8(data) -> np.ndarray:
    a = np.frombuffer(bytes(data), dtype=np.uint8) if not isinstance(data, np.ndarray) else data
    return np.ascontiguousarray(a, dtype=np.uint8)


UINT64_MAX = (1 << 64) - 1


def pack_match32(length: int, offset: int) -> int:
    return lib().or_pack_match32(length, offset)


def match_table(data) -> np.ndarray:
    a = _u8(data)
    out = np.zeros(max(len(a), 1), np.uint32)
    lib().or_match_table(_p(a), len(a), _p(out, u32p))
    return out[: len(a)]


def tile_find(data) -> np.ndarray:
    a = _u8(data)
    out = np.zeros(max(len(a), 1), np.uint32)
    lib().or_tile_find(_p(a), len(a), 1 << 20, _p(out, u32p))
    return out[: len(a)]


def radix_find(data) -> np.ndarray:
    a = _u8(data)
    out = np.zeros(max(len(a), 1), np.uint32)
    lib().or_radix_find(_p(a), len(a), 1 << 20, _p(out, u32p))
    return out[: len(a)]


def match_lz77(data, chunk: int | None = None):
    """(positions, descriptors) as MatchLZ77 returns them."""
    a = _u8(data)
    pos = np.zeros(max(len(a), 1), np.uint32)
    dsc = np.zeros(max(len(a), 1), np.uint32)
    if chunk is None:
        n = lib().or_match_lz77(_p(a), len(a), _p(pos, u32p), _p(dsc, u32p))
    else:
        n = lib().or_match_lz77_chunked(_p(a), len(a), chunk, _p(pos, u32p), _p(dsc, u32p))
    return pos[:n].copy(), dsc[:n].copy()


def streaming_chunk(n: int, chunk: int) -> int:
    return lib().or_streaming_chunk(n, chunk)


def tokenize_with(data, desc: np.ndarray):
    a = _u8(data)
    tiles = max((len(a) + 32767) // 32768, 1)
    cap = tiles * 36864 + 16
    c, o, l = np.zeros(cap, np.uint8), np.zeros(cap, np.uint8), np.zeros(cap, np.uint8)
    nc, no, nl = C.c_uint64(), C.c_uint64(), C.c_uint64()
    d = np.ascontiguousarray(desc, np.uint32)
    lib().or_tokenize(_p(a), len(a), _p(d, u32p), _p(c), C.byref(nc), _p(o), C.byref(no), _p(l), C.byref(nl))
    return bytes(c[: nc.value]), bytes(o[: no.value]), bytes(l[: nl.value])


def tokenize(data):
    """(cmd, off, lit) as Tokenize returns them."""
    return tokenize_with(data, match_table(data))


def tile_lengths(data, desc: np.ndarray) -> np.ndarray:
    a = _u8(data)
    tiles = (len(a) + 32767) // 32768
    out = np.zeros(max(3 * tiles, 1), np.uint32)
    d = np.ascontiguousarray(desc, np.uint32)
    lib().or_tokenize_tiles(_p(a), len(a), _p(d, u32p), _p(out, u32p))
    return out[: 3 * tiles].reshape(tiles, 3)


def split_commands(cmds):
    a = _u8(cmds)
    n = len(a)
    op, meta, var = (np.zeros(max(n, 1), np.uint8) for _ in range(3))
    a1, a2, a3 = C.c_uint64(), C.c_uint64(), C.c_uint64()
    r = lib().or_split_commands(_p(a), n, _p(op), C.byref(a1), _p(meta), C.byref(a2), _p(var), C.byref(a3))
    if r != 0:
        raise ValueError("malformed command stream")
    return bytes(op[: a1.value]), bytes(meta[: a2.value]), bytes(var[: a3.value])


def histogram(data) -> np.ndarray:
    a = _u8(data)
    out = np.zeros(256, np.uint32)
    lib().or_histogram(_p(a), len(a), _p(out, u32p))
    return out


def normalize_frequencies(counts) -> np.ndarray:
    c = np.ascontiguousarray(counts, np.uint32)
    out = np.zeros(256, np.uint16)
    lib().or_normalize_frequencies(_p(c, u32p), _p(out, u16p))
    return out


def normalize_freq(counts, target: int = 4096) -> np.ndarray:
    c = np.ascontiguousarray(counts, np.uint32)
    out = np.zeros(256, np.uint16)
    lib().or_normalize_freq(_p(c, u32p), target, _p(out, u16p))
    return out


def normalize_freq_tie_straddles(counts, target: int = 4096) -> bool:
    c = np.ascontiguousarray(counts, np.uint32)
    return bool(lib().or_normalize_freq_tie_straddles(_p(c, u32p), target))


def build_cdf(freq) -> np.ndarray:
    f = np.ascontiguousarray(freq, np.uint16)
    out = np.zeros(257, np.uint16)
    lib().or_build_cdf(_p(f, u16p), _p(out, u16p))
    return out


def serialize_matrix(freq) -> bytes:
    f = np.ascontiguousarray(freq, np.uint16)
    out = np.zeros(1024, np.uint8)
    n = lib().or_serialize_matrix(_p(f, u16p), _p(out))
    return bytes(out[:n])


def vans_encode(data, freq, flags: int) -> bytes:
    a = _u8(data)
    f = np.ascontiguousarray(freq, np.uint16)
    out = np.zeros(2 * len(a) + 1024, np.uint8)
    n = lib().or_vans_encode(_p(a), len(a), _p(f, u16p), flags, _p(out))
    return bytes(out[:n])


def adaptive_vans(data):
    a = _u8(data)
    out = np.zeros(2 * len(a) + 1024, np.uint8)
    n = lib().or_adaptive_vans(_p(a), len(a), _p(out))
    return None if n == UINT64_MAX else bytes(out[:n])


def vans_encode_host(data) -> bytes:
    a = _u8(data)
    out = np.zeros(2 * len(a) + 1024, np.uint8)
    n = lib().or_vans_encode_host(_p(a), len(a), _p(out))
    return bytes(out[:n])


def encode_meta8(data):
    a = _u8(data)
    out = np.zeros(2 * len(a) + 1024, np.uint8)
    n = lib().or_encode_meta8(_p(a), len(a), _p(out))
    return None if n == UINT64_MAX else bytes(out[:n])


def package_commands(cmds) -> bytes:
    a = _u8(cmds)
    out = np.zeros(len(a) + 1024, np.uint8)
    n = lib().or_package_commands(_p(a), len(a), _p(out))
    return bytes(out[:n])


def frame_bound(n: int) -> int:
    return lib().or_frame_bound(n)


def compress_p0(data) -> bytes:
    a = _u8(data)
    out = np.zeros(frame_bound(len(a)), np.uint8)
    n = lib().or_compress_p0(_p(a), len(a), _p(out))
    return bytes(out[:n])


def compress_p1(data) -> bytes:
    a = _u8(data)
    out = np.zeros(frame_bound(len(a)), np.uint8)
    n = lib().or_compress_p1(_p(a), len(a), _p(out))
    return bytes(out[:n])


def compress_p2(data) -> bytes:
    """P1 with Section 3 distance-coded (PackageOffsetsSection)."""
    a = _u8(data)
    out = np.zeros(frame_bound(len(a)), np.uint8)
    n = lib().or_compress_p2(_p(a), len(a), _p(out))
    return bytes(out[:n])


def compress_p3(data) -> bytes:
    """P2 with Section 4 as PackageLiteralsSection (V-ANS or a sheaf foliation)."""
    a = _u8(data)
    out = np.zeros(frame_bound(len(a)) + 4096, np.uint8)
    n = lib().or_compress_p3(_p(a), len(a), _p(out))
    return bytes(out[:n])


def sheaf_class(p2: int, p1: int, mode: int) -> int:
    return lib().or_sheaf_class(p2, p1, mode)


def decompose_fibers(lits, mode: int) -> list[bytes]:
    """The four fibers of a sheaf foliation (DecomposeFibers)."""
    a = _u8(lits)
    bufs = [np.zeros(max(len(a), 1), np.uint8) for _ in range(4)]
    ptrs = (u8p * 4)(*[_p(b) for b in bufs])
    l = np.zeros(4, np.uint64)
    lib().or_decompose_fibers(_p(a), len(a), mode, ptrs, _p(l, u64p))
    return [bytes(b[:int(k)]) for b, k in zip(bufs, l)]


def pack_sheaf(lits, mode: int) -> bytes:
    """PackEtaleSheaf container of the literals in one foliation mode."""
    a = _u8(lits)
    out = np.zeros(40 + 2 * len(a) + 4096, np.uint8)
    n = lib().or_pack_sheaf(_p(a), len(a), mode, _p(out))
    return bytes(out[:n])


def package_literals(lits) -> tuple[bytes, int]:
    """PackageLiteralsSection: (Section 4 bytes, flag nibble 0x80 or 0)."""
    a = _u8(lits)
    out = np.zeros(40 + 2 * len(a) + 4096, np.uint8)
    nib = C.c_uint8()
    n = lib().or_package_literals(_p(a), len(a), _p(out), C.byref(nib))
    return bytes(out[:n]), nib.value


def distance_to_code(d: int) -> tuple[int, int, int]:
    """(code, extra, extra bit count) of distance d (DistanceToCode)."""
    ex, nb = C.c_uint32(), C.c_uint32()
    c = lib().or_distance_to_code(d, C.byref(ex), C.byref(nb))
    return c, ex.value, nb.value


def dist_mode12(codes) -> bytes | None:
    """Mode 12 (0x0C) code stream of distance codes; None where the reference fails."""
    a = _u8(codes)
    out = np.zeros(4 << 20, np.uint8)
    n = lib().or_dist_mode12(_p(a), len(a), _p(out), len(out))
    return None if n == UINT64_MAX else bytes(out[:n])


def pack_distance_prefix(dists, cap: int = 2 << 20) -> bytes | None:
    """PackDistancePrefix (auto mode, V-ANS codes) into a cap-byte buffer; None on the reference's errors."""
    d = np.ascontiguousarray(np.asarray(dists, dtype=np.uint32))
    out = np.zeros(max(cap, 1), np.uint8)
    n = lib().or_pack_distance_prefix(_p(d, u32p), len(d), _p(out), cap)
    return None if n == UINT64_MAX else bytes(out[:n])


def package_offsets(dists) -> bytes:
    """PackageOffsetsSection: Section 3 bytes for these distances (b'' for none)."""
    d = np.ascontiguousarray(np.asarray(dists, dtype=np.uint32))
    out = np.zeros(5 * len(d) + 64, np.uint8)
    n = lib().or_package_offsets(_p(d, u32p), len(d), _p(out))
    return bytes(out[:n])


def raw_literals_misparse(lits) -> bool:
    a = _u8(lits)
    return bool(lib().or_raw_literals_misparse(_p(a), len(a)))


# --- the reference's own C99 decoder (oracle/_ref/libprzm_dec.so) ----------

def ref_decoder_path() -> str:
    return os.path.join(HERE, "_ref", "libprzm_dec.so")


def ref_decoder_available() -> bool:
    return os.path.exists(ref_decoder_path())


def dec() -> C.CDLL:
    global _DEC
    if _DEC is None:
        D = C.CDLL(ref_decoder_path())
        D.przm_decompress.restype = C.c_int32
        D.przm_decompress.argtypes = [u8p, C.c_size_t, u8p, C.c_size_t]
        D.przm_vans_decode_literals.restype = C.c_int32
        D.przm_vans_decode_literals.argtypes = [u8p, C.c_size_t, u8p, C.c_size_t]
        D.przm_vans_decode_meta8.restype = C.c_int32
        D.przm_vans_decode_meta8.argtypes = [u8p, C.c_size_t, u8p, C.c_size_t, C.c_size_t]
        D.przm_split_commands.restype = C.c_int32
        D.przm_split_commands.argtypes = [u8p, C.c_size_t, u8p, C.c_size_t, C.POINTER(C.c_size_t), u8p, C.c_size_t,
                                          C.POINTER(C.c_size_t), u8p, C.c_size_t, C.POINTER(C.c_size_t)]
        D.przm_distance_to_code.restype = C.c_int32
        D.przm_distance_to_code.argtypes = [C.c_uint32, u8p, u32p, u8p]
        D.przm_code_to_distance.restype = C.c_int32
        D.przm_code_to_distance.argtypes = [C.c_uint8, C.c_uint32, u32p]
        D.przm_vans_decode_dist4.restype = C.c_int32
        D.przm_vans_decode_dist4.argtypes = [u8p, C.c_size_t, u8p, C.c_size_t, C.c_size_t]
        D.przm_distance_prefix_decode.restype = C.c_int32
        D.przm_distance_prefix_decode.argtypes = [u8p, C.c_size_t, u8p, C.c_size_t, C.POINTER(C.c_size_t)]
        D.przm_context_classify.restype = C.c_uint8
        D.przm_context_classify.argtypes = [C.c_uint8, C.c_uint8]
        D.przm_context_classify_order2.restype = C.c_uint8
        D.przm_context_classify_order2.argtypes = [C.c_uint8, C.c_uint8]
        D.przm_reconstitute_fibers.restype = C.c_int32
        D.przm_reconstitute_fibers.argtypes = [u8p, C.c_size_t, u8p, u8p, u8p, u8p, C.c_size_t, C.c_size_t,
                                               C.c_size_t, C.c_size_t, C.c_uint8]
        _DEC = D
    return _DEC


def ref_decompress(frame: bytes, usize: int) -> bytes:
    f = _u8(frame)
    out = np.zeros(usize + 64, np.uint8)
    r = dec().przm_decompress(_p(f), len(f), _p(out), len(out))
    if r < 0:
        raise ValueError(f"reference decoder error {r}")
    return bytes(out[:r])


def ref_decode_vans_literals(container: bytes) -> bytes:
    """Decode a 'VA' container body (after the 8-byte header) of n symbols."""
    c = _u8(container)
    n = int.from_bytes(container[4:8], "little")
    out = np.zeros(n + 64, np.uint8)
    body = c[8:]
    r = dec().przm_vans_decode_literals(_p(body), len(body), _p(out), n)
    if r != 0:
        raise ValueError(f"reference V-ANS decode error {r}")
    return bytes(out[:n])


def ref_decode_meta8(container: bytes, n: int) -> bytes:
    c = _u8(container)
    out = np.zeros(n + 64, np.uint8)
    r = dec().przm_vans_decode_meta8(_p(c), len(c), _p(out), len(out), n)
    if r != 0:
        raise ValueError(f"reference Meta8 decode error {r}")
    return bytes(out[:n])


# --- the reference's own CUDA kernels (oracle/_ref/libprzm_ref_cuda.so) -----
# Compiled from gpu/kernel/przm_lz77.cu with the host shim ref_cuda_shim.cu
# (launch shapes of the Go bridge).  Arguments are raw device addresses; the
# callers (GPU tests) own the buffers.  Buffer contracts, from the kernels:
#   ref_histogram      d_hist 256 x u32, d_meta 4 x u32 (cleared first)
#   ref_vans_encode4x  d_temp >= 2n + 64 bytes (the serial bit stream before
#                      reversal), d_out >= 8 + mat_len + 16 + 2n + 64
#   ref_tokenize       d_matches n x u32; per 32 KiB chunk 36864 bytes of
#                      cmd/off/lit slot; d_lens 6 x chunks u32; d_totals 3 x
#                      u32; all input reads stay below the tile end.
#   cuda_lz77_match_batch        (the reference's own host wrapper,
#                      przm_lz77.cu:458-475) tile finder over n bytes in
#                      32 KiB tiles, <<<224, 256>>>; writes d_matches[0, n).
#   cuda_lz77_radix_strike_batch (przm_lz77.cu:477-502) clears the 2 MiB
#                      d_radix_table (2^19 u32) and runs the radix-strike
#                      kernel; writes d_matches[p] only where it finds a
#                      match, so the caller clears d_matches (n x u32) first.
#                      All reads stay below n.

_REFCUDA = None


def ref_cuda_path() -> str:
    return os.path.join(HERE, "_ref", "libprzm_ref_cuda.so")


def ref_cuda_available() -> bool:
    return os.path.exists(ref_cuda_path())


def ref_cuda() -> C.CDLL:
    global _REFCUDA
    if _REFCUDA is None:
        R = C.CDLL(ref_cuda_path())
        vp, u32, u64 = C.c_void_p, C.c_uint32, C.c_uint64
        R.ref_histogram.restype = C.c_int
        R.ref_histogram.argtypes = [vp, u32, vp, vp, vp]
        R.ref_vans_encode4x.restype = C.c_int
        R.ref_vans_encode4x.argtypes = [vp, u32, vp, vp, vp, u32, vp, vp, vp, vp]
        R.ref_tokenize.restype = C.c_int
        R.ref_tokenize.argtypes = [vp, u64, vp, vp, vp, vp, vp, vp, vp, vp, vp, u32, vp]
        R.cuda_lz77_match_batch.restype = C.c_int
        R.cuda_lz77_match_batch.argtypes = [vp, C.c_size_t, vp, C.c_size_t, vp]
        R.cuda_lz77_radix_strike_batch.restype = C.c_int
        R.cuda_lz77_radix_strike_batch.argtypes = [vp, C.c_size_t, vp, vp, C.c_size_t, vp]
        _REFCUDA = R
    return _REFCUDA


def ref_distance_to_code(d: int) -> tuple[int, int, int]:
    """The reference decoder's own distance coder (przm_distance_to_code)."""
    code, nb = C.c_uint8(), C.c_uint8()
    ex = C.c_uint32()
    r = dec().przm_distance_to_code(d, C.byref(code), C.byref(ex), C.byref(nb))
    if r != 0:
        raise ValueError(f"reference distance coder error {r}")
    return code.value, ex.value, nb.value


def ref_code_to_distance(code: int, extra: int) -> int:
    d = C.c_uint32()
    r = dec().przm_code_to_distance(code, extra, C.byref(d))
    if r != 0:
        raise ValueError(f"reference distance decoder error {r}")
    return d.value


def ref_decode_dist4(stream: bytes, n: int) -> bytes:
    """Decode a Mode 12 (0x0C) code stream of n codes with the reference decoder."""
    s = _u8(stream)
    out = np.zeros(n + 64, np.uint8)
    r = dec().przm_vans_decode_dist4(_p(s), len(s), _p(out), len(out), n)
    if r != 0:
        raise ValueError(f"reference Mode 12 decode error {r}")
    return bytes(out[:n])


def ref_distance_prefix_decode(container: bytes, cap: int) -> bytes:
    """Decode a distance-prefix container (0x06/0x0A/0x0B) into LEB128 varints."""
    s = _u8(container)
    out = np.zeros(cap + 64, np.uint8)
    n = C.c_size_t()
    r = dec().przm_distance_prefix_decode(_p(s), len(s), _p(out), cap, C.byref(n))
    if r != 0:
        raise ValueError(f"reference distance-prefix decode error {r}")
    return bytes(out[:n.value])


def ref_context_classify(p2: int, p1: int, mode: int) -> int:
    """The reference decoder's fiber class of a literal after p2, p1."""
    if mode < 3:
        return dec().przm_context_classify(p1, mode)
    return dec().przm_context_classify_order2(p2, p1)


def ref_reconstitute_fibers(fibers: list[bytes], mode: int) -> bytes:
    """Interleave four fibers back into the literals with the reference decoder."""
    n = sum(len(f) for f in fibers)
    out = np.zeros(n + 64, np.uint8)
    fs = [_u8(f if f else b"\0") for f in fibers]
    r = dec().przm_reconstitute_fibers(_p(out), n, *[_p(f) for f in fs], *[len(f) for f in fibers], mode)
    if r != 0:
        raise ValueError(f"reference reconstitution error {r}")
    return bytes(out[:n])
