"""Python mirror of the reference's Go ``gpu`` package (gpu/bridge.go,
gpu/types.go, gpu/memory.go) over the C ABI of libprzmgpu.so.

Method names and argument meanings follow the Go API; Go's ``error`` return
becomes a raised :class:`GPUError` carrying the C status code.  There is no CPU
fallback: every call runs the CUDA path, and a missing library or device raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

from . import _lib

L = _lib.lib

# ---- constants of gpu/types.go:8-16 and gpu/bridge.go:148-153 -------------
Window64K = 64 * 1024
Window1M = 1024 * 1024
Window8M = 8 * 1024 * 1024
MinMatchLen = 4
MaxMatchLen32 = 4095
MaxOffset32 = 1048575
MaxMatchLen64 = 65535
TokenizerTileSize = 32768
MaxTileCmdBytes = 36864
MaxTileOffBytes = 36864
MaxTileLitBytes = 36864

PROFILE_D2D = 0
PROFILE_ANS = 1
PROFILE_ANS_DIST = 2  # PROFILE_ANS with Section 3 as PackageOffsetsSection (the CPU compressor's Section 3)
PROFILE_ANS_SHEAF = 3  # PROFILE_ANS_DIST with Section 4 as PackageLiteralsSection (sheaf foliations)
TUNING_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")
NORM_GO = 0
NORM_CPU = 1


class GPUError(RuntimeError):
    """A failed call; ``code`` is the PRZMG_ERR_* status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} (status {code})")
        self.code = code


def _check(code: int) -> None:
    if code != 0:
        raise GPUError(code, L().przmg_last_error().decode(errors="replace"))


def _u8(data) -> np.ndarray:
    if isinstance(data, np.ndarray):
        return np.ascontiguousarray(data.reshape(-1).view(np.uint8))
    return np.frombuffer(bytes(data), dtype=np.uint8)


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data) if a.size else C.c_void_p(0)


# ---- types (gpu/types.go) ---------------------------------------------------
def PackMatch32(length: int, offset: int) -> int:
    """gpu/types.go:27-33"""
    if length < MinMatchLen or offset == 0:
        return 0
    return (min(length, MaxMatchLen32) << 20) | (offset & MaxOffset32)


def UnpackMatch32(desc: int) -> tuple[int, int]:
    """gpu/types.go:36-38"""
    return desc >> 20, desc & MaxOffset32


def IsMatch32(desc: int) -> bool:
    """gpu/types.go:41-43"""
    return (desc >> 20) >= MinMatchLen


@dataclass
class LZ77Match:
    Position: int
    Offset: int
    Length: int
    Literal: int = 0


@dataclass
class GPUProfile:
    IngressDMABytes: int = 0
    IngressDMATimeMs: float = 0.0
    IngressDMABandwidthGBps: float = 0.0
    KernelTimeMs: float = 0.0
    InternalVRAMBandwidthGBps: float = 0.0
    EgressDMABytes: int = 0
    EgressDMATimeMs: float = 0.0
    EgressDMABandwidthGBps: float = 0.0
    TotalRoundTripMs: float = 0.0
    EndToEndBandwidthGBps: float = 0.0
    PCIeOverheadPercent: float = 0.0
    DeviceName: str = ""
    SMCount: int = 0
    TotalVRAMBytes: int = 0
    PipelinedChunks: int = 0

    @staticmethod
    def of(p: "_lib.Profile") -> "GPUProfile":
        return GPUProfile(p.ingress_dma_bytes, p.ingress_dma_time_ms, p.ingress_dma_bandwidth_gbps, p.kernel_time_ms,
                          p.internal_vram_bandwidth_gbps, p.egress_dma_bytes, p.egress_dma_time_ms,
                          p.egress_dma_bandwidth_gbps, p.total_round_trip_ms, p.end_to_end_bandwidth_gbps,
                          p.pcie_overhead_percent, p.device_name.decode(errors="replace"), p.sm_count,
                          p.total_vram_bytes, p.pipelined_chunks)


@dataclass
class TokenizerProfile:
    KernelTimeMs: float = 0.0
    Pass1Ms: float = 0.0
    Pass2Ms: float = 0.0
    Pass3Ms: float = 0.0
    TotalRoundTripMs: float = 0.0
    ThroughputGBps: float = 0.0
    CmdBytes: int = 0
    OffsetBytes: int = 0
    LiteralBytes: int = 0
    NumChunks: int = 0

    @staticmethod
    def of(p: "_lib.TokProfile") -> "TokenizerProfile":
        return TokenizerProfile(p.kernel_time_ms, p.pass1_ms, p.pass2_ms, p.pass3_ms, p.total_round_trip_ms,
                                p.throughput_gbps, p.cmd_bytes, p.offset_bytes, p.literal_bytes, p.num_chunks)


@dataclass
class DeviceTokenStreams:
    DFinalCmds: int
    DFinalOffs: int
    DFinalLits: int
    DTotals: int
    CmdLen: int
    OffLen: int
    LitLen: int
    NumChunks: int
    Stream: int

    def _c(self) -> "_lib.DevStreams":
        return _lib.DevStreams(self.DFinalCmds, self.DFinalOffs, self.DFinalLits, self.DTotals, self.CmdLen,
                               self.OffLen, self.LitLen, self.NumChunks, self.Stream)


# ---- discovery / lifetime ---------------------------------------------------
def IsAvailable() -> bool:
    """gpu/bridge.go:61"""
    return bool(L().przmg_is_available())


def SetMockUnavailableForTest(unavailable: bool) -> None:
    """gpu/bridge.go:45"""
    L().przmg_set_mock_unavailable(1 if unavailable else 0)


def SetMockMatchErrorForTest(code: int | None) -> None:
    """gpu/bridge.go:50: any non-zero code makes the match/tokenize/compress
    calls fail with PRZMG_ERR_MOCK; None or 0 clears it."""
    L().przmg_set_mock_match_error(int(code or 0))


_GLOBAL: "GPUCompressor | None" = None


def GetGlobalCompressor() -> "GPUCompressor":
    """gpu/bridge.go:96-114: process-wide compressor on device 0."""
    global _GLOBAL
    if _GLOBAL is not None and _GLOBAL._h:
        return _GLOBAL
    h = C.c_void_p()
    _check(L().przmg_get_global(C.byref(h)))
    _GLOBAL = GPUCompressor(_handle=h)
    return _GLOBAL


def ResetGlobalCompressorForTest() -> None:
    """gpu/bridge.go:117-123"""
    global _GLOBAL
    if _GLOBAL is not None:
        _GLOBAL._h = None
    _GLOBAL = None
    L().przmg_reset_global_for_test()


def NormalizeFreq(counts, targetM: int = 4096) -> np.ndarray:
    """gpu/bridge.go:2777-2829"""
    c = np.ascontiguousarray(counts, np.uint32)
    out = np.zeros(256, np.uint16)
    L().przmg_normalize_freq(_ptr(c), targetM, _ptr(out))
    return out


def NormalizeFrequencies(counts) -> np.ndarray:
    """core/literals/literals.go:78-140"""
    c = np.ascontiguousarray(counts, np.uint32)
    out = np.zeros(256, np.uint16)
    L().przmg_normalize_frequencies(_ptr(c), _ptr(out))
    return out


def BuildCDF(freq) -> np.ndarray:
    """gpu/bridge.go:2832-2841"""
    f = np.ascontiguousarray(freq, np.uint16)
    out = np.zeros(257, np.uint16)
    L().przmg_build_cdf(_ptr(f), _ptr(out))
    return out


def SerializeMatrix(freq) -> bytes:
    """gpu/bridge.go:2844-2886"""
    f = np.ascontiguousarray(freq, np.uint16)
    out = np.zeros(1024, np.uint8)
    n = L().przmg_serialize_matrix(_ptr(f), _ptr(out))
    return bytes(out[:n])


def SizeClass(meanInputBytes: int) -> int:
    """Size class of a batch by its mean input size (0..3)."""
    return int(L().przmg_size_class(meanInputBytes))


def FrameBound(n: int) -> int:
    return int(L().przmg_frame_bound(n))


def AllocPinnedHost(size: int) -> int:
    """gpu/memory.go:51 (returns the host address)"""
    p = C.c_void_p()
    _check(L().przmg_alloc_pinned_host(size, C.byref(p)))
    return p.value or 0


def FreePinnedHost(ptr: int) -> None:
    """gpu/memory.go:78"""
    _check(L().przmg_free_pinned_host(C.c_void_p(ptr)))


class PinnedBuffer:
    """gpu/memory.go:91-95: a pinned slice (Bytes, a numpy view of the first
    len bytes) and its host address Ptr."""

    def __init__(self, Bytes: np.ndarray, Ptr: int):
        self.Bytes = Bytes
        self.Ptr = Ptr

    @staticmethod
    def _of(ptr: int, alloc: int, length: int) -> "PinnedBuffer":
        raw = (C.c_uint8 * alloc).from_address(ptr)
        return PinnedBuffer(np.frombuffer(raw, np.uint8)[:length], ptr)


class PinnedBufferPool:
    """gpu/memory.go:98-165 over przmg_pinned_pool_*: Get, Put, Close."""

    def __init__(self, bufSize: int, initialCap: int = 0):
        """NewPinnedBufferPool, gpu/memory.go:108"""
        h = C.c_void_p()
        _check(L().przmg_pinned_pool_create(bufSize, initialCap, C.byref(h)))
        self._h = h
        self.bufSize = bufSize

    @classmethod
    def _of(cls, handle, bufSize: int) -> "PinnedBufferPool":
        p = cls.__new__(cls)
        p._h = handle
        p.bufSize = bufSize
        return p

    def Get(self) -> PinnedBuffer:
        b = C.c_void_p()
        _check(L().przmg_pinned_pool_get(self._h, C.byref(b)))
        return PinnedBuffer._of(b.value, self.bufSize, self.bufSize)

    def Put(self, buf: PinnedBuffer) -> None:
        L().przmg_pinned_pool_put(self._h, C.c_void_p(buf.Ptr), len(buf.Bytes))

    def Pooled(self) -> int:
        return int(L().przmg_pinned_pool_pooled(self._h))

    def Close(self) -> None:
        if self._h:
            _check(L().przmg_pinned_pool_close(self._h))
        self._h = None


class GPUCompressor:
    """gpu/bridge.go:239-288: one device context with its own stream and
    grow-only device pools; calls on one instance are serialised."""

    def __init__(self, deviceID: int = 0, _handle=None):
        if _handle is not None:
            self._h = _handle
            self._owned = False
        else:
            h = C.c_void_p()
            _check(L().przmg_init(deviceID, C.byref(h)))
            self._h = h
            self._owned = True
        major, minor, sm = C.c_int32(), C.c_int32(), C.c_int32()
        vram = C.c_uint64()
        name = C.create_string_buffer(256)
        _check(L().przmg_device_info(self._h, C.byref(major), C.byref(minor), name, 256, C.byref(sm), C.byref(vram)))
        self.ComputeMajor = major.value
        self.ComputeMinor = minor.value
        self.DeviceName = name.value.decode(errors="replace")
        self.SMCount = sm.value
        self.TotalVRAMBytes = vram.value
        self.LoadTuning()

    @property
    def handle(self):
        return self._h

    # -- launch geometry per size class (przm_b200/tuning.json) --
    def SetTuning(self, sizeClass: int, front: int, ctasPerSM: int, verifyChunk: int) -> None:
        _check(L().przmg_set_tuning(self._h, sizeClass, front, ctasPerSM, verifyChunk))

    def GetTuning(self, sizeClass: int) -> dict[str, int]:
        f, c, v = C.c_int32(), C.c_int32(), C.c_int32()
        _check(L().przmg_get_tuning(self._h, sizeClass, C.byref(f), C.byref(c), C.byref(v)))
        return {"front": f.value, "ctas_per_sm": c.value, "verify_chunk": v.value}

    def LoadTuning(self, path: str | None = None) -> bool:
        """Applies the autotuner's table (przm_b200/tuning.json by default);
        False when there is none (the library's built-in values stay)."""
        import json
        path = path or TUNING_PATH
        if not os.path.exists(path):
            return False
        table = json.load(open(path))
        for cls, t in table.get("classes", {}).items():
            self.SetTuning(int(cls), int(t["front"]), int(t["ctas_per_sm"]), int(t["verify_chunk"]))
        return True

    def SetFrontWait(self, limitNs: int, addUnreachableWait: bool = False) -> None:
        """Limit of one wait of the persistent front end; the flag appends a
        wait that never ends to batches laid out afterwards (testing)."""
        _check(L().przmg_set_front_wait(self._h, limitNs, 1 if addUnreachableWait else 0))

    def Close(self) -> None:
        """gpu/bridge.go:513"""
        if self._h and self._owned:
            _check(L().przmg_close(self._h))
        self._h = None

    # -- match finding --
    def MatchLZ77(self, src) -> tuple[list[LZ77Match], GPUProfile]:
        """gpu/bridge.go:1480"""
        pos, off, ln, prof = self.MatchLZ77Arrays(src)
        return [LZ77Match(int(p), int(o), int(l)) for p, o, l in zip(pos, off, ln)], prof

    def MatchLZ77Arrays(self, src, chunk: int | None = None):
        """MatchLZ77 (or MatchLZ77Streaming when chunk is given) as numpy arrays
        (positions, offsets, lengths, profile)."""
        a = _u8(src)
        out = np.zeros(max(len(a), 1), dtype=_lib.MATCH_DTYPE)
        nout = C.c_uint64()
        p = _lib.Profile()
        if chunk is None:
            _check(L().przmg_match_lz77(self._h, _ptr(a), len(a), _ptr(out), len(out), C.byref(nout), C.byref(p)))
        else:
            _check(L().przmg_match_lz77_streaming(self._h, _ptr(a), len(a), chunk, _ptr(out), len(out),
                                                  C.byref(nout), C.byref(p)))
        m = out[: nout.value]
        return m["position"].copy(), m["offset"].copy(), m["length"].copy(), GPUProfile.of(p)

    def MatchLZ77Streaming(self, src, chunkSize: int) -> tuple[list[LZ77Match], GPUProfile]:
        """gpu/bridge.go:1461"""
        pos, off, ln, prof = self.MatchLZ77Arrays(src, chunkSize)
        return [LZ77Match(int(p), int(o), int(l)) for p, o, l in zip(pos, off, ln)], prof

    def MatchTable(self, src) -> np.ndarray:
        """Per-position descriptors used by Tokenize/CompressD2D (dMatch)."""
        a = _u8(src)
        out = np.zeros(max(len(a), 1), np.uint32)
        _check(L().przmg_match_table(self._h, _ptr(a), len(a), _ptr(out)))
        return out[: len(a)]

    # -- tokenization --
    def Tokenize(self, src) -> tuple[bytes, bytes, bytes, TokenizerProfile]:
        """gpu/bridge.go:1895"""
        a = _u8(src)
        tiles = max((len(a) + TokenizerTileSize - 1) // TokenizerTileSize, 1)
        cap = tiles * 36864
        cmd, off, lit = (np.zeros(cap, np.uint8) for _ in range(3))
        lens = (C.c_uint64 * 3)()
        p = _lib.TokProfile()
        _check(L().przmg_tokenize(self._h, _ptr(a), len(a), _ptr(cmd), cap, _ptr(off), cap, _ptr(lit), cap, lens,
                                  C.byref(p)))
        return bytes(cmd[: lens[0]]), bytes(off[: lens[1]]), bytes(lit[: lens[2]]), TokenizerProfile.of(p)

    def TokenizeDevice(self, src) -> tuple[DeviceTokenStreams, TokenizerProfile]:
        """gpu/bridge.go:2139 (pointers valid until the next call)"""
        a = _u8(src)
        d = _lib.DevStreams()
        p = _lib.TokProfile()
        _check(L().przmg_tokenize_device(self._h, _ptr(a), len(a), C.byref(d), C.byref(p)))
        return (DeviceTokenStreams(d.d_final_cmds, d.d_final_offs, d.d_final_lits, d.d_totals, d.cmd_len, d.off_len,
                                   d.lit_len, d.num_chunks, d.stream), TokenizerProfile.of(p))

    TokenizeDeviceZeroCopy = TokenizeDevice  # gpu/bridge.go:2247

    def TokenizeDeviceOnly(self, n: int) -> tuple[bytes, bytes, bytes, TokenizerProfile]:
        """gpu/bridge.go:1915: the tokenizer alone, again, on the input and
        match table staged by the last one-input call (n must be its size)."""
        tiles = max((n + TokenizerTileSize - 1) // TokenizerTileSize, 1)
        cap = tiles * 36864
        cmd, off, lit = (np.zeros(cap, np.uint8) for _ in range(3))
        lens = (C.c_uint64 * 3)()
        p = _lib.TokProfile()
        _check(L().przmg_tokenize_device_only(self._h, n, _ptr(cmd), cap, _ptr(off), cap, _ptr(lit), cap, lens,
                                              C.byref(p)))
        return bytes(cmd[: lens[0]]), bytes(off[: lens[1]]), bytes(lit[: lens[2]]), TokenizerProfile.of(p)

    def TokenizePointersDeviceOnly(self, n: int) -> tuple[DeviceTokenStreams, TokenizerProfile]:
        """gpu/bridge.go:2163 (pointers valid until the next call)"""
        d = _lib.DevStreams()
        p = _lib.TokProfile()
        _check(L().przmg_tokenize_pointers_device_only(self._h, n, C.byref(d), C.byref(p)))
        return (DeviceTokenStreams(d.d_final_cmds, d.d_final_offs, d.d_final_lits, d.d_totals, d.cmd_len, d.off_len,
                                   d.lit_len, d.num_chunks, d.stream), TokenizerProfile.of(p))

    def GetPinned(self, size: int) -> tuple["PinnedBuffer", "PinnedBufferPool"]:
        """gpu/bridge.go:452: a buffer from the context's pool of the next
        power-of-two size; Bytes is sliced to size (as in the reference)."""
        buf, pool = C.c_void_p(), C.c_void_p()
        _check(L().przmg_get_pinned(self._h, size, C.byref(buf), C.byref(pool)))
        p = PinnedBufferPool._of(pool, int(L().przmg_pinned_pool_buf_size(pool)))
        return PinnedBuffer._of(buf.value, p.bufSize, size), p

    def DownloadDeviceBytes(self, dPtr: int, size: int) -> bytes:
        """gpu/bridge.go:2253"""
        out = np.zeros(max(size, 1), np.uint8)
        _check(L().przmg_download_device_bytes(self._h, dPtr, size, _ptr(out)))
        return bytes(out[:size])

    # -- frames --
    def EncodeD2D(self, streams: DeviceTokenStreams, uSize: int, windowLog: int = 0) -> tuple[bytes, GPUProfile]:
        """gpu/bridge.go:2466"""
        cap = 64 + streams.CmdLen + streams.OffLen + streams.LitLen + 32
        out = np.zeros(cap, np.uint8)
        n = C.c_uint64()
        p = _lib.Profile()
        cs = streams._c()
        _check(L().przmg_encode_d2d(self._h, C.byref(cs), uSize, windowLog, _ptr(out), cap, C.byref(n), C.byref(p)))
        return bytes(out[: n.value]), GPUProfile.of(p)

    def CompressD2D(self, src) -> tuple[bytes, GPUProfile]:
        """gpu/bridge.go:2486"""
        return self.Compress(src, PROFILE_D2D)

    def Compress(self, src, profile: int = PROFILE_ANS) -> tuple[bytes, GPUProfile]:
        """One frame: PROFILE_D2D (CompressD2D bytes), PROFILE_ANS (match +
        tokenize + ANS frame, input < 16 MiB), PROFILE_ANS_DIST (that frame
        with a coded Section 3) or PROFILE_ANS_SHEAF (and a coded Section 4)."""
        a = _u8(src)
        cap = FrameBound(len(a))
        out = np.zeros(cap, np.uint8)
        n = C.c_uint64()
        p = _lib.Profile()
        fn = L().przmg_compress_d2d if profile == PROFILE_D2D else None
        if fn is not None:
            _check(fn(self._h, _ptr(a), len(a), _ptr(out), cap, C.byref(n), C.byref(p)))
        else:
            _check(L().przmg_compress(self._h, _ptr(a), len(a), profile, _ptr(out), cap, C.byref(n), C.byref(p)))
        return bytes(out[: n.value]), GPUProfile.of(p)

    def CompressBatch(self, inputs, profile: int = PROFILE_ANS, batched: bool = True):
        """Many inputs in one call; returns (frames, statuses, profile)."""
        arrs = [_u8(x) for x in inputs]
        outs = [np.zeros(FrameBound(len(a)), np.uint8) for a in arrs]
        jobs = (_lib.Job * max(len(arrs), 1))()
        for i, (a, o) in enumerate(zip(arrs, outs)):
            jobs[i].src = a.ctypes.data if a.size else None
            jobs[i].n = len(a)
            jobs[i].dst = o.ctypes.data
            jobs[i].cap = len(o)
        p = _lib.Profile()
        _check(L().przmg_compress_batch(self._h, jobs, len(arrs), profile, 1 if batched else 0, C.byref(p)))
        frames = [bytes(o[: jobs[i].out_len]) for i, o in enumerate(outs)]
        return frames, [jobs[i].status for i in range(len(arrs))], GPUProfile.of(p)

    def CompressPacked(self, host_in: np.ndarray, sizes, profile: int = PROFILE_ANS,
                       host_out: np.ndarray | None = None) -> tuple[np.ndarray, np.ndarray]:
        """Back-to-back inputs in one host buffer -> back-to-back frames and
        their sizes (one upload, one launch sequence, one download)."""
        sz = np.ascontiguousarray(sizes, np.uint64)
        if host_out is None:
            host_out = np.zeros(int(sum(FrameBound(int(s)) for s in sz)) + 64, np.uint8)
        out_sizes = np.zeros(max(len(sz), 1), np.uint32)
        total = C.c_uint64()
        _check(L().przmg_compress_packed(self._h, C.c_void_p(host_in.ctypes.data), _ptr(sz), len(sz), profile,
                                         C.c_void_p(host_out.ctypes.data), host_out.nbytes, _ptr(out_sizes),
                                         C.byref(total)))
        return host_out[: total.value], out_sizes[: len(sz)]

    # -- histogram / flat / V-ANS --
    def ComputeHistogramGPU(self, dIn: int, n: int, stream: int = 0):
        """gpu/bridge.go:2890 -> (counts, ms, GB/s)"""
        counts = np.zeros(256, np.uint32)
        ms, gb = C.c_double(), C.c_double()
        _check(L().przmg_compute_histogram_gpu(self._h, dIn, n, stream, _ptr(counts), C.byref(ms), C.byref(gb)))
        return counts, ms.value, gb.value

    def ComputeHistogramHost(self, src):
        """gpu/bridge.go:2961"""
        a = _u8(src)
        counts = np.zeros(256, np.uint32)
        p = _lib.Profile()
        _check(L().przmg_compute_histogram_host(self._h, _ptr(a), len(a), _ptr(counts), C.byref(p)))
        return counts, GPUProfile.of(p)

    def PackStreamFlatGPU(self, dIn: int, dOut: int, n: int, stream: int = 0):
        """gpu/bridge.go:3033 -> (n+5, ms, GB/s)"""
        ol = C.c_uint64()
        ms, gb = C.c_double(), C.c_double()
        _check(L().przmg_pack_stream_flat_gpu(self._h, dIn, dOut, n, stream, C.byref(ol), C.byref(ms), C.byref(gb)))
        return ol.value, ms.value, gb.value

    def PackStreamFlatHost(self, src):
        """gpu/bridge.go:3079"""
        a = _u8(src)
        out = np.zeros(len(a) + 8, np.uint8)
        ol = C.c_uint64()
        p = _lib.Profile()
        _check(L().przmg_pack_stream_flat_host(self._h, _ptr(a), len(a), _ptr(out), len(out), C.byref(ol), C.byref(p)))
        return bytes(out[: ol.value]), GPUProfile.of(p)

    def VANSEncode4xGPU(self, dIn: int, dOut: int, n: int, freq, cdf, matBytes: bytes, stream: int = 0):
        """gpu/bridge.go:3161 -> (size, ms, GB/s)"""
        f = np.ascontiguousarray(freq, np.uint16)
        c = np.ascontiguousarray(cdf, np.uint16)
        m = np.frombuffer(bytes(matBytes) or b"\0", np.uint8)
        ol = C.c_uint64()
        ms, gb = C.c_double(), C.c_double()
        _check(L().przmg_vans_encode4x_gpu(self._h, dIn, dOut, n, _ptr(f), _ptr(c), _ptr(m), len(matBytes), stream,
                                           C.byref(ol), C.byref(ms), C.byref(gb)))
        return ol.value, ms.value, gb.value

    def VANSEncode4xHost(self, src) -> tuple[bytes, GPUProfile]:
        """gpu/bridge.go:3233"""
        a = _u8(src)
        cap = 2 * len(a) + 1024
        out = np.zeros(cap, np.uint8)
        ol = C.c_uint64()
        p = _lib.Profile()
        _check(L().przmg_vans_encode4x_host(self._h, _ptr(a), len(a), _ptr(out), cap, C.byref(ol), C.byref(p)))
        return bytes(out[: ol.value]), GPUProfile.of(p)

    def VANSEncodeBatch(self, dIn: int, inOffs, lens, norm: int, dOut: int, outOffs, stream: int = 0) -> np.ndarray:
        """Histogram + normalise + V-ANS of many device streams (container sizes)."""
        io = np.ascontiguousarray(inOffs, np.uint64)
        ln = np.ascontiguousarray(lens, np.uint32)
        oo = np.ascontiguousarray(outOffs, np.uint64)
        ol = np.zeros(max(len(ln), 1), np.uint32)
        _check(L().przmg_vans_encode_batch(self._h, dIn, _ptr(io), _ptr(ln), len(ln), norm, dOut, _ptr(oo), _ptr(ol),
                                           stream))
        return ol[: len(ln)]

    def PackageOffsetsBatch(self, dDist: int, distOffs, counts, dOut: int, outOffs, outCaps,
                            stream: int = 0) -> np.ndarray:
        """PackageOffsetsSection (core/distance/distance.go:825) of many device
        uint32 distance arrays: Section 3 sizes (bytes written at dOut + outOffs)."""
        do = np.ascontiguousarray(distOffs, np.uint64)
        ct = np.ascontiguousarray(counts, np.uint32)
        oo = np.ascontiguousarray(outOffs, np.uint64)
        oc = np.ascontiguousarray(outCaps, np.uint64)
        ol = np.zeros(max(len(ct), 1), np.uint64)
        _check(L().przmg_package_offsets_batch(self._h, dDist, _ptr(do), _ptr(ct), len(ct), dOut, _ptr(oo), _ptr(oc),
                                               _ptr(ol), stream))
        return ol[: len(ct)]

    def PackageLiteralsBatch(self, dIn: int, inOffs, lens, dOut: int, outOffs, outCaps,
                             stream: int = 0) -> tuple[np.ndarray, np.ndarray]:
        """PackageLiteralsSection (core/literals/literals.go:664) of many device
        literal streams: (Section 4 sizes, flag nibbles 0x80 or 0)."""
        io = np.ascontiguousarray(inOffs, np.uint64)
        ln = np.ascontiguousarray(lens, np.uint32)
        oo = np.ascontiguousarray(outOffs, np.uint64)
        oc = np.ascontiguousarray(outCaps, np.uint64)
        ol = np.zeros(max(len(ln), 1), np.uint64)
        nb = np.zeros(max(len(ln), 1), np.uint8)
        _check(L().przmg_package_literals_batch(self._h, dIn, _ptr(io), _ptr(ln), len(ln), dOut, _ptr(oo), _ptr(oc),
                                                _ptr(ol), _ptr(nb), stream))
        return ol[: len(ln)], nb[: len(ln)]

    # -- the GPU decoder (decompress.go:380-700 semantics) --
    def Decompress(self, frame) -> bytes:
        """Decompress (api.go:44) on the device: one frame from host memory."""
        f = _u8(frame)
        if len(f) >= 8 and bytes(f[:4]) == b"PRZM":
            u = int(f[5]) | int(f[6]) << 8 | int(f[7]) << 16
        else:
            u = 0
        out = np.zeros(max(u, 1), np.uint8)
        n = C.c_uint64()
        _check(L().przmg_decompress(self._h, _ptr(f) if len(f) else None, len(f), _ptr(out), len(out), C.byref(n)))
        return bytes(out[: n.value])

    def DecompressBatchDevice(self, dSrc: int, srcOffs, srcLens, dDst: int, dstOffs, dstCaps,
                              stream: int = 0) -> tuple[np.ndarray, np.ndarray]:
        """Device-resident frames decoded on the device: (statuses, sizes)."""
        so = np.ascontiguousarray(srcOffs, np.uint64)
        sl = np.ascontiguousarray(srcLens, np.uint32)
        do = np.ascontiguousarray(dstOffs, np.uint64)
        dc = np.ascontiguousarray(dstCaps, np.uint32)
        st = np.zeros(max(len(sl), 1), np.int32)
        ol = np.zeros(max(len(sl), 1), np.uint64)
        _check(L().przmg_decompress_batch_device(self._h, dSrc, _ptr(so), _ptr(sl), len(sl), dDst, _ptr(do), _ptr(dc),
                                                 _ptr(st), _ptr(ol), stream))
        return st[: len(sl)], ol[: len(sl)]

    # -- benchmarks --
    def BenchmarkVRAMBandwidth(self, sizeMB: int = 256, iterations: int = 10) -> float:
        g = C.c_double()
        _check(L().przmg_benchmark_vram_bandwidth(self._h, sizeMB, iterations, C.byref(g)))
        return g.value

    def BenchmarkD2DEntropy(self, sizeMB: int = 16, iterations: int = 10) -> float:
        g = C.c_double()
        _check(L().przmg_benchmark_d2d_entropy(self._h, sizeMB, iterations, C.byref(g)))
        return g.value

    def BenchmarkEntropyVRAM(self, sizeMB: int = 16, iterations: int = 3) -> float:
        g = C.c_double()
        _check(L().przmg_benchmark_entropy_vram(self._h, sizeMB, iterations, C.byref(g)))
        return g.value


class DeviceBatch:
    """Inputs resident in HBM, compressed by one enqueue of the whole
    pipeline (optionally a replayed CUDA graph)."""

    def __init__(self, comp: GPUCompressor, sizes, profile: int = PROFILE_ANS):
        self.comp = comp
        self.sizes = np.ascontiguousarray(sizes, np.uint64)
        h = C.c_void_p()
        _check(L().przmg_batch_create(comp.handle, _ptr(self.sizes), len(self.sizes), profile, C.byref(h)))
        self._h = h
        self.in_offs = np.zeros(max(len(self.sizes), 1), np.uint64)
        self.out_offs = np.zeros(max(len(self.sizes), 1), np.uint64)
        d_in, d_out = C.c_uint64(), C.c_uint64()
        _check(L().przmg_batch_inputs(h, C.byref(d_in), _ptr(self.in_offs)))
        _check(L().przmg_batch_outputs(h, C.byref(d_out), _ptr(self.out_offs)))
        self.d_in = d_in.value
        self.d_out = d_out.value

    def enqueue(self, stream: int = 0, graph: bool = False) -> None:
        _check(L().przmg_batch_enqueue(self._h, stream, 1 if graph else 0))

    def enqueue_plain(self, stream: int = 0) -> int:
        """The pipeline once per input, input after input (plain per-input
        launches); returns the kernels launched."""
        n = C.c_int32()
        _check(L().przmg_batch_enqueue_plain(self._h, stream, C.byref(n)))
        return n.value

    def frame_sizes(self) -> np.ndarray:
        out = np.zeros(max(len(self.sizes), 1), np.uint32)
        _check(L().przmg_batch_sizes(self._h, _ptr(out)))
        return out[: len(self.sizes)]

    def info(self) -> dict[str, int]:
        """front (1: the persistent front end), size_class, ctas_per_sm, verify_chunk."""
        i = np.zeros(4, np.uint32)
        _check(L().przmg_batch_info(self._h, _ptr(i)))
        return {"front": int(i[0]), "size_class": int(i[1]), "ctas_per_sm": int(i[2]), "verify_chunk": int(i[3])}

    def launches(self) -> int:
        return int(L().przmg_batch_launch_count(self._h))

    def upload(self, host_packed: np.ndarray, stream: int = 0) -> None:
        """Back-to-back inputs (sum of sizes) from host memory (pinned for
        full speed) into the batch, asynchronously on `stream`."""
        _check(L().przmg_batch_upload(self._h, C.c_void_p(host_packed.ctypes.data), stream))

    def download(self, host_out: np.ndarray, stream: int = 0) -> tuple[int, np.ndarray]:
        """Synchronise and copy the frames back to back into host_out."""
        total = C.c_uint64()
        sizes = np.zeros(max(len(self.sizes), 1), np.uint32)
        _check(L().przmg_batch_download(self._h, C.c_void_p(host_out.ctypes.data), host_out.nbytes, C.byref(total),
                                        _ptr(sizes), stream))
        return total.value, sizes[: len(self.sizes)]

    def verify(self) -> int:
        """Every frame of the last run decoded on the device and compared with
        its input there: the number of frames that do not round-trip."""
        bad = C.c_uint64()
        _check(L().przmg_batch_verify(self._h, C.byref(bad)))
        return bad.value

    STAT_KEYS = ("input_bytes", "frame_bytes", "literal_bytes", "command_bytes", "offset_bytes", "rans_symbols",
                 "rans_emitted_bytes", "uncompressed_frames")

    def stats(self) -> dict[str, int]:
        """Totals of the last run."""
        s = np.zeros(8, np.uint64)
        _check(L().przmg_batch_stats(self._h, _ptr(s)))
        return {k: int(v) for k, v in zip(self.STAT_KEYS, s)}

    def stream_lens(self) -> np.ndarray:
        """(inputs, 6) stream lengths of the last run: commands, op, meta, var,
        offsets, literals."""
        out = np.zeros(max(len(self.sizes), 1) * 6, np.uint32)
        _check(L().przmg_batch_stream_lens(self._h, _ptr(out), len(out)))
        return out[: 6 * len(self.sizes)].reshape(-1, 6)

    def stage_times(self) -> dict[str, float]:
        """One enqueue with events between stages: {stage: device ms}."""
        ms = (C.c_float * 16)()
        n = C.c_int32()
        _check(L().przmg_batch_stage_times(self._h, ms, 16, C.byref(n)))
        return {L().przmg_stage_name(k).decode(): float(ms[k]) for k in range(n.value)}

    def close(self) -> None:
        if self._h:
            _check(L().przmg_batch_destroy(self._h))
        self._h = None


class Server:
    """Continuous-batching request engine over a compressor (przmg_serve_*):
    submit inputs from any thread, poll for frames.  Up to `max_inflight`
    batches run at once within `mem_budget` device bytes."""

    def __init__(self, comp: GPUCompressor, profile: int = PROFILE_ANS, mem_budget: int = 64 << 30,
                 max_inflight: int = 3, max_batch_bytes: int = 0):
        h = C.c_void_p()
        _check(L().przmg_serve_create(comp.handle, profile, mem_budget, max_inflight, max_batch_bytes, C.byref(h)))
        self._h = h

    def submit(self, src) -> int:
        a = _u8(src)
        rid = C.c_uint64()
        _check(L().przmg_serve_submit(self._h, C.c_void_p(a.ctypes.data), len(a), C.byref(rid)))
        return rid.value

    def poll(self, rid: int, cap: int, wait: bool = True):
        """(frame, t_submit_ns, t_done_ns), or None while pending (wait=False)."""
        out = np.empty(max(cap, 1), np.uint8)
        n, t0, t1 = C.c_uint64(), C.c_uint64(), C.c_uint64()
        r = L().przmg_serve_poll(self._h, rid, 1 if wait else 0, C.c_void_p(out.ctypes.data), cap, C.byref(n),
                                 C.byref(t0), C.byref(t1))
        if r == 0:
            return None
        _check(r if r < 0 else 0)
        return bytes(out[: n.value]), t0.value, t1.value

    STAT_KEYS = ("batches", "done", "bytes_in", "bytes_out", "max_batch", "max_concurrent", "pending", "live")

    def stats(self) -> dict[str, int]:
        s = np.zeros(8, np.uint64)
        _check(L().przmg_serve_stats(self._h, _ptr(s)))
        return {k: int(v) for k, v in zip(self.STAT_KEYS, s)}

    TIMING_KEYS = ("launch_ms", "wait_ms", "out_ms", "max_launch_ms", "max_wait_ms", "max_out_ms")

    def timing(self) -> dict[str, float]:
        t = np.zeros(6, np.float64)
        _check(L().przmg_serve_timing(self._h, _ptr(t)))
        return {k: round(float(v), 3) for k, v in zip(self.TIMING_KEYS, t)}

    def close(self) -> None:
        if self._h:
            _check(L().przmg_serve_destroy(self._h))
        self._h = None
