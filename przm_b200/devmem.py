"""Small device-memory helpers for tests and the benchmark: allocation and
copies on raw device addresses through the CUDA runtime that PyTorch loads
(plumbing only; the compression path lives in libprzmgpu.so)."""
from __future__ import annotations

import ctypes as C
import glob
import os

import numpy as np

_RT = None


def rt() -> C.CDLL:
    global _RT
    if _RT is None:
        import torch  # loads the runtime and creates the primary context lazily
        torch.cuda.init()
        cands = []
        try:
            import nvidia.cuda_runtime as cr
            cands += glob.glob(os.path.join(list(cr.__path__)[0], "lib", "libcudart.so*"))
        except ImportError:
            pass
        cands += ["libcudart.so.12", "libcudart.so"]
        last = None
        for c in cands:
            try:
                _RT = C.CDLL(c)
                break
            except OSError as e:
                last = e
        if _RT is None:
            raise OSError(f"CUDA runtime not found: {last}")
        _RT.cudaMalloc.argtypes = [C.POINTER(C.c_void_p), C.c_size_t]
        _RT.cudaFree.argtypes = [C.c_void_p]
        _RT.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
        _RT.cudaMemcpyAsync.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int, C.c_void_p]
        _RT.cudaDeviceSynchronize.argtypes = []
    return _RT


def _ck(r: int, what: str) -> None:
    if r != 0:
        raise RuntimeError(f"{what} failed with CUDA error {r}")


class DevBuf:
    def __init__(self, n: int):
        p = C.c_void_p()
        _ck(rt().cudaMalloc(C.byref(p), max(n, 16)), "cudaMalloc")
        self.ptr = p.value
        self.n = n

    def free(self) -> None:
        if self.ptr:
            rt().cudaFree(C.c_void_p(self.ptr))
        self.ptr = 0

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def alloc(n: int) -> DevBuf:
    return DevBuf(n)


def upload(a: np.ndarray) -> DevBuf:
    a = np.ascontiguousarray(a)
    b = DevBuf(a.nbytes)
    if a.nbytes:
        _ck(rt().cudaMemcpy(C.c_void_p(b.ptr), C.c_void_p(a.ctypes.data), a.nbytes, 4), "cudaMemcpy")
    return b


def upload_to(ptr: int, a: np.ndarray) -> None:
    a = np.ascontiguousarray(a)
    if a.nbytes:
        _ck(rt().cudaMemcpy(C.c_void_p(ptr), C.c_void_p(a.ctypes.data), a.nbytes, 4), "cudaMemcpy")


def copy(dst: int, src: int, n: int) -> None:
    if n:
        _ck(rt().cudaMemcpy(C.c_void_p(dst), C.c_void_p(src), n, 4), "cudaMemcpy")


def download(ptr: int, n: int) -> bytes:
    out = np.zeros(max(n, 1), np.uint8)
    if n:
        _ck(rt().cudaMemcpy(C.c_void_p(out.ctypes.data), C.c_void_p(ptr), n, 4), "cudaMemcpy")
    return bytes(out[:n])
