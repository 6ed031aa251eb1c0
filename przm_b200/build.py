"""Build the native libraries of the package in place.

    libprzmgpu.so    the CUDA path (sm_100a) and its C ABI (include/przmgpu.h)
    libprzm_gen.so   seeded synthetic input generators (host C)

Both land next to this file so they travel with the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _newer(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _sources(ext: tuple[str, ...]) -> list[str]:
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith(ext)]


def build_gpu(force: bool = False, verbose: bool = False) -> str:
    out = os.path.join(HERE, "libprzmgpu.so")
    deps = _sources((".cu", ".cuh", ".h", ".inc")) + [os.path.join(HERE, "..", "include", "przmgpu.h")]
    if force or _newer(out, deps):
        cmd = ["nvcc", *ARCH, "-O3", "-lineinfo", "-std=c++17", "-shared", "-Xcompiler", "-fPIC", "-o", out, os.path.join(CSRC, "api.cu"), "-lcudart"]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
    return out


def build_gen(force: bool = False) -> str:
    out = os.path.join(HERE, "libprzm_gen.so")
    src = os.path.join(CSRC, "przm_gen.c")
    if force or _newer(out, [src]):
        subprocess.run(["gcc", "-O2", "-std=c11", "-shared", "-fPIC", "-o", out, src, "-lm"], check=True)
    return out


def build_all(force: bool = False) -> None:
    build_gen(force)
    build_gpu(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
