"""B200-native PRZM compression path: LZ77 match finding, tokenization into
PRZM opcodes (Mode 8 op/meta/var split), byte histograms and 4-lane V-ANS,
as hand-written sm_100a CUDA behind the C ABI of include/przmgpu.h.

`przm_b200.gpu` mirrors the reference's Go `gpu` package API.
"""
from . import gpu, workloads  # noqa: F401
from .gpu import GPUCompressor, GPUError, GetGlobalCompressor, IsAvailable  # noqa: F401
