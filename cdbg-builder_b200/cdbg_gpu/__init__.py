"""Host-side Python mirror of the B200 implementation of cdbg-builder's
phase 1 (bucket-write) and phase 2 (bucket-process).

The work happens in libcdbg_gpu.so (CUDA kernels for sm_100a behind the
C-ABI of include/cdbg_gpu.h); this package binds it, reads the on-disk
artifacts and generates the synthetic benchmark workloads.
"""
from . import formats, native, synth  # noqa: F401
from .native import Engine, Server, best_m, host_batch  # noqa: F401
