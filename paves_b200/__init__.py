"""paves_b200 — B200-native (sm_100a) implementation of the PAVES GPU search
path: device-resident index layout, batched filtered exact / reduced
precision top-k scans, filtered HNSW level-0 beam search, the GPU worker's
micro-batch loop and a learned scan/graph router.

The compute lives in ``libpaves_gpu.so`` (CUDA + C++), exported through the
C ABI of ``include/paves_gpu.h`` (a drop-in for the reference backend's
``gpu_engine.h``). This package is the host-side mirror used by tests and
benchmarks.
"""
from ._lib import (FV_GPU_PREC_BF16, FV_GPU_PREC_FP8, FV_GPU_PREC_FP32,  # noqa: F401
                   FV_GPU_PREC_SQ8, lib)
from .index import GpuError, GpuIndex  # noqa: F401
from .pred import And, Cmp, In, Not, Or, concat, serialize  # noqa: F401
