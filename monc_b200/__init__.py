"""monc_b200: MONC's dynamical-core timestep as device-resident CUDA kernels for B200 (sm_100a).

The compute lives in libmoncgpu.so (C ABI in include/monc_gpu.h, sources in monc_b200/csrc);
this package holds its Python binding (api), the model configurations (config) and the seeded
initial states (init).
"""
from . import config, init  # noqa: F401

__all__ = ["config", "init", "api", "build"]
