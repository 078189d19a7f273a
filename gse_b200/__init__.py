"""gse_b200: B200-native (sm_100a) GSE-k reciprocal-space electrostatics.

The compute path is libgse_b200.so (CUDA kernels behind the C ABI in
include/gse_b200.h).  ``gse_b200.gse`` mirrors the reference's class API
(CpuGSEk, CpuGaussCharge, CpuGreensFuncGSE, CpuFFTSolver) on top of it.
"""
from ._lib import GseError  # noqa: F401

__all__ = ["GseError"]
