"""gse_b200: B200-native (sm_100a) GSE-k reciprocal-space electrostatics.

The compute path is libgse_b200.so (CUDA kernels behind the C ABI in
include/gse_b200.h).  Modules:

  gse_b200.gse            the reference's class API (CpuGSEk, CpuGaussCharge,
                          CpuGreensFuncGSE, CpuFFTSolver, CpuGrid, CpuEwaldRecip,
                          CpuEwaldDirect), Context, Batch, and the driver's text I/O
  gse_b200.torch_binding  a torch.autograd.Function over a Context
  gse_b200.multi          several GPUs: partitioned batches, max over ranks
  gse_b200.workloads      seeded synthetic systems of the benchmark shapes
  gse_b200.build          the in-tree build of the library and the C++ check program
"""
from ._lib import GseError  # noqa: F401

__all__ = ["GseError"]
