"""B200-native engine for the RGF hot path of NEGFtrans.

The compute lives in libnegfgpu.so (C ABI in include/negf_gpu.h, CUDA kernels
for sm_100a); this package is its host-side mirror of the reference's
interface (src/grid.f90, src/negf.f90, src/math_kernel.f90, src/main.f90).
"""
from .constants import A_0, HARTREE, K_B, PI  # noqa: F401

__all__ = ["A_0", "HARTREE", "K_B", "PI"]
