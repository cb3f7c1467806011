"""neonufft_b200: a B200-native (sm_100a) NUFFT engine with the GPU plan API of NeoNUFFT.

The compute path is libneonufft_b200.so (hand-written CUDA kernels + cuFFT) behind a C ABI
(include/neonufft_gpu.h). This package is the Python mirror of the reference's plan classes
over that ABI; it contains no numerical fallback.
"""
from .plan import (MODE_ORDER_CMCL, MODE_ORDER_FFT, Batch, GenericError, GPUError, InputError,
                   InternalError, MemoryAllocError, NotImplementedError_, Options, Plan, PlanT3,
                   check_device_status, direct_type1_f64, direct_type2_f64, direct_type3_f64,
                   kernel_launches)

__all__ = [
    "Options", "Plan", "PlanT3", "Batch", "MODE_ORDER_CMCL", "MODE_ORDER_FFT", "GenericError",
    "GPUError", "InputError", "InternalError", "MemoryAllocError", "NotImplementedError_",
    "direct_type1_f64", "direct_type2_f64", "direct_type3_f64", "kernel_launches",
    "check_device_status",
]
