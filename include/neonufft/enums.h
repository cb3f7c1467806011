/* Mode ordering and kernel selection, C-compatible.
 * Same enumerators and values as the reference API (include/neonufft/enums.h:6-13), so code
 * written against the reference compiles unchanged. */
#pragma once

enum NeonufftModeOrder {
  NEONUFFT_MODE_ORDER_FFT,
  NEONUFFT_MODE_ORDER_CMCL,
};

enum NeonufftKernelType { NEONUFFT_ES_KERNEL };

#ifndef __cplusplus
typedef enum NeonufftModeOrder NeonufftModeOrder;
typedef enum NeonufftKernelType NeonufftKernelType;
#endif
