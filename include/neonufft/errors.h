/* Error codes returned by every C-ABI entry point of the engine.
 * Same enumerators and numeric values as the reference (include/neonufft/errors.h:5-38). */
#pragma once

enum NeonufftError {
  NEONUFFT_SUCCESS,               /* no error */
  NEONUFFT_GENERIC_ERROR,         /* generic error */
  NEONUFFT_MEMORY_ALLOC_ERROR,    /* an allocation through the plan's allocator failed */
  NEONUFFT_UNKNOWN_ERROR,         /* unknown error (non-library exception) */
  NEONUFFT_INTERNAL_ERROR,        /* internal error, e.g. kernel width outside [2, 16] */
  NEONUFFT_INPUT_ERROR,           /* invalid argument */
  NEONUFFT_GPU_ERROR,             /* CUDA runtime or cuFFT error */
  NEONUFFT_NOT_IMPLEMENTED_ERROR, /* feature not implemented */
};

#ifndef __cplusplus
typedef enum NeonufftError NeonufftError;
#endif
