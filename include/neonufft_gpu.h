/*
 * neonufft_gpu.h -- C ABI of the B200 NUFFT engine (libneonufft_b200.so).
 *
 * This is the drop-in boundary for the GPU plan of NeoNUFFT. Every entry point takes plain
 * pointers and sizes and returns a NeonufftError; nothing here depends on C++ or on torch.
 * The C++ classes neonufft::gpu::Plan / neonufft::gpu::PlanT3 (include/neonufft/gpu/plan.hpp)
 * are header-only shims over these functions, so C++ code written against the reference
 * compiles and links against this library unchanged.
 *
 * Conventions shared by all entry points:
 *  - All array pointers are DEVICE pointers owned by the caller, as in the reference
 *    (reference include/neonufft/gpu/plan.hpp:30-41).
 *  - Coordinates are passed as `dim` separate arrays (structure of arrays), `loc[d]` holding
 *    the d-th coordinate of every point, of type float (NNB_FLOAT) or double (NNB_DOUBLE).
 *  - Complex data is interleaved (cuComplex / cuDoubleComplex layout).
 *  - Grids and mode arrays are column-major: dimension 0 varies fastest.
 *  - Work is asynchronous on the plan's stream, except where noted (point setup synchronises,
 *    as the reference does: src/neonufft/gpu/plan_impl.hpp:151).
 *  - On failure the function returns an error code and nnb_last_error_message() describes it.
 */
#ifndef NEONUFFT_GPU_H
#define NEONUFFT_GPU_H

#include <stddef.h>
#include <stdint.h>

#include "neonufft/enums.h"
#include "neonufft/errors.h"

#if defined(__GNUC__)
#define NNB_API __attribute__((visibility("default")))
#else
#define NNB_API
#endif

#ifdef __cplusplus
extern "C" {
#else
typedef enum NeonufftError NeonufftError;
#endif

/* Floating-point type of a plan (the reference instantiates T = float, double:
 * src/neonufft/gpu/plan.cpp:47-53). */
typedef enum NnbPrecision { NNB_FLOAT = 0, NNB_DOUBLE = 1 } NnbPrecision;

/* Plan options. The first nine fields mirror neonufft::Options
 * (reference include/neonufft/plan.hpp:19-29). The remaining fields are engine extensions;
 * zero selects the automatic choice. */
typedef struct NnbOptions {
  double tol;
  double upsampfac;
  double recenter_threshold;
  int num_threads;          /* ignored on the GPU, as in the reference */
  int sort_input;           /* ignored: points are always bin-sorted */
  int sort_output;          /* ignored: points are always bin-sorted */
  int kernel_approximation; /* ignored: the ES kernel is always evaluated directly */
  int order;                /* NeonufftModeOrder */
  int kernel_type;          /* NeonufftKernelType */
  int tile[3];              /* subproblem tile (bin) shape in fine-grid cells; 0 = automatic.
                               Method 3 takes {2|4|8, 8|16, 1} (16 rows: single precision) and
                               {4, 4, 1} (single precision); the default is {4, 8, 1}.
                               Method 5 uses {4, 4, 1} */
  int spread_method;        /* 0 = automatic (3 for 3D plans with kernel width <= 8, else 1);
                               1 = warp-private shared-memory slabs; 2 = thread per point;
                               3 = sliding z-window held in registers (3D, width <= 8);
                               4 = method 3 with the row updates on the tensor cores (TF32 with
                               split operands; 3D, single precision, width 5 to 8);
                               5 = spreading on the tcgen05 tensor cores with the region's
                               accumulator in tensor memory (3D, single precision, width <= 8,
                               tiles {4, 4, 1}); interpolation as method 3 */
  int n_spread;             /* kernel width override in [2, 16]; 0 = the reference heuristic */
  int reserved[7];
} NnbOptions;

/* Fills *opt with the reference defaults (tol 1e-3, upsampfac 2, recenter 0.1, CMCL). */
NNB_API void nnb_options_default(NnbOptions* opt);

/* Device allocator used for every buffer a plan owns. Mirrors neonufft::Allocator
 * (reference include/neonufft/allocator.hpp:12-21) as two callbacks. A NULL allocator pointer
 * or NULL callbacks select cudaMalloc / cudaFree (reference src/neonufft/gpu/device_allocator.cpp).
 * `allocate` returns NULL to signal failure; the plan then fails with
 * NEONUFFT_MEMORY_ALLOC_ERROR. */
typedef void* (*NnbAllocateFn)(void* ctx, size_t size);
typedef void (*NnbDeallocateFn)(void* ctx, void* ptr);
typedef struct NnbAllocator {
  NnbAllocateFn allocate;
  NnbDeallocateFn deallocate;
  void* ctx;
} NnbAllocator;

typedef struct NnbPlan_s* NnbPlan;
typedef struct NnbPlanT3_s* NnbPlanT3;

/* ---------------------------------------------------------------------------------------
 * Type 1 / type 2 plan.
 * ------------------------------------------------------------------------------------- */

/* Creates a type-1/2 plan and sets its points.
 * Replaces gpu::Plan<T,DIM>::Plan (reference include/neonufft/gpu/plan.hpp:30-32).
 * dim in {1,2,3}; modes[d] >= 1; sign is the sign of the exponent; stream is a cudaStream_t
 * (NULL = legacy default stream). Synchronises the stream. */
NNB_API NeonufftError nnb_plan_create(NnbPlan* plan, NnbPrecision precision, int dim,
                              const NnbOptions* opt, int sign, int64_t num_nu,
                              const void* const* loc, const int64_t* modes, void* stream,
                              const NnbAllocator* alloc);

/* Replaces the point set. Replaces gpu::Plan<T,DIM>::set_points
 * (reference include/neonufft/gpu/plan.hpp:41). Synchronises the stream. */
NNB_API NeonufftError nnb_plan_set_points(NnbPlan plan, int64_t num_nu, const void* const* loc);

/* Type 1: out[k] = sum_j in[j] exp(i*sign*k.x_j), k in the modes box, written with
 * out_strides (in elements). Replaces gpu::Plan<T,DIM>::transform_type_1
 * (reference include/neonufft/gpu/plan.hpp:34-35). */
NNB_API NeonufftError nnb_plan_transform_type_1(NnbPlan plan, const void* in, void* out,
                                        const int64_t* out_strides);

/* `count` type-1 transforms of the plan's points (engine extension; the reference's type-1/2
 * plan transforms one vector per call): strength vector v at in + v * in_bdist, its modes at
 * out + v * out_bdist (elements; out_bdist at least the span of the strided mode box). Single
 * precision on the z-window kernels (spread methods 3 with the default or 4-row tiles) spreads
 * the vectors two at a time, each staged point serving both, into two fine grids of its own
 * (four when count > 2: the FFTs and deconvolutions of one pair run on an internal stream of
 * the plan while the next pair spreads; the plan's stream waits for them before the call
 * returns, so work enqueued on it afterwards sees every output); other plans run the
 * transforms one at a time. Same results as `count` calls of nnb_plan_transform_type_1. */
NNB_API NeonufftError nnb_plan_transform_type_1_many(NnbPlan plan, int64_t count, const void* in,
                                                     int64_t in_bdist, void* out,
                                                     int64_t out_bdist,
                                                     const int64_t* out_strides);

/* Type 2: out[j] = sum_k in[k] exp(i*sign*k.x_j), in read with in_strides (in elements).
 * Replaces gpu::Plan<T,DIM>::transform_type_2 (reference include/neonufft/gpu/plan.hpp:37-39). */
NNB_API NeonufftError nnb_plan_transform_type_2(NnbPlan plan, const void* in, const int64_t* in_strides,
                                        void* out);

/* Destroys the plan and frees its buffers (reference pImpl deleter,
 * src/neonufft/gpu/plan.cpp:16-21). Accepts NULL. */
NNB_API NeonufftError nnb_plan_destroy(NnbPlan plan);

/* ---------------------------------------------------------------------------------------
 * Type 3 plan.
 * ------------------------------------------------------------------------------------- */

/* Device memory in bytes of the fine grids a type-3 plan with these bounds would allocate.
 * Replaces gpu::PlanT3<T,DIM>::grid_memory_size (reference include/neonufft/gpu/plan.hpp:52-56).
 * Bounds are passed as double; for NNB_FLOAT they are rounded to float first. */
NNB_API NeonufftError nnb_plan_t3_grid_memory_size(NnbPrecision precision, int dim, const NnbOptions* opt,
                                           const double* input_min, const double* input_max,
                                           const double* output_min, const double* output_max,
                                           uint64_t* size);

/* Creates a type-3 plan from point sets (bounds computed on the device).
 * Replaces gpu::PlanT3<T,DIM>::PlanT3(opt, sign, num_in, input_points, num_out, output_points,
 * stream, batch_size, alloc) (reference include/neonufft/gpu/plan.hpp:58-61). Synchronises. */
NNB_API NeonufftError nnb_plan_t3_create(NnbPlanT3* plan, NnbPrecision precision, int dim,
                                 const NnbOptions* opt, int sign, int64_t num_in,
                                 const void* const* input_points, int64_t num_out,
                                 const void* const* output_points, void* stream,
                                 int64_t batch_size, const NnbAllocator* alloc);

/* Creates a type-3 plan from coordinate bounds; points are set later.
 * Replaces gpu::PlanT3<T,DIM>::PlanT3(opt, sign, input_min, input_max, output_min, output_max,
 * stream, batch_size, alloc) (reference include/neonufft/gpu/plan.hpp:63-66). */
NNB_API NeonufftError nnb_plan_t3_create_bounds(NnbPlanT3* plan, NnbPrecision precision, int dim,
                                        const NnbOptions* opt, int sign, const double* input_min,
                                        const double* input_max, const double* output_min,
                                        const double* output_max, void* stream,
                                        int64_t batch_size, const NnbAllocator* alloc);

/* Replaces gpu::PlanT3::set_input_points (reference include/neonufft/gpu/plan.hpp:68-69). */
NNB_API NeonufftError nnb_plan_t3_set_input_points(NnbPlanT3 plan, int64_t num_in,
                                           const void* const* input_points);

/* Replaces gpu::PlanT3::set_output_points (reference include/neonufft/gpu/plan.hpp:71-72). */
NNB_API NeonufftError nnb_plan_t3_set_output_points(NnbPlanT3 plan, int64_t num_out,
                                            const void* const* output_points);

/* Accumulates batch_size input vectors (batch b at in + b*bdist; bdist <= 0 means num_in).
 * Replaces gpu::PlanT3::add_input (reference include/neonufft/gpu/plan.hpp:74). */
NNB_API NeonufftError nnb_plan_t3_add_input(NnbPlanT3 plan, const void* in, int64_t bdist);

/* Computes batch_size outputs (batch b at out + b*bdist; bdist <= 0 means num_out).
 * Replaces gpu::PlanT3::transform (reference include/neonufft/gpu/plan.hpp:76). */
NNB_API NeonufftError nnb_plan_t3_transform(NnbPlanT3 plan, void* out, int64_t bdist);

/* Clears the accumulated input. Replaces gpu::PlanT3::reset
 * (reference include/neonufft/gpu/plan.hpp:78). */
NNB_API NeonufftError nnb_plan_t3_reset(NnbPlanT3 plan);

/* Destroys a type-3 plan. Accepts NULL. */
NNB_API NeonufftError nnb_plan_t3_destroy(NnbPlanT3 plan);

/* ---------------------------------------------------------------------------------------
 * Support.
 * ------------------------------------------------------------------------------------- */

/* Message of the last failing call on this thread ("" if none). */
NNB_API const char* nnb_last_error_message(void);

/* Default device allocator: neonufft::gpu::DeviceAllocator::allocate / deallocate
 * (reference include/neonufft/gpu/device_allocator.hpp:14-21). */
NNB_API NeonufftError nnb_device_alloc(void** ptr, size_t size);
NNB_API NeonufftError nnb_device_free(void* ptr);

/* Plan introspection (engine extension, no reference counterpart). */
typedef struct NnbPlanInfo {
  int dim;
  int precision;       /* NnbPrecision */
  int n_spread;        /* kernel width w */
  int spread_method;   /* method actually used */
  double es_beta;      /* ES kernel shape parameter (as used, i.e. rounded to T) */
  int64_t grid[3];     /* FFT grid (fine grid) dims; 1 for unused dims */
  int64_t spread_grid[3]; /* type 3: spread grid dims; type 1/2: equals grid */
  int tile[3];         /* subproblem tile shape */
  int64_t num_in;      /* points (type 1/2) or sources (type 3) */
  int64_t num_out;     /* type 3 targets */
  int64_t batch_size;
  uint64_t device_bytes; /* bytes currently held through the allocator */
  double input_offset[3], output_offset[3], gamma[3], h[3]; /* type 3 geometry */
} NnbPlanInfo;
NNB_API NeonufftError nnb_plan_info(NnbPlan plan, NnbPlanInfo* info);
NNB_API NeonufftError nnb_plan_t3_info(NnbPlanT3 plan, NnbPlanInfo* info);

/* Per-stage device timing (engine extension). When enabled, the plan records CUDA events on
 * its stream around each stage; nnb_*_stage_times adds the elapsed milliseconds since the last
 * reset into ms[NNB_STAGE_COUNT] (synchronises the stream) and launch counts into count[]. */
enum NnbStage {
  NNB_STAGE_BIN = 0,     /* point binning: rescale, count, scan, permutation */
  NNB_STAGE_SPREAD = 1,  /* ES spreading kernel (the grid is zeroed just before, outside) */
  NNB_STAGE_FFT = 2,     /* cuFFT */
  NNB_STAGE_DECONV = 3,  /* deconvolution (downsample / upsample) */
  NNB_STAGE_INTERP = 4,  /* ES interpolation */
  NNB_STAGE_PHASE = 5,   /* type-3 pre/post phase and bounds */
  NNB_STAGE_COUNT = 6
};
NNB_API NeonufftError nnb_plan_enable_timing(NnbPlan plan, int enable);
NNB_API NeonufftError nnb_plan_stage_times(NnbPlan plan, double* ms, int64_t* count, int reset);
NNB_API NeonufftError nnb_plan_t3_enable_timing(NnbPlanT3 plan, int enable);
NNB_API NeonufftError nnb_plan_t3_stage_times(NnbPlanT3 plan, double* ms, int64_t* count, int reset);

/* FP64 direct NUDFT on the GPU, for accuracy measurement (engine extension; the reference
 * computes the same sums on the CPU in tests/nuft_direct_kernels.cpp:73-293).
 * Coordinates and data are double; sampled outputs only:
 *   type 1: out[s] = sum_j in[j] exp(i*sign*k_s.x_j) for the mode multi-indices k_s given in
 *           modes_idx (num_samples x dim, int64, signed mode numbers);
 *   type 2: out[s] = sum_k in[k] exp(i*sign*k.x_{p_s}) for the points p_s listed in point_idx,
 *           modes in CMCL order, column-major, n_modes[d] per dim;
 *   type 3: out[s] = sum_j in[j] exp(i*sign*s_{t}.x_j) for the targets listed in target_idx. */
NNB_API NeonufftError nnb_direct_type1_f64(int dim, int sign, int64_t num_nu, const double* const* loc,
                                   const double* in, int64_t num_samples, const int64_t* modes_idx,
                                   double* out, void* stream);
NNB_API NeonufftError nnb_direct_type2_f64(int dim, int sign, const int64_t* n_modes, const double* in,
                                   const double* const* loc, int64_t num_samples,
                                   const int64_t* point_idx, double* out, void* stream);
NNB_API NeonufftError nnb_direct_type3_f64(int dim, int sign, int64_t num_in, const double* const* in_loc,
                                   const double* in, const double* const* out_loc,
                                   int64_t num_samples, const int64_t* target_idx, double* out,
                                   void* stream);

/* Allocation-free FP64 direct type-1 sum (engine extension; it has no counterpart in the
 * reference). Same arguments and results as nnb_direct_type1_f64, for callers that cannot call
 * cudaMalloc (a caller-owned memory pool holding the whole device, or code that must not
 * allocate after start-up): the per-block partial sums go to a fixed 16 MiB scratch array in
 * the library's own device memory, kept on every GPU that loads the library until exit, and are
 * added in a fixed order, so the result is also bit-reproducible. Limit:
 * num_samples * ceil(num_nu / 4096) <= 1048576, else NEONUFFT_INPUT_ERROR. Nothing is
 * allocated; the first call on a device looks up the scratch address (make it before any
 * stream capture) and keeps it for the life of the process, so do not call this entry point
 * after cudaDeviceReset (or any other destruction of the device's primary context) in the same
 * process. All calls share the scratch: calls that overlap on the GPU race. */
NNB_API NeonufftError nnb_direct_type1_f64_noalloc(int dim, int sign, int64_t num_nu,
                                                   const double* const* loc, const double* in,
                                                   int64_t num_samples,
                                                   const int64_t* modes_idx, double* out,
                                                   void* stream);

/* Host-only parameter queries (engine extensions; no GPU needed). They expose the engine's own
 * restatement of the reference's heuristics so that sizing can be planned ahead:
 *  - ES kernel width w, shape beta and c = 4/w^2 as used by a plan of this precision
 *    (reference src/neonufft/es_kernel_param.hpp:24-56);
 *  - type-3 geometry per dimension: spread grid nf1, FFT grid, input centre C, output centre D,
 *    gamma and h (reference src/neonufft/util/grid_info_t3.hpp:18-52,
 *    src/contrib/es_kernel/util.hpp:64-105);
 *  - deconvolution factors (-1)^k / phi_hat(2 pi k / nf), k = 0..nf/2, in double. */
NNB_API NeonufftError nnb_es_kernel_params(double tol, double upsampfac, NnbPrecision precision,
                                           int* n_spread, double* beta, double* c);
NNB_API NeonufftError nnb_plan_t3_geometry(NnbPrecision precision, int dim, const NnbOptions* opt,
                                           const double* input_min, const double* input_max,
                                           const double* output_min, const double* output_max,
                                           int64_t* spread_grid, int64_t* fft_grid,
                                           double* input_offset, double* output_offset,
                                           double* gamma, double* h);
NNB_API NeonufftError nnb_deconv_factors(double tol, double upsampfac, NnbPrecision precision,
                                         int64_t nf, double* out);

/* ---------------------------------------------------------------------------------------
 * Batched execution of many independent type-1 / type-2 transforms of uneven sizes.
 * No counterpart in the reference, which runs one plan at a time; this is the engine's
 * batch entry point (one plan per transform, spread over internal streams by estimated cost).
 * ------------------------------------------------------------------------------------- */
typedef struct NnbBatch_s* NnbBatch;

typedef enum NnbBatchMode {
  NNB_BATCH_SERIAL = 0,      /* one transform after the other */
  NNB_BATCH_STREAMS = 1,     /* the internal streams run concurrently */
  NNB_BATCH_GRAPH = 2,       /* the concurrent launch sequence captured once in a CUDA graph */
  NNB_BATCH_FUSED = 3,       /* as STREAMS, but the z-window spreading (type 1) and interpolation
                                (type 2) steps of all 3D transforms that share a kernel shape run
                                as one persistent launch over a queue of all their work items */
  NNB_BATCH_FUSED_GRAPH = 4  /* FUSED captured once in a CUDA graph */
} NnbBatchMode;

/* Creates an empty batch with default options `opt` (NULL = defaults), num_streams in [1, 64]
 * internal streams, forked from and joined into `stream`. */
NNB_API NeonufftError nnb_batch_create(NnbBatch* batch, NnbPrecision precision,
                                       const NnbOptions* opt, int num_streams, void* stream,
                                       const NnbAllocator* alloc);

/* Adds a type-1 (type = 1: in = strengths, out = modes with `strides`) or type-2 (type = 2:
 * in = modes with `strides`, out = values at the points) transform and bins its points
 * (synchronising its stream). `opt` overrides the batch options for this transform (NULL =
 * the batch's). The input and output pointers are kept: every execution reads and writes the
 * same buffers. *index receives the transform's index (may be NULL). */
NNB_API NeonufftError nnb_batch_add(NnbBatch batch, int dim, int type, int sign, int64_t num_nu,
                                    const void* const* loc, const int64_t* modes,
                                    const void* in, void* out, const int64_t* strides,
                                    const NnbOptions* opt, int64_t* index);

/* Runs every transform of the batch on the batch stream (mode: NnbBatchMode). Asynchronous. */
NNB_API NeonufftError nnb_batch_execute(NnbBatch batch, int mode);

/* Number of transforms; information on transform `index`. */
NNB_API NeonufftError nnb_batch_size(NnbBatch batch, int64_t* count);
NNB_API NeonufftError nnb_batch_info(NnbBatch batch, int64_t index, NnbPlanInfo* info);

/* Waits for the batch's work and frees it. */
NNB_API NeonufftError nnb_batch_destroy(NnbBatch batch);

/* ---------------------------------------------------------------------------------------
 * Multilayer perceptron of the learned cost model (FP32, device pointers, asynchronous on
 * `stream`). No counterpart in the reference: the engine's tuner predicts run times of
 * transform configurations with it. n_layers weight layers, widths[0..n_layers]; hidden layers
 * tanh, output linear; parameters per layer: W (widths[l] x widths[l-1], row-major) then b.
 * acts / dacts hold sum_{l>=1} widths[l] * batch floats (the output is the last block).
 * ------------------------------------------------------------------------------------- */
NNB_API NeonufftError nnb_mlp_param_count(int n_layers, const int* widths, int64_t* count);
NNB_API NeonufftError nnb_mlp_forward(int n_layers, const int* widths, const float* params,
                                      const float* x, int64_t batch, float* acts, void* stream);
/* On entry the last block of dacts holds dLoss/dOutput; dacts is overwritten. */
NNB_API NeonufftError nnb_mlp_backward(int n_layers, const int* widths, const float* params,
                                       const float* x, const float* acts, float* dacts,
                                       int64_t batch, float* grads, void* stream);
/* dy = 2 (y - target) / n and loss = mean squared error (one float). */
NNB_API NeonufftError nnb_mlp_mse(const float* y, const float* target, int64_t n, float* dy,
                                  float* loss, void* stream);
NNB_API NeonufftError nnb_mlp_adam(int64_t n, float* params, const float* grads, float* m,
                                   float* v, float lr, float beta1, float beta2, float eps,
                                   int64_t step, void* stream);

/* Library version string. */
/* 1 for the bounds-checked debugging build (libneonufft_b200_checked.so, compiled with
 * -DNNB_CHECKED: device bounds checks on the hot kernels' grid, record and output indices, and a
 * device synchronisation after every call that reports a failed check as
 * NEONUFFT_INTERNAL_ERROR), 0 for the normal build. Engine extension; the reference's
 * counterpart is its debug-build sync-and-check after each launch
 * (src/neonufft/gpu/util/runtime.hpp:27-30). */
NNB_API int nnb_is_checked_build(void);

/* Synchronises the current device and reads the engine's device status: NEONUFFT_GPU_ERROR (with
 * a message) if a bounded wait inside an engine kernel gave up since the last call -- the
 * tensor-core spreading (spread method 5) waits at most 2 s for its matrix products, then
 * abandons the work item, frees its tensor memory and records the failure here instead of
 * hanging -- else NEONUFFT_SUCCESS. The status is cleared by the call. Engine extension; the
 * reference has no device-side waits. */
NNB_API NeonufftError nnb_check_device_status(void);
NNB_API const char* nnb_version(void);

/* Number of engine kernels this process has launched so far (all plans and devices; cuFFT's
 * kernels are not counted). Engine extension for launch accounting. */
NNB_API int64_t nnb_kernel_launches(void);

#ifdef __cplusplus
}  /* extern "C" */
#endif

#endif /* NEONUFFT_GPU_H */
