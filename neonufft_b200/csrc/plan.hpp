// Plan implementations behind the C ABI.
//
// PlanImpl<T> follows the reference GPU type-1/2 plan (src/neonufft/gpu/plan_impl.hpp:41-152);
// PlanT3Impl<T> follows the reference GPU type-3 plan (src/neonufft/gpu/plan_t3_impl.hpp:54-306).
// The step sequence and the results are the reference's; the kernels, the data layout and the
// precision choices are the engine's own (see the kernel files).
#pragma once

#include <memory>

#include "runtime.hpp"

namespace nnb {

class PlanBase {
public:
  virtual ~PlanBase() = default;
  virtual void set_points(i64 M, const void* const* loc) = 0;
  virtual void transform_type_1(const void* in, void* out, const i64* out_strides) = 0;
  virtual void transform_type_2(const void* in, const i64* in_strides, void* out) = 0;
  // `count` type-1 transforms of the plan's points: input vector v at in + v in_bdist, output
  // v at out + v out_bdist (elements). The base runs them one at a time.
  virtual void transform_type_1_many(i64 count, const void* in, i64 in_bdist, void* out,
                                     i64 out_bdist, const i64* out_strides);
  virtual void info(NnbPlanInfo* info) const = 0;
  virtual StageTimer& timer() = 0;
  virtual cudaStream_t stream() const = 0;

  // Hooks for persistent batched execution (batch.cu): a plan whose spreading or interpolation
  // runs on the z-window kernels can leave that step of a transform to one persistent launch
  // over many plans. fused_key is false if the plan cannot, else a key that is equal for plans
  // one launch can serve (precision aside: a batch has one).
  virtual bool fused_key(int* key) const {
    (void)key;
    return false;
  }
  // Host description of the step of transform `type` (a ZSpreadJob<T> or ZInterpJob<T>).
  virtual void fused_job(int type, const void* in, void* out, void* job) const;
  // Work before the step, on the plan's stream: type 1 clears the fine grid; type 2 deconvolves
  // `in` into it and transforms it; both build the step's work list.
  virtual void fused_pre(int type, const void* in, const i64* strides);
  // Work after the step, on the plan's stream: type 1 transforms and deconvolves into `out`.
  virtual void fused_post(int type, void* out, const i64* strides);
};

class PlanT3Base {
public:
  virtual ~PlanT3Base() = default;
  virtual void set_input_points(i64 M, const void* const* pts) = 0;
  virtual void set_output_points(i64 K, const void* const* pts) = 0;
  virtual void add_input(const void* in, i64 bdist) = 0;
  virtual void transform(void* out, i64 bdist) = 0;
  virtual void reset() = 0;
  virtual void info(NnbPlanInfo* info) const = 0;
  virtual StageTimer& timer() = 0;
  virtual cudaStream_t stream() const = 0;
};

std::unique_ptr<PlanBase> make_plan(NnbPrecision prec, int dim, const NnbOptions& opt, int sign,
                                    i64 M, const void* const* loc, const i64* modes,
                                    cudaStream_t stream, const NnbAllocator* alloc);

std::unique_ptr<PlanT3Base> make_plan_t3(NnbPrecision prec, int dim, const NnbOptions& opt,
                                         int sign, i64 M, const void* const* in_pts, i64 K,
                                         const void* const* out_pts, cudaStream_t stream,
                                         i64 batch, const NnbAllocator* alloc);

std::unique_ptr<PlanT3Base> make_plan_t3_bounds(NnbPrecision prec, int dim,
                                                const NnbOptions& opt, int sign,
                                                const double* in_min, const double* in_max,
                                                const double* out_min, const double* out_max,
                                                cudaStream_t stream, i64 batch,
                                                const NnbAllocator* alloc);

u64 t3_grid_memory_size(NnbPrecision prec, int dim, const NnbOptions& opt, const double* in_min,
                        const double* in_max, const double* out_min, const double* out_max);

void validate_options(const NnbOptions& opt);

}  // namespace nnb
