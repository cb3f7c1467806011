// GPU plans, source-compatible with the reference (include/neonufft/gpu/plan.hpp:25-82).
//
// Header-only shims over the engine's C ABI (neonufft_gpu.h): each method forwards to one
// extern "C" entry point and converts a returned NeonufftError into the matching exception of
// <neonufft/exceptions.hpp>. Explicitly usable for T in {float, double} and DIM in {1, 2, 3},
// like the reference's explicit instantiations (src/neonufft/gpu/plan.cpp:47-53, :115-121).
#pragma once

#include <neonufft/allocator.hpp>
#include <neonufft/enums.h>
#include <neonufft/exceptions.hpp>
#include <neonufft/gpu/device_allocator.hpp>
#include <neonufft/gpu/types.hpp>
#include <neonufft/plan.hpp>
#include <neonufft/types.hpp>
#include <neonufft_gpu.h>

#include <array>
#include <cstddef>
#include <cstdint>
#include <memory>
#include <type_traits>
#include <utility>

namespace neonufft {
namespace gpu {

namespace detail {

inline void check(NeonufftError err) {
  if (err == NEONUFFT_SUCCESS) return;
  const char* msg = nnb_last_error_message();
  switch (err) {
    case NEONUFFT_INPUT_ERROR: throw InputError(msg);
    case NEONUFFT_MEMORY_ALLOC_ERROR: throw MemoryAllocError(msg);
    case NEONUFFT_INTERNAL_ERROR: throw InternalError(msg);
    case NEONUFFT_GPU_ERROR: throw GPUError(msg);
    case NEONUFFT_NOT_IMPLEMENTED_ERROR: throw NotImplementedError(msg);
    default: throw GenericError(msg);
  }
}

inline NnbOptions to_c(const Options& o) {
  NnbOptions c;
  nnb_options_default(&c);
  c.tol = o.tol;
  c.upsampfac = o.upsampfac;
  c.recenter_threshold = o.recenter_threshold;
  c.num_threads = o.num_threads;
  c.sort_input = o.sort_input;
  c.sort_output = o.sort_output;
  c.kernel_approximation = o.kernel_approximation;
  c.order = static_cast<int>(o.order);
  c.kernel_type = static_cast<int>(o.kernel_type);
  return c;
}

inline void* alloc_cb(void* ctx, std::size_t size) {
  try {
    return static_cast<Allocator*>(ctx)->allocate(size);
  } catch (...) {
    return nullptr;
  }
}
inline void dealloc_cb(void* ctx, void* ptr) { static_cast<Allocator*>(ctx)->deallocate(ptr); }

inline NnbAllocator to_c(Allocator* a) { return NnbAllocator{&alloc_cb, &dealloc_cb, a}; }

template <typename T>
constexpr NnbPrecision precision() {
  return std::is_same_v<T, float> ? NNB_FLOAT : NNB_DOUBLE;
}

}  // namespace detail

template <typename T, std::size_t DIM>
class Plan {
public:
  static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>);
  static_assert(DIM == 1 || DIM == 2 || DIM == 3);

  Plan(Options opt, int sign, IntType num_nu, std::array<const T*, DIM> loc,
       std::array<IntType, DIM> modes, StreamType stream,
       std::shared_ptr<Allocator> device_alloc = std::make_shared<DeviceAllocator>())
      : alloc_(std::move(device_alloc)), impl_(nullptr, &nnb_plan_destroy) {
    const NnbOptions c_opt = detail::to_c(opt);
    const NnbAllocator c_alloc = detail::to_c(alloc_.get());
    const void* c_loc[DIM];
    std::int64_t c_modes[DIM];
    for (std::size_t d = 0; d < DIM; ++d) {
      c_loc[d] = loc[d];
      c_modes[d] = modes[d];
    }
    NnbPlan p = nullptr;
    detail::check(nnb_plan_create(&p, detail::precision<T>(), int(DIM), &c_opt, sign, num_nu,
                                  c_loc, c_modes, stream, alloc_ ? &c_alloc : nullptr));
    impl_.reset(p);
  }

  void transform_type_1(const ComplexType<T>* in, ComplexType<T>* out,
                        std::array<IntType, DIM> out_strides) {
    std::int64_t s[DIM];
    for (std::size_t d = 0; d < DIM; ++d) s[d] = out_strides[d];
    detail::check(nnb_plan_transform_type_1(impl_.get(), in, out, s));
  }

  void transform_type_2(const ComplexType<T>* in, std::array<IntType, DIM> in_strides,
                        ComplexType<T>* out) {
    std::int64_t s[DIM];
    for (std::size_t d = 0; d < DIM; ++d) s[d] = in_strides[d];
    detail::check(nnb_plan_transform_type_2(impl_.get(), in, s, out));
  }

  void set_points(IntType num_nu, std::array<const T*, DIM> loc) {
    const void* c_loc[DIM];
    for (std::size_t d = 0; d < DIM; ++d) c_loc[d] = loc[d];
    detail::check(nnb_plan_set_points(impl_.get(), num_nu, c_loc));
  }

  // Engine extension: the C handle, for nnb_plan_info / nnb_plan_stage_times.
  NnbPlan native_handle() const { return impl_.get(); }

private:
  std::shared_ptr<Allocator> alloc_;  // destroyed after impl_
  std::unique_ptr<NnbPlan_s, NeonufftError (*)(NnbPlan)> impl_;
};

template <typename T, std::size_t DIM>
class PlanT3 {
public:
  static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>);
  static_assert(DIM == 1 || DIM == 2 || DIM == 3);

  static std::uint64_t grid_memory_size(const Options& opt, std::array<T, DIM> input_min,
                                        std::array<T, DIM> input_max,
                                        std::array<T, DIM> output_min,
                                        std::array<T, DIM> output_max) {
    const NnbOptions c_opt = detail::to_c(opt);
    double a[DIM], b[DIM], c[DIM], e[DIM];
    for (std::size_t d = 0; d < DIM; ++d) {
      a[d] = input_min[d];
      b[d] = input_max[d];
      c[d] = output_min[d];
      e[d] = output_max[d];
    }
    std::uint64_t size = 0;
    detail::check(nnb_plan_t3_grid_memory_size(detail::precision<T>(), int(DIM), &c_opt, a, b, c,
                                               e, &size));
    return size;
  }

  PlanT3(Options opt, int sign, IntType num_in, std::array<const T*, DIM> input_points,
         IntType num_out, std::array<const T*, DIM> output_points, StreamType stream,
         IntType batch_size = 1,
         std::shared_ptr<Allocator> device_alloc = std::make_shared<DeviceAllocator>())
      : alloc_(std::move(device_alloc)), impl_(nullptr, &nnb_plan_t3_destroy) {
    const NnbOptions c_opt = detail::to_c(opt);
    const NnbAllocator c_alloc = detail::to_c(alloc_.get());
    const void* in_p[DIM];
    const void* out_p[DIM];
    for (std::size_t d = 0; d < DIM; ++d) {
      in_p[d] = input_points[d];
      out_p[d] = output_points[d];
    }
    NnbPlanT3 p = nullptr;
    detail::check(nnb_plan_t3_create(&p, detail::precision<T>(), int(DIM), &c_opt, sign, num_in,
                                     in_p, num_out, out_p, stream, batch_size,
                                     alloc_ ? &c_alloc : nullptr));
    impl_.reset(p);
  }

  PlanT3(Options opt, int sign, std::array<T, DIM> input_min, std::array<T, DIM> input_max,
         std::array<T, DIM> output_min, std::array<T, DIM> output_max, StreamType stream,
         IntType batch_size = 1,
         std::shared_ptr<Allocator> device_alloc = std::make_shared<DeviceAllocator>())
      : alloc_(std::move(device_alloc)), impl_(nullptr, &nnb_plan_t3_destroy) {
    const NnbOptions c_opt = detail::to_c(opt);
    const NnbAllocator c_alloc = detail::to_c(alloc_.get());
    double a[DIM], b[DIM], c[DIM], e[DIM];
    for (std::size_t d = 0; d < DIM; ++d) {
      a[d] = input_min[d];
      b[d] = input_max[d];
      c[d] = output_min[d];
      e[d] = output_max[d];
    }
    NnbPlanT3 p = nullptr;
    detail::check(nnb_plan_t3_create_bounds(&p, detail::precision<T>(), int(DIM), &c_opt, sign,
                                            a, b, c, e, stream, batch_size,
                                            alloc_ ? &c_alloc : nullptr));
    impl_.reset(p);
  }

  void set_input_points(IntType num_in, std::array<const T*, DIM> input_points) {
    const void* p[DIM];
    for (std::size_t d = 0; d < DIM; ++d) p[d] = input_points[d];
    detail::check(nnb_plan_t3_set_input_points(impl_.get(), num_in, p));
  }

  void set_output_points(IntType num_out, std::array<const T*, DIM> output_points) {
    const void* p[DIM];
    for (std::size_t d = 0; d < DIM; ++d) p[d] = output_points[d];
    detail::check(nnb_plan_t3_set_output_points(impl_.get(), num_out, p));
  }

  void add_input(const ComplexType<T>* in, IntType bdist = 0) {
    detail::check(nnb_plan_t3_add_input(impl_.get(), in, bdist));
  }

  void transform(ComplexType<T>* out, IntType bdist = 0) {
    detail::check(nnb_plan_t3_transform(impl_.get(), out, bdist));
  }

  void reset() { detail::check(nnb_plan_t3_reset(impl_.get())); }

  NnbPlanT3 native_handle() const { return impl_.get(); }

private:
  std::shared_ptr<Allocator> alloc_;  // destroyed after impl_
  std::unique_ptr<NnbPlanT3_s, NeonufftError (*)(NnbPlanT3)> impl_;
};

}  // namespace gpu
}  // namespace neonufft
