// extern "C" entry points (declared in include/neonufft_gpu.h). Each one runs its body under
// a guard that converts the engine's exceptions (the reference's hierarchy,
// include/neonufft/exceptions.hpp) into NeonufftError codes and records the message.
#include <new>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "neonufft_gpu.h"
#include "batch.hpp"
#include "plan.hpp"

struct NnbBatch_s {
  std::unique_ptr<nnb::Batch> impl;
};
struct NnbPlan_s {
  std::unique_ptr<nnb::PlanBase> impl;
};
struct NnbPlanT3_s {
  std::unique_ptr<nnb::PlanT3Base> impl;
};

namespace {

thread_local std::string t_last_error;

template <typename F>
NeonufftError guard(F&& f) noexcept {
  try {
    f();
    nnb::check_device_records();  // checked build only: synchronise, report failed checks
    return NEONUFFT_SUCCESS;
  } catch (const neonufft::GenericError& e) {
    t_last_error = e.what();
    return e.error_code();
  } catch (const std::bad_alloc&) {
    t_last_error = "Neonufft:: host memory allocation failed";
    return NEONUFFT_MEMORY_ALLOC_ERROR;
  } catch (const std::exception& e) {
    t_last_error = e.what();
    return NEONUFFT_UNKNOWN_ERROR;
  } catch (...) {
    t_last_error = "Neonufft:: unknown error";
    return NEONUFFT_UNKNOWN_ERROR;
  }
}

NnbOptions opts_or_default(const NnbOptions* opt) {
  NnbOptions o;
  if (opt) {
    o = *opt;
  } else {
    nnb_options_default(&o);
  }
  return o;
}

void need(const void* p, const char* what) {
  if (!p) nnb::throw_input(std::string("null ") + what);
}

}  // namespace

extern "C" {

void nnb_options_default(NnbOptions* opt) {
  if (!opt) return;
  *opt = NnbOptions{};
  opt->tol = 0.001;
  opt->upsampfac = 2.0;
  opt->recenter_threshold = 0.1;
  opt->num_threads = 0;
  opt->sort_input = 1;
  opt->sort_output = 1;
  opt->kernel_approximation = 0;
  opt->order = NEONUFFT_MODE_ORDER_CMCL;
  opt->kernel_type = NEONUFFT_ES_KERNEL;
}

const char* nnb_last_error_message(void) { return t_last_error.c_str(); }

NeonufftError nnb_batch_create(NnbBatch* batch, NnbPrecision precision, const NnbOptions* opt,
                               int num_streams, void* stream, const NnbAllocator* alloc) {
  return guard([&] {
    need(batch, "batch handle");
    *batch = nullptr;
    auto b = std::make_unique<NnbBatch_s>();
    b->impl = std::make_unique<nnb::Batch>(precision, opts_or_default(opt), num_streams,
                                           static_cast<cudaStream_t>(stream), alloc);
    *batch = b.release();
  });
}

NeonufftError nnb_batch_add(NnbBatch batch, int dim, int type, int sign, int64_t num_nu,
                            const void* const* loc, const int64_t* modes, const void* in,
                            void* out, const int64_t* strides, const NnbOptions* opt,
                            int64_t* index) {
  return guard([&] {
    need(batch, "batch");
    const int64_t i =
        batch->impl->add(dim, type, sign, num_nu, loc, modes, in, out, strides, opt);
    if (index) *index = i;
  });
}

NeonufftError nnb_batch_execute(NnbBatch batch, int mode) {
  return guard([&] {
    need(batch, "batch");
    batch->impl->execute(mode);
  });
}

NeonufftError nnb_batch_size(NnbBatch batch, int64_t* count) {
  return guard([&] {
    need(batch, "batch");
    need(count, "count");
    *count = batch->impl->size();
  });
}

NeonufftError nnb_batch_info(NnbBatch batch, int64_t index, NnbPlanInfo* info) {
  return guard([&] {
    need(batch, "batch");
    need(info, "info");
    batch->impl->plan(index).info(info);
  });
}

NeonufftError nnb_batch_destroy(NnbBatch batch) {
  return guard([&] { delete batch; });
}

NeonufftError nnb_mlp_param_count(int n_layers, const int* widths, int64_t* count) {
  return guard([&] {
    need(count, "count");
    *count = nnb::mlp_param_count(n_layers, widths);
  });
}

NeonufftError nnb_mlp_forward(int n_layers, const int* widths, const float* params,
                              const float* x, int64_t batch, float* acts, void* stream) {
  return guard([&] {
    need(params, "params");
    need(acts, "activations");
    if (batch > 0) need(x, "inputs");
    nnb::mlp_forward(n_layers, widths, params, x, batch, acts, static_cast<cudaStream_t>(stream));
  });
}

NeonufftError nnb_mlp_backward(int n_layers, const int* widths, const float* params,
                               const float* x, const float* acts, float* dacts, int64_t batch,
                               float* grads, void* stream) {
  return guard([&] {
    need(params, "params");
    need(acts, "activations");
    need(dacts, "activation gradients");
    need(grads, "gradients");
    if (batch > 0) need(x, "inputs");
    nnb::mlp_backward(n_layers, widths, params, x, acts, dacts, batch, grads,
                      static_cast<cudaStream_t>(stream));
  });
}

NeonufftError nnb_mlp_mse(const float* y, const float* target, int64_t n, float* dy, float* loss,
                          void* stream) {
  return guard([&] {
    need(y, "outputs");
    need(target, "targets");
    need(dy, "output gradients");
    need(loss, "loss");
    nnb::mlp_mse(y, target, n, dy, loss, static_cast<cudaStream_t>(stream));
  });
}

NeonufftError nnb_mlp_adam(int64_t n, float* params, const float* grads, float* m, float* v,
                           float lr, float beta1, float beta2, float eps, int64_t step,
                           void* stream) {
  return guard([&] {
    need(params, "params");
    need(grads, "gradients");
    need(m, "first moments");
    need(v, "second moments");
    nnb::mlp_adam(n, params, grads, m, v, lr, beta1, beta2, eps, step,
                  static_cast<cudaStream_t>(stream));
  });
}

const char* nnb_version(void) { return "neonufft_b200 0.1.0 (sm_100a)"; }

int64_t nnb_kernel_launches(void) { return nnb::g_kernel_launches.load(); }

NeonufftError nnb_check_device_status(void) {
  return guard([&] {
    NNB_CUDA(cudaDeviceSynchronize());
    if (nnb::read_tc_status(true)) {
      throw neonufft::GPUError(
          "Neonufft:: tensor-core spreading: a bounded wait for the matrix products gave up");
    }
  });
}

int nnb_is_checked_build(void) {
#ifdef NNB_CHECKED
  return 1;
#else
  return 0;
#endif
}

NeonufftError nnb_device_alloc(void** ptr, size_t size) {
  return guard([&] {
    need(ptr, "pointer");
    *ptr = nullptr;
    if (size == 0) return;
    NNB_CUDA(cudaMalloc(ptr, size));
  });
}

NeonufftError nnb_device_free(void* ptr) {
  return guard([&] {
    if (ptr) NNB_CUDA(cudaFree(ptr));
  });
}

NeonufftError nnb_plan_create(NnbPlan* plan, NnbPrecision precision, int dim,
                              const NnbOptions* opt, int sign, int64_t num_nu,
                              const void* const* loc, const int64_t* modes, void* stream,
                              const NnbAllocator* alloc) {
  return guard([&] {
    need(plan, "plan handle");
    *plan = nullptr;
    auto p = std::make_unique<NnbPlan_s>();
    p->impl = nnb::make_plan(precision, dim, opts_or_default(opt), sign, num_nu, loc, modes,
                             static_cast<cudaStream_t>(stream), alloc);
    *plan = p.release();
  });
}

NeonufftError nnb_plan_set_points(NnbPlan plan, int64_t num_nu, const void* const* loc) {
  return guard([&] {
    need(plan, "plan");
    plan->impl->set_points(num_nu, loc);
  });
}

NeonufftError nnb_plan_transform_type_1(NnbPlan plan, const void* in, void* out,
                                        const int64_t* out_strides) {
  return guard([&] {
    need(plan, "plan");
    plan->impl->transform_type_1(in, out, out_strides);
  });
}

NeonufftError nnb_plan_transform_type_1_many(NnbPlan plan, int64_t count, const void* in,
                                             int64_t in_bdist, void* out, int64_t out_bdist,
                                             const int64_t* out_strides) {
  return guard([&] {
    need(plan, "plan");
    plan->impl->transform_type_1_many(count, in, in_bdist, out, out_bdist, out_strides);
  });
}

NeonufftError nnb_plan_transform_type_2(NnbPlan plan, const void* in, const int64_t* in_strides,
                                        void* out) {
  return guard([&] {
    need(plan, "plan");
    plan->impl->transform_type_2(in, in_strides, out);
  });
}

NeonufftError nnb_plan_destroy(NnbPlan plan) {
  return guard([&] { delete plan; });
}

NeonufftError nnb_plan_info(NnbPlan plan, NnbPlanInfo* info) {
  return guard([&] {
    need(plan, "plan");
    need(info, "info");
    plan->impl->info(info);
  });
}

NeonufftError nnb_plan_enable_timing(NnbPlan plan, int enable) {
  return guard([&] {
    need(plan, "plan");
    plan->impl->timer().enable(enable != 0);
  });
}

NeonufftError nnb_plan_stage_times(NnbPlan plan, double* ms, int64_t* count, int reset) {
  return guard([&] {
    need(plan, "plan");
    plan->impl->timer().collect(plan->impl->stream(), ms, count, reset != 0);
  });
}

NeonufftError nnb_plan_t3_grid_memory_size(NnbPrecision precision, int dim, const NnbOptions* opt,
                                           const double* input_min, const double* input_max,
                                           const double* output_min, const double* output_max,
                                           uint64_t* size) {
  return guard([&] {
    need(size, "size");
    *size = nnb::t3_grid_memory_size(precision, dim, opts_or_default(opt), input_min, input_max,
                                     output_min, output_max);
  });
}

NeonufftError nnb_plan_t3_create(NnbPlanT3* plan, NnbPrecision precision, int dim,
                                 const NnbOptions* opt, int sign, int64_t num_in,
                                 const void* const* input_points, int64_t num_out,
                                 const void* const* output_points, void* stream,
                                 int64_t batch_size, const NnbAllocator* alloc) {
  return guard([&] {
    need(plan, "plan handle");
    *plan = nullptr;
    auto p = std::make_unique<NnbPlanT3_s>();
    p->impl = nnb::make_plan_t3(precision, dim, opts_or_default(opt), sign, num_in, input_points,
                                num_out, output_points, static_cast<cudaStream_t>(stream),
                                batch_size, alloc);
    *plan = p.release();
  });
}

NeonufftError nnb_plan_t3_create_bounds(NnbPlanT3* plan, NnbPrecision precision, int dim,
                                        const NnbOptions* opt, int sign, const double* input_min,
                                        const double* input_max, const double* output_min,
                                        const double* output_max, void* stream,
                                        int64_t batch_size, const NnbAllocator* alloc) {
  return guard([&] {
    need(plan, "plan handle");
    *plan = nullptr;
    auto p = std::make_unique<NnbPlanT3_s>();
    p->impl = nnb::make_plan_t3_bounds(precision, dim, opts_or_default(opt), sign, input_min,
                                       input_max, output_min, output_max,
                                       static_cast<cudaStream_t>(stream), batch_size, alloc);
    *plan = p.release();
  });
}

NeonufftError nnb_plan_t3_set_input_points(NnbPlanT3 plan, int64_t num_in,
                                           const void* const* input_points) {
  return guard([&] {
    need(plan, "plan");
    plan->impl->set_input_points(num_in, input_points);
  });
}

NeonufftError nnb_plan_t3_set_output_points(NnbPlanT3 plan, int64_t num_out,
                                            const void* const* output_points) {
  return guard([&] {
    need(plan, "plan");
    plan->impl->set_output_points(num_out, output_points);
  });
}

NeonufftError nnb_plan_t3_add_input(NnbPlanT3 plan, const void* in, int64_t bdist) {
  return guard([&] {
    need(plan, "plan");
    plan->impl->add_input(in, bdist);
  });
}

NeonufftError nnb_plan_t3_transform(NnbPlanT3 plan, void* out, int64_t bdist) {
  return guard([&] {
    need(plan, "plan");
    plan->impl->transform(out, bdist);
  });
}

NeonufftError nnb_plan_t3_reset(NnbPlanT3 plan) {
  return guard([&] {
    need(plan, "plan");
    plan->impl->reset();
  });
}

NeonufftError nnb_plan_t3_destroy(NnbPlanT3 plan) {
  return guard([&] { delete plan; });
}

NeonufftError nnb_plan_t3_info(NnbPlanT3 plan, NnbPlanInfo* info) {
  return guard([&] {
    need(plan, "plan");
    need(info, "info");
    plan->impl->info(info);
  });
}

NeonufftError nnb_plan_t3_enable_timing(NnbPlanT3 plan, int enable) {
  return guard([&] {
    need(plan, "plan");
    plan->impl->timer().enable(enable != 0);
  });
}

NeonufftError nnb_plan_t3_stage_times(NnbPlanT3 plan, double* ms, int64_t* count, int reset) {
  return guard([&] {
    need(plan, "plan");
    plan->impl->timer().collect(plan->impl->stream(), ms, count, reset != 0);
  });
}

NeonufftError nnb_es_kernel_params(double tol, double upsampfac, NnbPrecision precision,
                                   int* n_spread, double* beta, double* c) {
  return guard([&] {
    NnbOptions o;
    nnb_options_default(&o);
    o.tol = tol;
    o.upsampfac = upsampfac;
    nnb::validate_options(o);
    const nnb::KernelParam kp = nnb::kernel_param(tol, upsampfac, precision == NNB_FLOAT);
    if (n_spread) *n_spread = kp.w;
    if (beta) *beta = kp.beta;
    if (c) *c = kp.c;
  });
}

NeonufftError nnb_plan_t3_geometry(NnbPrecision precision, int dim, const NnbOptions* opt,
                                   const double* input_min, const double* input_max,
                                   const double* output_min, const double* output_max,
                                   int64_t* spread_grid, int64_t* fft_grid, double* input_offset,
                                   double* output_offset, double* gamma, double* h) {
  return guard([&] {
    const NnbOptions o = opts_or_default(opt);
    nnb::validate_options(o);
    if (dim < 1 || dim > 3) nnb::throw_input("dimension must be 1, 2 or 3");
    need(input_min, "bounds");
    need(input_max, "bounds");
    need(output_min, "bounds");
    need(output_max, "bounds");
    const bool single = precision == NNB_FLOAT;
    const nnb::KernelParam kp = nnb::kernel_param(o.tol, o.upsampfac, single, o.n_spread);
    for (int d = 0; d < dim; ++d) {
      int64_t nf1, nfft;
      double C, D, g, hh;
      if (single) {
        const auto r = nnb::t3_geometry<float>(kp.w, o.upsampfac, float(o.recenter_threshold),
                                               float(input_min[d]), float(input_max[d]),
                                               float(output_min[d]), float(output_max[d]));
        nf1 = r.spread_grid; nfft = r.fft_grid; C = r.input_offset; D = r.output_offset;
        g = r.gamma; hh = r.h;
      } else {
        const auto r = nnb::t3_geometry<double>(kp.w, o.upsampfac, o.recenter_threshold,
                                                input_min[d], input_max[d], output_min[d],
                                                output_max[d]);
        nf1 = r.spread_grid; nfft = r.fft_grid; C = r.input_offset; D = r.output_offset;
        g = r.gamma; hh = r.h;
      }
      if (spread_grid) spread_grid[d] = nf1;
      if (fft_grid) fft_grid[d] = nfft;
      if (input_offset) input_offset[d] = C;
      if (output_offset) output_offset[d] = D;
      if (gamma) gamma[d] = g;
      if (h) h[d] = hh;
    }
  });
}

NeonufftError nnb_deconv_factors(double tol, double upsampfac, NnbPrecision precision, int64_t nf,
                                 double* out) {
  return guard([&] {
    need(out, "output");
    if (nf < 1) nnb::throw_input("grid size must be positive");
    const nnb::KernelParam kp = nnb::kernel_param(tol, upsampfac, precision == NNB_FLOAT);
    const std::vector<double> f = nnb::deconv_factors(kp, nf);
    for (size_t i = 0; i < f.size(); ++i) out[i] = f[i];
  });
}

NeonufftError nnb_direct_type1_f64(int dim, int sign, int64_t num_nu, const double* const* loc,
                                   const double* in, int64_t num_samples, const int64_t* modes_idx,
                                   double* out, void* stream) {
  return guard([&] {
    if (dim < 1 || dim > 3) nnb::throw_input("dimension must be 1, 2 or 3");
    need(out, "output");
    if (num_samples > 0) need(modes_idx, "mode indices");
    if (num_nu > 0) {
      need(loc, "coordinates");
      need(in, "input");
    }
    nnb::launch_direct_type1(dim, sign < 0 ? -1 : 1, num_nu, loc, in, num_samples, modes_idx,
                             out, static_cast<cudaStream_t>(stream));
  });
}

NeonufftError nnb_direct_type1_f64_noalloc(int dim, int sign, int64_t num_nu,
                                           const double* const* loc, const double* in,
                                           int64_t num_samples, const int64_t* modes_idx,
                                           double* out, void* stream) {
  return guard([&] {
    if (dim < 1 || dim > 3) nnb::throw_input("dimension must be 1, 2 or 3");
    if (num_nu < 0 || num_samples < 0) nnb::throw_input("negative size");
    need(out, "output");
    if (num_samples > 0) need(modes_idx, "mode indices");
    if (num_nu > 0) {
      need(loc, "coordinates");
      need(in, "input");
    }
    nnb::launch_direct_type1_noalloc(dim, sign < 0 ? -1 : 1, num_nu, loc, in, num_samples,
                                     modes_idx, out, static_cast<cudaStream_t>(stream));
  });
}

NeonufftError nnb_direct_type2_f64(int dim, int sign, const int64_t* n_modes, const double* in,
                                   const double* const* loc, int64_t num_samples,
                                   const int64_t* point_idx, double* out, void* stream) {
  return guard([&] {
    if (dim < 1 || dim > 3) nnb::throw_input("dimension must be 1, 2 or 3");
    need(n_modes, "modes");
    need(in, "input");
    need(out, "output");
    if (num_samples > 0) {
      need(loc, "coordinates");
      need(point_idx, "point indices");
    }
    nnb::launch_direct_type2(dim, sign < 0 ? -1 : 1, n_modes, in, loc, num_samples, point_idx,
                             out, static_cast<cudaStream_t>(stream));
  });
}

NeonufftError nnb_direct_type3_f64(int dim, int sign, int64_t num_in, const double* const* in_loc,
                                   const double* in, const double* const* out_loc,
                                   int64_t num_samples, const int64_t* target_idx, double* out,
                                   void* stream) {
  return guard([&] {
    if (dim < 1 || dim > 3) nnb::throw_input("dimension must be 1, 2 or 3");
    need(out, "output");
    if (num_in > 0) {
      need(in_loc, "input coordinates");
      need(in, "input");
    }
    if (num_samples > 0) {
      need(out_loc, "output coordinates");
      need(target_idx, "target indices");
    }
    nnb::launch_direct_type3(dim, sign < 0 ? -1 : 1, num_in, in_loc, in, out_loc, num_samples,
                             target_idx, out, static_cast<cudaStream_t>(stream));
  });
}

}  // extern "C"
