// ORACLE -- test infrastructure only (reference pin). Compiled by oracle/Makefile together with
// the reference's own sources into oracle/_ref/libneonufft_ref.so; nothing of the engine links it.
//
// extern "C" wrappers over the reference's own code, used to pin the engine and the oracle:
//  - parameter heuristics: KernelParameters (src/neonufft/es_kernel_param.hpp:14-57),
//    GridInfoT3 (src/neonufft/util/grid_info_t3.hpp:18-52), set_nhg_type3 / next235even
//    (src/contrib/es_kernel/util.hpp:39-105), legendre_compute_glr
//    (src/contrib/legendre_rule/legendre_rule_fast.cpp:30) -- pure host code;
//  - the reference GPU plans gpu::Plan / gpu::PlanT3 (include/neonufft/gpu/plan.hpp:25-82),
//    built from the reference's CUDA sources for sm_100a, run on device pointers.
#include <array>
#include <cstdint>
#include <exception>
#include <memory>

#include "contrib/es_kernel/util.hpp"
#include "contrib/legendre_rule/legendre_rule_fast.hpp"
#include "neonufft/config.h"
#include "neonufft/es_kernel_param.hpp"
#include "neonufft/exceptions.hpp"
#include "neonufft/gpu/plan.hpp"
#include "neonufft/util/grid_info_t3.hpp"

using neonufft::IntType;

namespace {

template <typename T>
void kparam(double tol, double upsampfac, int* w, double* beta, double* c) {
  neonufft::KernelParameters<T> p(tol, upsampfac, false);
  *w = p.n_spread;
  *beta = double(p.es_beta);
  *c = double(p.es_c);
}

template <typename T>
void t3geo(int w, double upsampfac, double recenter, double in_min, double in_max, double out_min,
           double out_max, double* out, int64_t* grids) {
  std::array<T, 1> a{T(in_min)}, b{T(in_max)}, c{T(out_min)}, d{T(out_max)};
  neonufft::GridInfoT3<T, 1> g(w, upsampfac, T(recenter), a, b, c, d);
  T h = 0, gam = 0;
  neonufft::contrib::set_nhg_type3<T>(g.output_half_extent[0], g.input_half_extent[0],
                                       T(upsampfac), g.spread_grid_size[0], &h, &gam);
  out[0] = double(g.input_offsets[0]);
  out[1] = double(g.output_offsets[0]);
  out[2] = double(g.input_half_extent[0]);
  out[3] = double(g.output_half_extent[0]);
  out[4] = double(h);
  out[5] = double(gam);
  grids[0] = g.spread_grid_size[0];
  grids[1] = g.fft_grid_size[0];
}

template <typename T, std::size_t D>
void run12(int type, const neonufft::Options& opt, int sign, int64_t M, const void* const* loc,
           const int64_t* modes, const void* in, void* out, const int64_t* strides) {
  std::array<const T*, D> l;
  std::array<IntType, D> m, s;
  for (std::size_t d = 0; d < D; ++d) {
    l[d] = static_cast<const T*>(loc[d]);
    m[d] = modes[d];
    s[d] = strides[d];
  }
  neonufft::gpu::Plan<T, D> plan(opt, sign, M, l, m, nullptr);
  using CT = neonufft::gpu::ComplexType<T>;
  if (type == 1) {
    plan.transform_type_1(static_cast<const CT*>(in), static_cast<CT*>(out), s);
  } else {
    plan.transform_type_2(static_cast<const CT*>(in), s, static_cast<CT*>(out));
  }
  cudaStreamSynchronize(nullptr);
}

template <typename T, std::size_t D>
void run3(const neonufft::Options& opt, int sign, int64_t M, const void* const* in_pts, int64_t K,
          const void* const* out_pts, int batch, const void* in, void* out) {
  std::array<const T*, D> a, b;
  for (std::size_t d = 0; d < D; ++d) {
    a[d] = static_cast<const T*>(in_pts[d]);
    b[d] = static_cast<const T*>(out_pts[d]);
  }
  neonufft::gpu::PlanT3<T, D> plan(opt, sign, M, a, K, b, nullptr, batch);
  using CT = neonufft::gpu::ComplexType<T>;
  plan.add_input(static_cast<const CT*>(in), M);
  plan.transform(static_cast<CT*>(out), K);
  cudaStreamSynchronize(nullptr);
}

// Persistent reference plan (for timing the reference GPU path without plan creation).
struct RefPlan12Base {
  virtual ~RefPlan12Base() = default;
  virtual void set_points(int64_t M, const void* const* loc) = 0;
  virtual void t1(const void* in, void* out, const int64_t* strides) = 0;
  virtual void t2(const void* in, const int64_t* strides, void* out) = 0;
};

template <typename T, std::size_t D>
struct RefPlan12 final : RefPlan12Base {
  using CT = neonufft::gpu::ComplexType<T>;
  std::unique_ptr<neonufft::gpu::Plan<T, D>> plan;
  RefPlan12(const neonufft::Options& opt, int sign, int64_t M, const void* const* loc,
            const int64_t* modes) {
    std::array<const T*, D> l;
    std::array<IntType, D> m;
    for (std::size_t d = 0; d < D; ++d) {
      l[d] = static_cast<const T*>(loc[d]);
      m[d] = modes[d];
    }
    plan = std::make_unique<neonufft::gpu::Plan<T, D>>(opt, sign, M, l, m, nullptr);
  }
  void set_points(int64_t M, const void* const* loc) override {
    std::array<const T*, D> l;
    for (std::size_t d = 0; d < D; ++d) l[d] = static_cast<const T*>(loc[d]);
    plan->set_points(M, l);
  }
  void t1(const void* in, void* out, const int64_t* strides) override {
    std::array<IntType, D> s;
    for (std::size_t d = 0; d < D; ++d) s[d] = strides[d];
    plan->transform_type_1(static_cast<const CT*>(in), static_cast<CT*>(out), s);
  }
  void t2(const void* in, const int64_t* strides, void* out) override {
    std::array<IntType, D> s;
    for (std::size_t d = 0; d < D; ++d) s[d] = strides[d];
    plan->transform_type_2(static_cast<const CT*>(in), s, static_cast<CT*>(out));
  }
};

int code_of(const std::exception_ptr& e) {
  try {
    std::rethrow_exception(e);
  } catch (const neonufft::GenericError& g) {
    return int(g.error_code());
  } catch (...) {
    return 3;
  }
}

}  // namespace

extern "C" {

__attribute__((visibility("default"))) void ref_kernel_param(double tol, double upsampfac,
                                                             int is_float, int* w, double* beta,
                                                             double* c) {
  if (is_float) {
    kparam<float>(tol, upsampfac, w, beta, c);
  } else {
    kparam<double>(tol, upsampfac, w, beta, c);
  }
}

__attribute__((visibility("default"))) void ref_t3_geometry(int is_float, int w, double upsampfac,
                                                            double recenter, double in_min,
                                                            double in_max, double out_min,
                                                            double out_max, double* out,
                                                            int64_t* grids) {
  if (is_float) {
    t3geo<float>(w, upsampfac, recenter, in_min, in_max, out_min, out_max, out, grids);
  } else {
    t3geo<double>(w, upsampfac, recenter, in_min, in_max, out_min, out_max, out, grids);
  }
}

__attribute__((visibility("default"))) int64_t ref_next235even(int64_t n) {
  return neonufft::contrib::next235even(n);
}

__attribute__((visibility("default"))) void ref_legendre(int n, double* x, double* w) {
  neonufft::contrib::quadrature::legendre_compute_glr(n, x, w);
}

__attribute__((visibility("default"))) int ref_gpu_type12(int is_float, int dim, int type,
                                                          double tol, double upsampfac, int sign,
                                                          int order, int64_t M,
                                                          const void* const* loc,
                                                          const int64_t* modes, const void* in,
                                                          void* out, const int64_t* strides) {
  try {
    neonufft::Options opt;
    opt.tol = tol;
    opt.upsampfac = upsampfac;
    opt.order = order ? NEONUFFT_MODE_ORDER_CMCL : NEONUFFT_MODE_ORDER_FFT;
    if (is_float) {
      if (dim == 1) run12<float, 1>(type, opt, sign, M, loc, modes, in, out, strides);
      if (dim == 2) run12<float, 2>(type, opt, sign, M, loc, modes, in, out, strides);
      if (dim == 3) run12<float, 3>(type, opt, sign, M, loc, modes, in, out, strides);
    } else {
      if (dim == 1) run12<double, 1>(type, opt, sign, M, loc, modes, in, out, strides);
      if (dim == 2) run12<double, 2>(type, opt, sign, M, loc, modes, in, out, strides);
      if (dim == 3) run12<double, 3>(type, opt, sign, M, loc, modes, in, out, strides);
    }
    return 0;
  } catch (...) {
    return code_of(std::current_exception());
  }
}

// Persistent reference type-1/2 plan on the legacy default stream: create, set points,
// transform (asynchronous, as in the reference), destroy. Returns 0 or a NeonufftError code.
__attribute__((visibility("default"))) int ref_plan12_create(void** handle, int is_float, int dim,
                                                             double tol, double upsampfac,
                                                             int sign, int64_t M,
                                                             const void* const* loc,
                                                             const int64_t* modes) {
  try {
    neonufft::Options opt;
    opt.tol = tol;
    opt.upsampfac = upsampfac;
    RefPlan12Base* p = nullptr;
    if (is_float) {
      if (dim == 1) p = new RefPlan12<float, 1>(opt, sign, M, loc, modes);
      if (dim == 2) p = new RefPlan12<float, 2>(opt, sign, M, loc, modes);
      if (dim == 3) p = new RefPlan12<float, 3>(opt, sign, M, loc, modes);
    } else {
      if (dim == 1) p = new RefPlan12<double, 1>(opt, sign, M, loc, modes);
      if (dim == 2) p = new RefPlan12<double, 2>(opt, sign, M, loc, modes);
      if (dim == 3) p = new RefPlan12<double, 3>(opt, sign, M, loc, modes);
    }
    *handle = p;
    return 0;
  } catch (...) {
    return code_of(std::current_exception());
  }
}

__attribute__((visibility("default"))) int ref_plan12_set_points(void* h, int64_t M,
                                                                 const void* const* loc) {
  try {
    static_cast<RefPlan12Base*>(h)->set_points(M, loc);
    return 0;
  } catch (...) {
    return code_of(std::current_exception());
  }
}

__attribute__((visibility("default"))) int ref_plan12_t1(void* h, const void* in, void* out,
                                                         const int64_t* strides) {
  try {
    static_cast<RefPlan12Base*>(h)->t1(in, out, strides);
    return 0;
  } catch (...) {
    return code_of(std::current_exception());
  }
}

__attribute__((visibility("default"))) int ref_plan12_t2(void* h, const void* in,
                                                         const int64_t* strides, void* out) {
  try {
    static_cast<RefPlan12Base*>(h)->t2(in, strides, out);
    return 0;
  } catch (...) {
    return code_of(std::current_exception());
  }
}

__attribute__((visibility("default"))) void ref_plan12_destroy(void* h) {
  delete static_cast<RefPlan12Base*>(h);
}

__attribute__((visibility("default"))) int ref_gpu_type3(int is_float, int dim, double tol,
                                                         double upsampfac, int sign, int64_t M,
                                                         const void* const* in_pts, int64_t K,
                                                         const void* const* out_pts, int batch,
                                                         const void* in, void* out) {
  try {
    neonufft::Options opt;
    opt.tol = tol;
    opt.upsampfac = upsampfac;
    if (is_float) {
      if (dim == 1) run3<float, 1>(opt, sign, M, in_pts, K, out_pts, batch, in, out);
      if (dim == 2) run3<float, 2>(opt, sign, M, in_pts, K, out_pts, batch, in, out);
      if (dim == 3) run3<float, 3>(opt, sign, M, in_pts, K, out_pts, batch, in, out);
    } else {
      if (dim == 1) run3<double, 1>(opt, sign, M, in_pts, K, out_pts, batch, in, out);
      if (dim == 2) run3<double, 2>(opt, sign, M, in_pts, K, out_pts, batch, in, out);
      if (dim == 3) run3<double, 3>(opt, sign, M, in_pts, K, out_pts, batch, in, out);
    }
    return 0;
  } catch (...) {
    return code_of(std::current_exception());
  }
}

}  // extern "C"
