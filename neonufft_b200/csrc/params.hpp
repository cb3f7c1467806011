// Host-side parameter math of the engine, all in double precision:
//  - ES kernel parameters from (tol, upsampfac)      (reference src/neonufft/es_kernel_param.hpp:24-56)
//  - fine-grid sizes for types 1/2                    (reference src/neonufft/gpu/plan_impl.hpp:56-60)
//  - type-3 geometry (centres, half extents, grids)   (reference src/neonufft/util/grid_info_t3.hpp:18-52,
//                                                      src/contrib/es_kernel/util.hpp:39-105)
//  - Gauss-Legendre nodes (own Newton iteration; the reference uses the Glaser-Liu-Rokhlin
//    method, src/contrib/legendre_rule/legendre_rule_fast.cpp:30)
//  - deconvolution factors 1/phi_hat(k) on the fine grid (reference
//    src/neonufft/kernels/fseries_kernel.cpp:33-77, src/neonufft/gpu/kernels/fseries_kernel.cu:24-67)
#pragma once

#include <array>
#include <cstdint>
#include <vector>

namespace nnb {

struct KernelParam {
  int w = 0;              // n_spread
  double beta = 0;        // ES shape parameter, already rounded to the plan's precision
  double c = 0;           // 4 / w^2, rounded to the plan's precision
  double half_width = 0;  // w / 2
  double upsampfac = 2.0;
};

// `single` selects rounding of beta and c to float (the reference stores them as T).
// `w_override` in [2, 16] replaces the width heuristic (beta then follows the same rule).
KernelParam kernel_param(double tol, double upsampfac, bool single, int w_override = 0);

// Fine grid size of a type-1/2 plan along one dimension: max(2w, floor(modes * upsampfac)).
std::int64_t fine_grid_size(std::int64_t modes, double upsampfac, int w);

// Smallest even integer >= n whose prime factors are 2, 3 and 5 (n <= 2 gives 2).
std::int64_t next235even(std::int64_t n);

// Type-3 geometry for one dimension. T is the precision the reference computes it in; the
// engine reproduces the same rounding so that grid sizes agree with the reference exactly.
template <typename T>
struct T3Dim {
  T input_offset = 0, output_offset = 0;
  T input_half_extent = 0, output_half_extent = 0;
  std::int64_t spread_grid = 0;  // nf1
  std::int64_t fft_grid = 0;     // next235even(max(2w, upsampfac * nf1))
  T h = 0;                       // 2 pi / nf1
  T gamma = 0;                   // nf1 / (2 upsampfac S)
};

template <typename T>
T3Dim<T> t3_geometry(int w, double upsampfac, T recenter_threshold, T in_min, T in_max,
                     T out_min, T out_max);

// Gauss-Legendre rule with n nodes on [-1, 1], nodes sorted descending (positive first).
void gauss_legendre(int n, std::vector<double>& nodes, std::vector<double>& weights);

// Quadrature of the ES kernel's Fourier transform on [0, w/2]: phi_hat(xi) =
// sum_q kv[q] * cos(xi * z[q]) with z[q] in [0, w/2] and kv[q] = w * W_q * phi(z_q).
struct PhiHatQuad {
  std::vector<double> z;
  std::vector<double> kv;
};
PhiHatQuad phi_hat_quadrature(const KernelParam& kp);

// ES kernel value in double precision (with the plan's rounded beta and c).
double es_kernel(const KernelParam& kp, double x);

// corr[k] = (-1)^k / phi_hat(2 pi k / nf), k = 0 .. nf/2 (nf/2 + 1 values).
std::vector<double> deconv_factors(const KernelParam& kp, std::int64_t nf);

}  // namespace nnb
