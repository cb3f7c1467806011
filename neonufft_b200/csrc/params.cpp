// Host-side parameter math (see params.hpp for the reference files each function follows).
#include "params.hpp"

#include <algorithm>
#include <cmath>
#include <cstddef>

namespace nnb {

namespace {
constexpr double kPiD = 3.14159265358979323846264338327950288;
}

KernelParam kernel_param(double tol, double upsampfac, bool single, int w_override) {
  // Width heuristic and beta factors of the reference (src/neonufft/es_kernel_param.hpp:27-55):
  // w = ceil(-log10(tol/10)) for upsampfac 2, else ceil(-ln(tol) / (pi sqrt(1 - 1/upsampfac))),
  // clamped to [2, 16]; beta = f(w) * w with FINUFFT's factors, or Eq. 4.5 of the FINUFFT paper
  // (0.97 pi (1 - 1/(2 upsampfac))) when upsampfac != 2.
  int w = 2;
  if (upsampfac == 2.0) {
    w = int(std::ceil(-std::log10(tol / 10.0)));
  } else {
    w = int(std::ceil(-std::log(tol) / (kPiD * std::sqrt(1.0 - 1.0 / upsampfac))));
  }
  w = std::max(2, w);
  w = std::min(16, w);
  if (w_override >= 2 && w_override <= 16) w = w_override;

  double beta_fac = 2.30;
  if (w == 2) beta_fac = 2.20;
  if (w == 3) beta_fac = 2.26;
  if (w == 4) beta_fac = 2.38;
  if (upsampfac != 2.0) beta_fac = 0.97 * kPiD * (1.0 - 1.0 / (2 * upsampfac));

  KernelParam kp;
  kp.w = w;
  kp.upsampfac = upsampfac;
  kp.half_width = w / 2.0;
  const double beta = beta_fac * w;
  if (single) {
    // The reference stores beta as T and the device kernel uses c = 4.f / float(w * w).
    kp.beta = double(float(beta));
    kp.c = double(4.f / float(w * w));
  } else {
    kp.beta = beta;
    kp.c = 4.0 / double(w * w);
  }
  return kp;
}

std::int64_t fine_grid_size(std::int64_t modes, double upsampfac, int w) {
  // std::max<std::size_t>(2w, modes * upsampfac): the product is truncated to an integer.
  const auto scaled = static_cast<std::size_t>(double(modes) * upsampfac);
  return static_cast<std::int64_t>(std::max<std::size_t>(std::size_t(2 * w), scaled));
}

std::int64_t next235even(std::int64_t n) {
  if (n <= 2) return 2;
  if (n % 2 == 1) n += 1;
  for (std::int64_t cand = n;; cand += 2) {
    std::int64_t r = cand;
    for (std::int64_t f : {2, 3, 5}) {
      while (r % f == 0) r /= f;
    }
    if (r == 1) return cand;
  }
}

template <typename T>
T3Dim<T> t3_geometry(int w, double upsampfac, T recenter_threshold, T in_min, T in_max,
                     T out_min, T out_max) {
  // Centres and half extents, recentred to 0 when the offset is small relative to the extent
  // (reference src/neonufft/util/grid_info_t3.hpp:26-42), all in T like the reference.
  T3Dim<T> g;
  g.input_offset = (in_max + in_min) / 2;
  g.output_offset = (out_max + out_min) / 2;
  g.input_half_extent =
      std::max(std::abs(in_max - g.input_offset), std::abs(in_min - g.input_offset));
  g.output_half_extent =
      std::max(std::abs(out_max - g.output_offset), std::abs(out_min - g.output_offset));
  if (std::abs(g.input_offset) < recenter_threshold * g.input_half_extent) {
    g.input_offset = 0;
    g.input_half_extent = std::max(std::abs(in_max), std::abs(in_min));
  }
  if (std::abs(g.output_offset) < recenter_threshold * g.output_half_extent) {
    g.output_offset = 0;
    g.output_half_extent = std::max(std::abs(out_max), std::abs(out_min));
  }

  // Spread grid size nf1 = 2 upsampfac X S / pi + w + 1 with X, S guarded against zero, at
  // least 2w, rounded up to even (reference src/contrib/es_kernel/util.hpp:64-88). The
  // reference evaluates the product in double (leading 2.0 literal) from T-rounded factors.
  const T up_t = T(upsampfac);
  const T pi_t = T(kPiD);
  const T S = g.output_half_extent;
  const T X = g.input_half_extent;
  T X_safe = X, S_safe = S;
  if (X == T(0)) {
    if (S == T(0)) {
      X_safe = 1;
      S_safe = 1;
    } else {
      X_safe = std::max(X_safe, T(1) / S);
    }
  } else {
    S_safe = std::max(S_safe, T(1) / X);
  }
  std::int64_t nf1 = static_cast<std::int64_t>(2.0 * double(up_t) * double(S_safe) *
                                                   double(X_safe) / double(pi_t) +
                                               double(w + 1));
  if (nf1 < 2 * w) nf1 = 2 * w;
  nf1 += nf1 % 2;
  g.spread_grid = nf1;

  // FFT grid: next235even(max(2w, nf1 * upsampfac)) (reference grid_info_t3.hpp:49-50).
  const auto scaled = static_cast<std::size_t>(double(nf1) * upsampfac);
  g.fft_grid = next235even(
      static_cast<std::int64_t>(std::max<std::size_t>(std::size_t(2 * w), scaled)));

  // h = 2 pi / nf1, gamma = nf1 / (2 upsampfac S) with S guarded (reference util.hpp:92-105).
  g.h = T(2) * pi_t / T(nf1);
  T S_g = S;
  if (X == T(0) && S == T(0)) {
    S_g = 1;
  } else if (S == T(0)) {
    S_g = std::max(S_g, T(1) / X);
  }
  g.gamma = T(double(T(nf1)) / (2.0 * double(up_t) * double(S_g)));
  return g;
}

template T3Dim<float> t3_geometry<float>(int, double, float, float, float, float, float);
template T3Dim<double> t3_geometry<double>(int, double, double, double, double, double, double);

void gauss_legendre(int n, std::vector<double>& nodes, std::vector<double>& weights) {
  // Newton iteration on the three-term recurrence of P_n from the Tricomi initial guesses
  // x_i ~ cos(pi (i - 1/4) / (n + 1/2)); weights 2 / ((1 - x^2) P_n'(x)^2).
  nodes.assign(n, 0.0);
  weights.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    double x = std::cos(kPiD * (i + 0.75) / (n + 0.5));
    double dp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = x;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2.0 * k - 1.0) * x * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      const double pn = (n == 0) ? 1.0 : (n == 1 ? x : p1);
      const double pn1 = (n == 1) ? 1.0 : p0;
      dp = n * (x * pn - pn1) / (x * x - 1.0);
      const double dx = pn / dp;
      x -= dx;
      if (std::abs(dx) < 1e-16 * std::max(1.0, std::abs(x))) {
        // one more polish step for the derivative at the converged node
        double q0 = 1.0, q1 = x;
        for (int k = 2; k <= n; ++k) {
          const double q2 = ((2.0 * k - 1.0) * x * q1 - (k - 1.0) * q0) / k;
          q0 = q1;
          q1 = q2;
        }
        dp = n * (x * q1 - q0) / (x * x - 1.0);
        break;
      }
    }
    nodes[i] = x;
    weights[i] = 2.0 / ((1.0 - x * x) * dp * dp);
  }
}

double es_kernel(const KernelParam& kp, double x) {
  const double arg = 1.0 - kp.c * x * x;
  if (arg <= 0.0) return 0.0;
  return std::exp(kp.beta * (std::sqrt(arg) - 1.0));
}

PhiHatQuad phi_hat_quadrature(const KernelParam& kp) {
  // The kernel is even, so only the q nodes on (0, 1] of a 2q-node rule are used:
  // integral_{-w/2}^{w/2} phi(z) cos(xi z) dz = w * sum_q W_q phi(z_q w/2) cos(xi z_q w/2).
  // q = w + w%2 + 10 nodes, the count of the reference CPU path
  // (src/neonufft/kernels/fseries_kernel.cpp:35), evaluated in double precision.
  const int q = kp.w + (kp.w % 2) + 10;
  std::vector<double> x, wt;
  gauss_legendre(2 * q, x, wt);
  PhiHatQuad out;
  out.z.resize(q);
  out.kv.resize(q);
  for (int i = 0; i < q; ++i) {
    const double z = x[i] * kp.half_width;  // x[i] > 0 for i < q
    out.z[i] = z;
    out.kv[i] = double(kp.w) * wt[i] * es_kernel(kp, z);
  }
  return out;
}

std::vector<double> deconv_factors(const KernelParam& kp, std::int64_t nf) {
  const PhiHatQuad quad = phi_hat_quadrature(kp);
  const std::int64_t n_out = nf / 2 + 1;
  std::vector<double> corr(n_out);
  const double alpha = 2.0 * kPiD / double(nf);
  for (std::int64_t k = 0; k < n_out; ++k) {
    double sum = 0.0;
    for (std::size_t i = 0; i < quad.z.size(); ++i) {
      sum += quad.kv[i] * std::cos(alpha * double(k) * quad.z[i]);
    }
    corr[k] = ((k % 2) ? -1.0 : 1.0) / sum;
  }
  return corr;
}

}  // namespace nnb
