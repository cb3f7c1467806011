// ORACLE -- test infrastructure only. Used by tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline as the checker; never by the engine.
//
// CPU restatement of the reference's CPU NUFFT kernels (scalar C++ + OpenMP; the reference
// vectorises the same loops with Google Highway, which is absent here), plus the FP64 direct
// NUDFT sums that define the transforms. Heavy loops only; the plan logic, the FFT (scipy) and
// the deconvolution live in oracle.py.
//
//  - direct sums:      tests/nuft_direct_kernels.cpp:73-293 (reference), in double
//  - ES kernel:        src/neonufft/kernels/es_kernel_eval.hpp:39-45 (EsKernelDirect::eval_scalar)
//  - rescale:          src/neonufft/kernels/rescale_loc_kernel.cpp:33-74 (type 1/2), :78-130 (type 3)
//  - spreading:        src/neonufft/kernels/spreading_kernel.cpp:55-163 (padded grid, padding
//                      w/2 + 2 from src/neonufft/util/spread_padding.hpp:10-12)
//  - padding fold:     src/neonufft/kernels/fold_padding.cpp:27-135
//  - interpolation:    src/neonufft/kernels/interpolation_kernel.cpp:109-263 (periodic wrap)
//
// Precision: every restated kernel is templated on T (float or double) and computes in T, as the
// reference CPU path does; the direct sums are always double.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <vector>

namespace {

using i64 = std::int64_t;

// ---- direct sums ------------------------------------------------------------------------------
inline i64 k_offset(i64 n) { return n % 2 ? (n - 1) / 2 : n / 2; }

template <typename T>
inline T es_eval(T x, T beta, T c) {
  const T arg = T(1) - c * x * x;
  if (arg <= 0) return 0;
  return std::exp(beta * (std::sqrt(arg) - T(1)));
}

template <typename T>
void rescale(i64 n, const T* loc, T offset, T scale, int t3, T* out) {
  constexpr T pi = T(3.14159265358979323846);
  const T two_pi_inv = 1 / (2 * pi);
  for (i64 i = 0; i < n; ++i) {
    T l = loc[i];
    if (t3) l = (l - offset) * scale;
    l = (l + pi) * two_pi_inv;
    l = l - std::floor(l);
    out[i] = l;
  }
}

// One point's kernel values and padded start index along one dimension.
template <typename T>
inline void ker_values(T p, i64 n, int w, T beta, T c, T* ker, i64* start, i64 pad) {
  const T half_width = T(w) / T(2);
  const T loc = p * T(n);
  const T s = std::ceil(loc - half_width);
  *start = i64(s) + pad;
  const T x = s - loc;
  for (int k = 0; k < w; ++k) ker[k] = es_eval<T>(x + T(k), beta, c);
}

// Spreads points [begin, end) into the padded grid (dims nf + 2 pad), in T arithmetic, in the
// reference's multiplication order ((c * kz) * ky) * kx.
template <typename T>
void spread_range(int dim, int w, T beta, T c, i64 begin, i64 end, const T* const* p,
                  const std::complex<T>* in, const std::complex<T>* pre, const i64* nf,
                  std::complex<T>* grid) {
  const i64 pad = w / 2 + 2;
  const i64 P0 = nf[0] + 2 * pad;
  const i64 P1 = dim > 1 ? nf[1] + 2 * pad : 1;
  T kx[16], ky[16], kz[16];
  i64 s0, s1 = 0, s2 = 0;
  for (i64 j = begin; j < end; ++j) {
    ker_values<T>(p[0][j], nf[0], w, beta, c, kx, &s0, pad);
    if (dim > 1) ker_values<T>(p[1][j], nf[1], w, beta, c, ky, &s1, pad);
    if (dim > 2) ker_values<T>(p[2][j], nf[2], w, beta, c, kz, &s2, pad);
    std::complex<T> v = in[j];
    if (pre) v *= pre[j];
    if (dim == 1) {
      for (int a = 0; a < w; ++a) grid[s0 + a] += v * kx[a];
    } else if (dim == 2) {
      for (int b = 0; b < w; ++b) {
        const std::complex<T> vy = v * ky[b];
        std::complex<T>* row = grid + (s1 + b) * P0 + s0;
        for (int a = 0; a < w; ++a) row[a] += vy * kx[a];
      }
    } else {
      for (int cz = 0; cz < w; ++cz) {
        const std::complex<T> vz = v * kz[cz];
        for (int b = 0; b < w; ++b) {
          const std::complex<T> vyz = vz * ky[b];
          std::complex<T>* row = grid + ((s2 + cz) * P1 + (s1 + b)) * P0 + s0;
          for (int a = 0; a < w; ++a) row[a] += vyz * kx[a];
        }
      }
    }
  }
}

// Interpolation at points [begin, end) from the unpadded grid with periodic wrap.
template <typename T>
void interp_range(int dim, int w, T beta, T c, i64 begin, i64 end, const T* const* p,
                  const std::complex<T>* grid, const i64* nf, std::complex<T>* out) {
  T kx[16], ky[16], kz[16];
  i64 s0, s1 = 0, s2 = 0;
  auto wrap = [](i64 i, i64 n) {
    if (i < 0) return i + n;
    if (i >= n) return i - n;
    return i;
  };
  for (i64 j = begin; j < end; ++j) {
    ker_values<T>(p[0][j], nf[0], w, beta, c, kx, &s0, 0);
    if (dim > 1) ker_values<T>(p[1][j], nf[1], w, beta, c, ky, &s1, 0);
    if (dim > 2) ker_values<T>(p[2][j], nf[2], w, beta, c, kz, &s2, 0);
    std::complex<T> acc = 0;
    const int wy = dim > 1 ? w : 1;
    const int wz = dim > 2 ? w : 1;
    for (int cz = 0; cz < wz; ++cz) {
      const i64 iz = dim > 2 ? wrap(s2 + cz, nf[2]) : 0;
      for (int b = 0; b < wy; ++b) {
        const i64 iy = dim > 1 ? wrap(s1 + b, nf[1]) : 0;
        const std::complex<T>* row = grid + (iz * (dim > 1 ? nf[1] : 1) + iy) * nf[0];
        std::complex<T> r = 0;
        for (int a = 0; a < w; ++a) r += row[wrap(s0 + a, nf[0])] * kx[a];
        T kyz = T(1);
        if (dim > 1) kyz = ky[b];
        if (dim > 2) kyz = ky[b] * kz[cz];
        acc += kyz * r;
      }
    }
    out[j] = acc;
  }
}

template <typename T>
void fold_padding(int dim, int w, const i64* nf, std::complex<T>* pg, std::complex<T>* grid) {
  // Adds the padding periodically onto the interior and copies the interior out.
  const i64 pad = w / 2 + 2;
  const i64 P0 = nf[0] + 2 * pad;
  const i64 P1 = dim > 1 ? nf[1] + 2 * pad : 1;
  const i64 P2 = dim > 2 ? nf[2] + 2 * pad : 1;
  const i64 n1 = dim > 1 ? nf[1] : 1, n2 = dim > 2 ? nf[2] : 1;
  std::fill(grid, grid + nf[0] * n1 * n2, std::complex<T>(0));
  for (i64 z = 0; z < P2; ++z) {
    const i64 gz = dim > 2 ? ((z - pad) % n2 + n2) % n2 : 0;
    for (i64 y = 0; y < P1; ++y) {
      const i64 gy = dim > 1 ? ((y - pad) % n1 + n1) % n1 : 0;
      const std::complex<T>* src = pg + (z * P1 + y) * P0;
      std::complex<T>* dst = grid + (gz * n1 + gy) * nf[0];
      for (i64 x = 0; x < P0; ++x) {
        const i64 gx = ((x - pad) % nf[0] + nf[0]) % nf[0];
        dst[gx] += src[x];
      }
    }
  }
}

}  // namespace

extern "C" {

int oracle_num_threads() { return omp_get_max_threads(); }
void oracle_set_threads(int n) { omp_set_num_threads(n > 0 ? n : 1); }

// out[k] for the full CMCL mode box (column-major), out interleaved complex double.
void oracle_direct_type1(int dim, int sign, i64 M, const double* const* x, const double* c,
                         const i64* modes, double* out) {
  const i64 n0 = modes[0], n1 = dim > 1 ? modes[1] : 1, n2 = dim > 2 ? modes[2] : 1;
  const i64 total = n0 * n1 * n2;
  const auto* in = reinterpret_cast<const std::complex<double>*>(c);
  auto* o = reinterpret_cast<std::complex<double>*>(out);
#pragma omp parallel for schedule(dynamic, 4)
  for (i64 m = 0; m < total; ++m) {
    const i64 i0 = m % n0, i1 = (m / n0) % n1, i2 = m / (n0 * n1);
    const double k0 = double(i0 - k_offset(n0)) * sign;
    const double k1 = dim > 1 ? double(i1 - k_offset(n1)) * sign : 0.0;
    const double k2 = dim > 2 ? double(i2 - k_offset(n2)) * sign : 0.0;
    std::complex<double> s = 0;
    for (i64 j = 0; j < M; ++j) {
      double ph = k0 * x[0][j];
      if (dim > 1) ph += k1 * x[1][j];
      if (dim > 2) ph += k2 * x[2][j];
      s += in[j] * std::complex<double>(std::cos(ph), std::sin(ph));
    }
    o[m] = s;
  }
}

void oracle_direct_type2(int dim, int sign, const i64* modes, const double* f, i64 M,
                         const double* const* x, double* out) {
  const i64 n0 = modes[0], n1 = dim > 1 ? modes[1] : 1, n2 = dim > 2 ? modes[2] : 1;
  const auto* in = reinterpret_cast<const std::complex<double>*>(f);
  auto* o = reinterpret_cast<std::complex<double>*>(out);
#pragma omp parallel for schedule(dynamic, 16)
  for (i64 j = 0; j < M; ++j) {
    std::complex<double> s = 0;
    for (i64 i2 = 0; i2 < n2; ++i2) {
      for (i64 i1 = 0; i1 < n1; ++i1) {
        double ph12 = 0;
        if (dim > 1) ph12 += double(i1 - k_offset(n1)) * x[1][j];
        if (dim > 2) ph12 += double(i2 - k_offset(n2)) * x[2][j];
        const std::complex<double>* row = in + (i2 * n1 + i1) * n0;
        for (i64 i0 = 0; i0 < n0; ++i0) {
          const double ph = sign * (double(i0 - k_offset(n0)) * x[0][j] + ph12);
          s += row[i0] * std::complex<double>(std::cos(ph), std::sin(ph));
        }
      }
    }
    o[j] = s;
  }
}

void oracle_direct_type3(int dim, int sign, i64 M, const double* const* x, const double* c,
                         i64 K, const double* const* s, double* out) {
  const auto* in = reinterpret_cast<const std::complex<double>*>(c);
  auto* o = reinterpret_cast<std::complex<double>*>(out);
#pragma omp parallel for schedule(dynamic, 16)
  for (i64 k = 0; k < K; ++k) {
    std::complex<double> acc = 0;
    for (i64 j = 0; j < M; ++j) {
      double ph = x[0][j] * s[0][k];
      if (dim > 1) ph += x[1][j] * s[1][k];
      if (dim > 2) ph += x[2][j] * s[2][k];
      ph *= sign;
      acc += in[j] * std::complex<double>(std::cos(ph), std::sin(ph));
    }
    o[k] = acc;
  }
}

// ---- restated reference CPU kernels (T = float: _f32, T = double: _f64) ----------------------
#define ORACLE_DEFINE(T, SUF)                                                                    \
  void oracle_rescale_##SUF(i64 n, const T* loc, T offset, T scale, int t3, T* out) {            \
    rescale<T>(n, loc, offset, scale, t3, out);                                                  \
  }                                                                                              \
  /* Serial spread into the padded grid, then periodic fold into grid (nf dims). */              \
  void oracle_spread_##SUF(int dim, int w, T beta, T c, i64 M, const T* const* p, const T* in,   \
                           const T* pre, const i64* nf, T* grid) {                               \
    const i64 pad = w / 2 + 2;                                                                   \
    i64 pc = 1;                                                                                  \
    for (int d = 0; d < dim; ++d) pc *= nf[d] + 2 * pad;                                         \
    std::vector<std::complex<T>> pg(pc, std::complex<T>(0));                                     \
    spread_range<T>(dim, w, beta, c, 0, M, p, reinterpret_cast<const std::complex<T>*>(in),      \
                    reinterpret_cast<const std::complex<T>*>(pre), nf, pg.data());               \
    fold_padding<T>(dim, w, nf, pg.data(), reinterpret_cast<std::complex<T>*>(grid));            \
  }                                                                                              \
  /* Slab-parallel spread (type 3, reference plan_t3_impl.hpp:128-161, :290-327): slabs of at   \
     least w + 4 cells along the last dimension, even slabs then odd slabs. */                  \
  void oracle_spread_slabs_##SUF(int dim, int w, T beta, T c, i64 M, const T* const* p,          \
                                 const T* in, const T* pre, const i64* nf, T* grid) {            \
    const i64 pad = w / 2 + 2;                                                                   \
    i64 pc = 1;                                                                                  \
    for (int d = 0; d < dim; ++d) pc *= nf[d] + 2 * pad;                                         \
    std::vector<std::complex<T>> pg(pc, std::complex<T>(0));                                     \
    const int ld = dim - 1;                                                                      \
    const i64 width = w + 4;                                                                     \
    i64 nslab = std::max<i64>(1, std::min<i64>(6 * omp_get_max_threads(), nf[ld] / width));      \
    const i64 slab_len = (nf[ld] + nslab - 1) / nslab;                                           \
    std::vector<std::vector<i64>> members(nslab);                                                \
    std::vector<T> pts[3];                                                                       \
    for (i64 j = 0; j < M; ++j) {                                                                \
      i64 s = i64(p[ld][j] * T(nf[ld])) / slab_len;                                              \
      s = std::min<i64>(std::max<i64>(s, 0), nslab - 1);                                         \
      members[s].push_back(j);                                                                   \
    }                                                                                            \
    const auto* cin = reinterpret_cast<const std::complex<T>*>(in);                              \
    const auto* cpre = reinterpret_cast<const std::complex<T>*>(pre);                            \
    for (int parity = 0; parity < 2; ++parity) {                                                 \
      _Pragma("omp parallel for schedule(dynamic, 1)") for (i64 s = parity; s < nslab; s += 2) { \
        const auto& mem = members[s];                                                            \
        std::vector<T> q[3];                                                                     \
        std::vector<std::complex<T>> v(mem.size());                                              \
        for (int d = 0; d < dim; ++d) q[d].resize(mem.size());                                   \
        for (size_t t = 0; t < mem.size(); ++t) {                                                \
          for (int d = 0; d < dim; ++d) q[d][t] = p[d][mem[t]];                                  \
          v[t] = cin[mem[t]];                                                                    \
          if (cpre) v[t] *= cpre[mem[t]];                                                        \
        }                                                                                        \
        const T* qp[3] = {q[0].data(), dim > 1 ? q[1].data() : nullptr,                         \
                          dim > 2 ? q[2].data() : nullptr};                                      \
        spread_range<T>(dim, w, beta, c, 0, i64(mem.size()), qp, v.data(), nullptr, nf,          \
                        pg.data());                                                              \
      }                                                                                          \
    }                                                                                            \
    fold_padding<T>(dim, w, nf, pg.data(), reinterpret_cast<std::complex<T>*>(grid));            \
  }                                                                                              \
  /* OpenMP-parallel interpolation (reference plan_impl.hpp:115-125). */                         \
  void oracle_interp_##SUF(int dim, int w, T beta, T c, const T* grid, const i64* nf, i64 M,     \
                           const T* const* p, T* out) {                                          \
    const int nt = omp_get_max_threads();                                                        \
    _Pragma("omp parallel for schedule(static)") for (int t = 0; t < nt; ++t) {                  \
      const i64 b = M * t / nt, e = M * (t + 1) / nt;                                            \
      interp_range<T>(dim, w, beta, c, b, e, p, reinterpret_cast<const std::complex<T>*>(grid),  \
                      nf, reinterpret_cast<std::complex<T>*>(out));                              \
    }                                                                                            \
  }

ORACLE_DEFINE(float, f32)
ORACLE_DEFINE(double, f64)

}  // extern "C"
