// Type-3 helper kernels: coordinate bounds, pre-phase and post-phase, all in double precision.
//
//  - min_max replaces the reference's 2*D CUB reductions (src/neonufft/gpu/kernels/min_max_kernel.cu:16-39)
//    by one pass per coordinate array with order-preserving integer atomics.
//  - prephase follows src/neonufft/gpu/kernels/prephase_kernel.cu:35-50:
//    pre_j = exp(i sign sum_d x_jd D_d), evaluated in double and rounded to the plan precision.
//  - postphase follows src/neonufft/gpu/kernels/postphase_kernel.cu:27-76:
//    post_k = exp(i sign sum_d (s_kd - D_d) C_d) / prod_d phi_hat((s_kd - D_d) gamma_d h_d),
//    with phi_hat by Gauss-Legendre quadrature, all in double.
#include <cstring>

#include "kernels.cuh"

namespace nnb {

namespace {

constexpr int kT3Threads = 256;

__device__ __forceinline__ unsigned long long enc_double(double v) {
  const unsigned long long b = __double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}

template <typename T>
__global__ void __launch_bounds__(kT3Threads)
    min_max_kernel(int dim, CoordPtrs<T> x, i64 M, unsigned long long* out) {
  for (int d = 0; d < dim; ++d) {
    double lo = 1.0 / 0.0, hi = -1.0 / 0.0;
    for (i64 i = blockIdx.x * i64(kT3Threads) + threadIdx.x; i < M;
         i += i64(gridDim.x) * kT3Threads) {
      const double v = double(x.p[d][i]);
      if (v == v) {
        lo = fmin(lo, v);
        hi = fmax(hi, v);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&out[2 * d], enc_double(lo));
      atomicMax(&out[2 * d + 1], enc_double(hi));
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kT3Threads)
    prephase_kernel(int dim, int sign, CoordPtrs<T> x, i64 M, double D0, double D1, double D2,
                    cplx_t<T>* pre) {
  for (i64 i = blockIdx.x * i64(kT3Threads) + threadIdx.x; i < M;
       i += i64(gridDim.x) * kT3Threads) {
    double ph = double(x.p[0][i]) * D0;
    if (dim > 1) ph += double(x.p[1][i]) * D1;
    if (dim > 2) ph += double(x.p[2][i]) * D2;
    double s, c;
    sincos(ph, &s, &c);
    pre[i] = cplx_t<T>{T(c), T(sign * s)};
  }
}

struct PostGeom {
  double D[3];
  double C[3];
  double scale[3];
};

template <typename T>
__global__ void __launch_bounds__(kT3Threads)
    postphase_kernel(int dim, int sign, CoordPtrs<T> s, i64 K, PostGeom geo, PostphaseQuad q,
                     cplx_t<T>* post) {
  for (i64 i = blockIdx.x * i64(kT3Threads) + threadIdx.x; i < K;
       i += i64(gridDim.x) * kT3Threads) {
    double phi_hat = 1.0;
    double phase = 0.0;
    for (int d = 0; d < dim; ++d) {
      const double t = double(s.p[d][i]) - geo.D[d];
      const double xi = t * geo.scale[d];
      double sum = 0.0;
      for (int k = 0; k < q.n; ++k) sum += q.kv[k] * cos(xi * q.z[k]);
      phi_hat *= sum;
      phase += t * geo.C[d];
    }
    double sn, cs;
    sincos(phase, &sn, &cs);
    post[i] = cplx_t<T>{T(cs / phi_hat), T(sign * sn / phi_hat)};
  }
}

int grid_for(i64 n) {
  i64 g = (n + kT3Threads - 1) / kT3Threads;
  if (g > 148 * 16) g = 148 * 16;
  if (g < 1) g = 1;
  return int(g);
}

}  // namespace

void init_min_max(unsigned long long* enc_host, int n) {
  for (int i = 0; i < n; ++i) enc_host[i] = (i % 2 == 0) ? ~0ull : 0ull;
}

void decode_min_max(const unsigned long long* enc, int n, double* out) {
  for (int i = 0; i < n; ++i) {
    unsigned long long b = enc[i];
    b = (b & 0x8000000000000000ull) ? (b & ~0x8000000000000000ull) : ~b;
    double v;
    static_assert(sizeof(v) == sizeof(b), "");
    memcpy(&v, &b, sizeof(v));
    out[i] = v;
  }
}

template <typename T>
void launch_min_max(int dim, CoordPtrs<T> x, i64 M, unsigned long long* enc_out,
                    cudaStream_t stream) {
  if (M <= 0) return;
  min_max_kernel<T><<<grid_for(M), kT3Threads, 0, stream>>>(dim, x, M, enc_out);
  NNB_LAUNCH_CHECK();
}

template <typename T>
void launch_prephase(int dim, int sign, CoordPtrs<T> x, i64 M, const double* D, cplx_t<T>* pre,
                     cudaStream_t stream) {
  if (M <= 0) return;
  prephase_kernel<T><<<grid_for(M), kT3Threads, 0, stream>>>(
      dim, sign, x, M, D[0], dim > 1 ? D[1] : 0.0, dim > 2 ? D[2] : 0.0, pre);
  NNB_LAUNCH_CHECK();
}

template <typename T>
void launch_postphase(int dim, int sign, CoordPtrs<T> s, i64 K, const double* out_offset,
                      const double* in_offset, const double* scale, const PostphaseQuad& q,
                      cplx_t<T>* post, cudaStream_t stream) {
  if (K <= 0) return;
  PostGeom geo{};
  for (int d = 0; d < dim; ++d) {
    geo.D[d] = out_offset[d];
    geo.C[d] = in_offset[d];
    geo.scale[d] = scale[d];
  }
  postphase_kernel<T><<<grid_for(K), kT3Threads, 0, stream>>>(dim, sign, s, K, geo, q, post);
  NNB_LAUNCH_CHECK();
}

template void launch_min_max<float>(int, CoordPtrs<float>, i64, unsigned long long*, cudaStream_t);
template void launch_min_max<double>(int, CoordPtrs<double>, i64, unsigned long long*, cudaStream_t);
template void launch_prephase<float>(int, int, CoordPtrs<float>, i64, const double*, float2*, cudaStream_t);
template void launch_prephase<double>(int, int, CoordPtrs<double>, i64, const double*, double2*, cudaStream_t);
template void launch_postphase<float>(int, int, CoordPtrs<float>, i64, const double*, const double*, const double*, const PostphaseQuad&, float2*, cudaStream_t);
template void launch_postphase<double>(int, int, CoordPtrs<double>, i64, const double*, const double*, const double*, const PostphaseQuad&, double2*, cudaStream_t);

}  // namespace nnb
