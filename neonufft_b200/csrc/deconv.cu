// Deconvolution by the kernel's Fourier transform, with mode reordering.
//
// downsample (type 1) follows the reference's downsample_{1,2,3}d_kernel
// (src/neonufft/gpu/kernels/downsample_kernel.cu:18-191): mode k of the user's box (CMCL order
// k = i - N/2, or FFT order) is read from fine cell k mod nf and scaled by prod_d corr_d[|k_d|].
// upsample (type 2, type-3 stage 2) is the inverse (reference upsample_kernel.cu:18-196), but
// here one kernel writes every fine cell -- zero outside the mode box -- so the separate grid
// memset of the reference (src/neonufft/gpu/plan_impl.hpp:117) is fused away.
#include "kernels.cuh"

namespace nnb {

namespace {

constexpr int kDeconvThreads = 256;

__device__ __forceinline__ i64 mode_of_index(i64 i, i64 n, int order) {
  const i64 n_neg = n / 2;
  if (order == NEONUFFT_MODE_ORDER_CMCL) return i - n_neg;
  const i64 n_nonneg = n - n_neg;
  return i < n_nonneg ? i : i - n;
}

__device__ __forceinline__ i64 index_of_mode(i64 k, i64 n, int order) {
  const i64 n_neg = n / 2;
  if (order == NEONUFFT_MODE_ORDER_CMCL) return k + n_neg;
  return k >= 0 ? k : k + n;
}

// Elements spanned by the user's strided mode array: 1 + sum_d (modes_d - 1) stride_d.
template <typename T>
__device__ __forceinline__ i64 mode_array_extent(const DeconvArgs<T>& a) {
  i64 e = 1;
  for (int d = 0; d < a.dim; ++d) e += (a.modes[d] - 1) * a.stride[d];
  return e;
}

template <typename T>
__global__ void __launch_bounds__(kDeconvThreads)
    downsample_kernel(DeconvArgs<T> a, const cplx_t<T>* __restrict__ fine,
                      cplx_t<T>* __restrict__ out) {
  const i64 i0 = blockIdx.x * i64(kDeconvThreads) + threadIdx.x;
  if (i0 >= a.modes[0]) return;
  const i64 i1 = blockIdx.y;
  const i64 i2 = blockIdx.z;
  const i64 k0 = mode_of_index(i0, a.modes[0], a.order);
  T c = a.corr[0][k0 < 0 ? -k0 : k0];
  i64 f = k0 >= 0 ? k0 : a.nf[0] + k0;
  i64 o = i0 * a.stride[0];
  if (a.dim > 1) {
    const i64 k1 = mode_of_index(i1, a.modes[1], a.order);
    c *= a.corr[1][k1 < 0 ? -k1 : k1];
    f += (k1 >= 0 ? k1 : a.nf[1] + k1) * a.nf[0];
    o += i1 * a.stride[1];
  }
  if (a.dim > 2) {
    const i64 k2 = mode_of_index(i2, a.modes[2], a.order);
    c *= a.corr[2][k2 < 0 ? -k2 : k2];
    f += (k2 >= 0 ? k2 : a.nf[2] + k2) * a.nf[0] * a.nf[1];
    o += i2 * a.stride[2];
  }
  if (!NNB_CHECK_INDEX(f, a.nf[0] * a.nf[1] * a.nf[2]) ||
      !NNB_CHECK_INDEX(o, mode_array_extent(a))) {
    return;
  }
  const cplx_t<T> v = fine[f];
  out[o] = cplx_t<T>{v.x * c, v.y * c};
}

template <typename T>
__global__ void __launch_bounds__(kDeconvThreads)
    upsample_kernel(DeconvArgs<T> a, const cplx_t<T>* __restrict__ in,
                    cplx_t<T>* __restrict__ fine) {
  const i64 j0 = blockIdx.x * i64(kDeconvThreads) + threadIdx.x;
  if (j0 >= a.nf[0]) return;
  const i64 j1 = blockIdx.y;
  const i64 j2 = blockIdx.z;
  const i64 f = j0 + (j1 + j2 * a.nf[1]) * a.nf[0];

  // Fine cell j holds mode k = j (j < n_nonneg) or k = j - nf (j >= nf - n_neg); zero between.
  bool inside = true;
  T c = 1;
  i64 src = 0;
  const i64 js[3] = {j0, j1, j2};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (d >= a.dim) break;
    const i64 n = a.modes[d];
    const i64 n_neg = n / 2;
    const i64 n_nonneg = n - n_neg;
    const i64 j = js[d];
    i64 k;
    if (j < n_nonneg) {
      k = j;
    } else if (j >= a.nf[d] - n_neg) {
      k = j - a.nf[d];
    } else {
      inside = false;
      break;
    }
    c *= a.corr[d][k < 0 ? -k : k];
    src += index_of_mode(k, n, a.order) * a.stride[d];
  }
  if (!NNB_CHECK_INDEX(f, a.nf[0] * a.nf[1] * a.nf[2])) return;
  if (!inside) {
    fine[f] = cplx_t<T>{T(0), T(0)};
    return;
  }
  if (!NNB_CHECK_INDEX(src, mode_array_extent(a))) return;
  const cplx_t<T> v = in[src];
  fine[f] = cplx_t<T>{v.x * c, v.y * c};
}

}  // namespace

template <typename T>
void launch_downsample(const DeconvArgs<T>& a, const cplx_t<T>* fine, cplx_t<T>* out,
                       cudaStream_t stream) {
  const i64 m1 = a.dim > 1 ? a.modes[1] : 1;
  const i64 m2 = a.dim > 2 ? a.modes[2] : 1;
  if (m1 > 65535 || m2 > 65535) throw_input("mode count above 65535 in dimension 1 or 2");
  dim3 grid(unsigned((a.modes[0] + kDeconvThreads - 1) / kDeconvThreads), unsigned(m1),
            unsigned(m2));
  downsample_kernel<T><<<grid, kDeconvThreads, 0, stream>>>(a, fine, out);
  NNB_LAUNCH_CHECK();
}

template <typename T>
void launch_upsample(const DeconvArgs<T>& a, const cplx_t<T>* in, cplx_t<T>* fine,
                     cudaStream_t stream) {
  const i64 n1 = a.dim > 1 ? a.nf[1] : 1;
  const i64 n2 = a.dim > 2 ? a.nf[2] : 1;
  if (n1 > 65535 || n2 > 65535) throw_input("fine grid above 65535 in dimension 1 or 2");
  dim3 grid(unsigned((a.nf[0] + kDeconvThreads - 1) / kDeconvThreads), unsigned(n1),
            unsigned(n2));
  upsample_kernel<T><<<grid, kDeconvThreads, 0, stream>>>(a, in, fine);
  NNB_LAUNCH_CHECK();
}

template void launch_downsample<float>(const DeconvArgs<float>&, const float2*, float2*, cudaStream_t);
template void launch_downsample<double>(const DeconvArgs<double>&, const double2*, double2*, cudaStream_t);
template void launch_upsample<float>(const DeconvArgs<float>&, const float2*, float2*, cudaStream_t);
template void launch_upsample<double>(const DeconvArgs<double>&, const double2*, double2*, cudaStream_t);

}  // namespace nnb
