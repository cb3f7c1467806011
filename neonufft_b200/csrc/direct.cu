// FP64 direct NUDFT sums on the GPU for sampled outputs (accuracy measurement only).
// Same sums as the reference's test oracle (tests/nuft_direct_kernels.cpp:73-293): mode numbers
// k = i - floor(N/2) in CMCL order, phase sign * k.x, evaluated here in double with sincos.
// Each block accumulates one sample over one chunk of the summation range and adds its partial
// sum with double atomics, so the result is order-independent up to rounding.
#include "kernels.cuh"

namespace nnb {

namespace {

constexpr int kDirectThreads = 256;
constexpr int kDirectChunk = kDirectThreads * 16;

__device__ __forceinline__ void block_add2(double sx, double sy, double* out) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
  }
  __shared__ double red[2][kDirectThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = sx;
    red[1][warp] = sy;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < kDirectThreads / 32; ++w) {
      a += red[0][w];
      b += red[1][w];
    }
    atomicAdd(out, a);
    atomicAdd(out + 1, b);
  }
}

struct Loc3 {
  const double* p[3];
};

__global__ void __launch_bounds__(kDirectThreads)
    direct_type1_kernel(int dim, int sign, i64 M, Loc3 x, const double2* in, const i64* modes_idx,
                        double* out) {
  const i64 s = blockIdx.y;
  double k[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) k[d] = double(modes_idx[s * dim + d]) * sign;
  const i64 begin = i64(blockIdx.x) * kDirectChunk;
  const i64 end = min(M, begin + kDirectChunk);
  double sx = 0, sy = 0;
  for (i64 j = begin + threadIdx.x; j < end; j += kDirectThreads) {
    double ph = k[0] * x.p[0][j];
    if (dim > 1) ph += k[1] * x.p[1][j];
    if (dim > 2) ph += k[2] * x.p[2][j];
    double sn, cs;
    sincos(ph, &sn, &cs);
    const double2 c = in[j];
    sx += c.x * cs - c.y * sn;
    sy += c.x * sn + c.y * cs;
  }
  block_add2(sx, sy, out + 2 * s);
}

__global__ void __launch_bounds__(kDirectThreads)
    direct_type2_kernel(int dim, int sign, i64 n0, i64 n1, i64 n2, const double2* in, Loc3 x,
                        const i64* point_idx, double* out) {
  const i64 s = blockIdx.y;
  const i64 p = point_idx[s];
  double xp[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) xp[d] = x.p[d][p] * sign;
  const i64 total = n0 * n1 * n2;
  const i64 begin = i64(blockIdx.x) * kDirectChunk;
  const i64 end = min(total, begin + kDirectChunk);
  double sx = 0, sy = 0;
  for (i64 m = begin + threadIdx.x; m < end; m += kDirectThreads) {
    const i64 i0 = m % n0;
    const i64 r = m / n0;
    const i64 i1 = r % n1;
    const i64 i2 = r / n1;
    double ph = double(i0 - n0 / 2) * xp[0];
    if (dim > 1) ph += double(i1 - n1 / 2) * xp[1];
    if (dim > 2) ph += double(i2 - n2 / 2) * xp[2];
    double sn, cs;
    sincos(ph, &sn, &cs);
    const double2 c = in[m];
    sx += c.x * cs - c.y * sn;
    sy += c.x * sn + c.y * cs;
  }
  block_add2(sx, sy, out + 2 * s);
}

__global__ void __launch_bounds__(kDirectThreads)
    direct_type3_kernel(int dim, int sign, i64 M, Loc3 x, const double2* in, Loc3 t,
                        const i64* target_idx, double* out) {
  const i64 s = blockIdx.y;
  const i64 q = target_idx[s];
  double tq[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) tq[d] = t.p[d][q];
  const i64 begin = i64(blockIdx.x) * kDirectChunk;
  const i64 end = min(M, begin + kDirectChunk);
  double sx = 0, sy = 0;
  for (i64 j = begin + threadIdx.x; j < end; j += kDirectThreads) {
    double ph = x.p[0][j] * tq[0];
    if (dim > 1) ph += x.p[1][j] * tq[1];
    if (dim > 2) ph += x.p[2][j] * tq[2];
    ph *= sign;
    double sn, cs;
    sincos(ph, &sn, &cs);
    const double2 c = in[j];
    sx += c.x * cs - c.y * sn;
    sy += c.x * sn + c.y * cs;
  }
  block_add2(sx, sy, out + 2 * s);
}

Loc3 make_loc(int dim, const double* const* loc) {
  Loc3 l{{nullptr, nullptr, nullptr}};
  for (int d = 0; d < dim; ++d) l.p[d] = loc[d];
  return l;
}

void check_samples(i64 S) {
  if (S > 65535) throw_input("at most 65535 samples per direct-sum call");
}

}  // namespace

void launch_direct_type1(int dim, int sign, i64 M, const double* const* loc, const double* in,
                         i64 S, const i64* modes_idx, double* out, cudaStream_t stream) {
  check_samples(S);
  NNB_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * 2 * S, stream));
  if (S <= 0 || M <= 0) return;
  dim3 grid(unsigned((M + kDirectChunk - 1) / kDirectChunk), unsigned(S));
  direct_type1_kernel<<<grid, kDirectThreads, 0, stream>>>(
      dim, sign, M, make_loc(dim, loc), reinterpret_cast<const double2*>(in), modes_idx, out);
  NNB_LAUNCH_CHECK();
}

void launch_direct_type2(int dim, int sign, const i64* n_modes, const double* in,
                         const double* const* loc, i64 S, const i64* point_idx, double* out,
                         cudaStream_t stream) {
  check_samples(S);
  NNB_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * 2 * S, stream));
  const i64 n0 = n_modes[0], n1 = dim > 1 ? n_modes[1] : 1, n2 = dim > 2 ? n_modes[2] : 1;
  const i64 total = n0 * n1 * n2;
  if (S <= 0 || total <= 0) return;
  dim3 grid(unsigned((total + kDirectChunk - 1) / kDirectChunk), unsigned(S));
  direct_type2_kernel<<<grid, kDirectThreads, 0, stream>>>(
      dim, sign, n0, n1, n2, reinterpret_cast<const double2*>(in), make_loc(dim, loc), point_idx,
      out);
  NNB_LAUNCH_CHECK();
}

void launch_direct_type3(int dim, int sign, i64 M, const double* const* in_loc, const double* in,
                         const double* const* out_loc, i64 S, const i64* target_idx,
                         double* out, cudaStream_t stream) {
  check_samples(S);
  NNB_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * 2 * S, stream));
  if (S <= 0 || M <= 0) return;
  dim3 grid(unsigned((M + kDirectChunk - 1) / kDirectChunk), unsigned(S));
  direct_type3_kernel<<<grid, kDirectThreads, 0, stream>>>(
      dim, sign, M, make_loc(dim, in_loc), reinterpret_cast<const double2*>(in),
      make_loc(dim, out_loc), target_idx, out);
  NNB_LAUNCH_CHECK();
}

}  // namespace nnb
