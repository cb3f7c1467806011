// FP64 direct type-1 sum for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: code running inside a memory pool that owns the whole
// device, applications that forbid allocation after start-up, or host code invoked where an
// allocation would implicitly synchronise the device. This entry point computes the same
// sampled sums as nnb_direct_type1_f64 (direct.cu) without allocating anything: each block
// writes its partial sum into a fixed scratch array that lives in the library's own device
// memory (a file-scope __device__ array, present on every GPU that loads the library until the
// process exits), and a second kernel adds the partial sums of each sample in a fixed order.
//
// The scratch holds kNoAllocMaxPartials partial sums, i.e. num_samples * ceil(num_nu / 4096)
// must not exceed 1,048,576 (16 MiB of double2); larger requests fail with an input error.
// All calls share the one array and every partial sum a call reads is written by that same
// call, so no clearing is needed; two calls that overlap on the GPU (different streams or host
// threads without ordering between them) race on the array and must be avoided.
// The first call on each device looks up the array's device address (cudaGetSymbolAddress,
// with that device current) and caches it; make that first call before any stream capture.
#include <mutex>

#include "kernels.cuh"
#include "neonufft_gpu.h"

namespace nnb {

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaChunk = kNaThreads * 16;
constexpr long long kNoAllocMaxPartials = 1ll << 20;

// The scratch array. In host code its name is only a stand-in for the device symbol; kernels
// receive the device address obtained from cudaGetSymbolAddress.
static __device__ __align__(256) double2 g_noalloc_partials[kNoAllocMaxPartials];

struct Loc3 {
  const double* p[3];
};

__global__ void __launch_bounds__(kNaThreads)
    noalloc_partials_kernel(int dim, int sign, i64 M, Loc3 x, const double2* in,
                            const i64* modes_idx, i64 chunks, double2* partials) {
  const i64 s = blockIdx.y;
  double k[3] = {0, 0, 0};
  for (int d = 0; d < dim; ++d) k[d] = double(modes_idx[s * dim + d]) * sign;
  const i64 begin = i64(blockIdx.x) * kNaChunk;
  const i64 end = min(M, begin + kNaChunk);
  double sx = 0, sy = 0;
  for (i64 j = begin + threadIdx.x; j < end; j += kNaThreads) {
    double ph = k[0] * x.p[0][j];
    if (dim > 1) ph += k[1] * x.p[1][j];
    if (dim > 2) ph += k[2] * x.p[2][j];
    double sn, cs;
    sincos(ph, &sn, &cs);
    const double2 c = in[j];
    sx += c.x * cs - c.y * sn;
    sy += c.x * sn + c.y * cs;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
  }
  __shared__ double red[2][kNaThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = sx;
    red[1][warp] = sy;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < kNaThreads / 32; ++w) {
      a += red[0][w];
      b += red[1][w];
    }
    partials[s * chunks + blockIdx.x] = double2{a, b};
  }
}

__global__ void __launch_bounds__(kNaThreads)
    noalloc_reduce_kernel(i64 chunks, const double2* partials, double* out) {
  const i64 s = blockIdx.x;
  double sx = 0, sy = 0;
  for (i64 c = threadIdx.x; c < chunks; c += kNaThreads) {
    const double2 v = partials[s * chunks + c];
    sx += v.x;
    sy += v.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    sx += __shfl_xor_sync(0xffffffffu, sx, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
  }
  __shared__ double red[2][kNaThreads / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = sx;
    red[1][warp] = sy;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < kNaThreads / 32; ++w) {
      a += red[0][w];
      b += red[1][w];
    }
    out[2 * s] = a;
    out[2 * s + 1] = b;
  }
}

// Device address of the scratch array on the current device, resolved once per device.
double2* scratch_on_current_device() {
  static std::mutex mu;
  static double2* addr[64] = {nullptr};
  int dev = 0;
  NNB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw_internal("device index out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    NNB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_partials));
    addr[dev] = static_cast<double2*>(p);
  }
  return addr[dev];
}

}  // namespace

void launch_direct_type1_noalloc(int dim, int sign, i64 M, const double* const* loc,
                                 const double* in, i64 S, const i64* modes_idx, double* out,
                                 cudaStream_t stream) {
  if (S > 65535) throw_input("at most 65535 samples per direct-sum call");
  if (S <= 0) return;
  const i64 chunks = (M + kNaChunk - 1) / kNaChunk;
  if (chunks > kNoAllocMaxPartials / S) {
    throw_input("num_samples * ceil(num_nu / 4096) exceeds the 1048576 partial sums of the "
                "fixed scratch");
  }
  double2* partials = scratch_on_current_device();
  if (chunks > 0) {
    Loc3 l{{nullptr, nullptr, nullptr}};
    for (int d = 0; d < dim; ++d) l.p[d] = loc[d];
    const dim3 grid{unsigned(chunks), unsigned(S), 1u};
    noalloc_partials_kernel<<<grid, kNaThreads, 0, stream>>>(
        dim, sign, M, l, reinterpret_cast<const double2*>(in), modes_idx, chunks, partials);
    NNB_LAUNCH_CHECK();
  }
  noalloc_reduce_kernel<<<unsigned(S), kNaThreads, 0, stream>>>(chunks, partials, out);
  NNB_LAUNCH_CHECK();
}

}  // namespace nnb
