// ES interpolation by shared-memory subproblem tiles.
//
// Replaces the reference's interpolation (src/neonufft/gpu/kernels/interpolation_kernel.cu:27-457),
// where each warp gathers its point's w^d cells straight from global memory in the user's
// point order. Here one CTA owns one tile: the tile plus its (w-1)-cell halo is staged once
// into shared memory (coalesced along x, periodic wrap), then each warp takes the tile's
// bin-sorted points one at a time: lanes evaluate the w*d kernel values, sweep the footprint
// in shared memory, and reduce with shuffles. The optional per-point factor (type-3 postphase)
// is applied before the result is written to the point's original position.
#include "kernels.cuh"

namespace nnb {

namespace {

constexpr int kInterpThreads = 256;
constexpr int kKerStride = 16;

template <int W, int DIM>
struct Footprint {
  static constexpr int cells = (DIM == 1) ? W : (DIM == 2 ? W * W : W * W * W);
};

template <typename T, int DIM, int W>
__global__ void __launch_bounds__(kInterpThreads) interp_tiles_kernel(InterpArgs<T> a) {
  using C = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];

  const BinGeom& g = a.g;
  const i64 bin = blockIdx.x;
  const u32 start = a.pts.bin_start[bin];
  const u32 end = a.pts.bin_start[bin + 1];
  if (start == end) return;

  const int P0 = g.tile[0] + W - 1;
  const int P1 = DIM > 1 ? g.tile[1] + W - 1 : 1;
  const int P2 = DIM > 2 ? g.tile[2] + W - 1 : 1;
  const int ncell = P0 * P1 * P2;

  C* tile = reinterpret_cast<C*>(smem_raw);
  T* kbuf = reinterpret_cast<T*>(tile + ncell);

  const i64 t0 = bin % g.ntiles[0];
  const i64 t1 = DIM > 1 ? (bin / g.ntiles[0]) % g.ntiles[1] : 0;
  const i64 t2 = DIM > 2 ? bin / (i64(g.ntiles[0]) * g.ntiles[1]) : 0;
  const i64 o0 = t0 * g.tile[0], o1 = t1 * g.tile[1], o2 = t2 * g.tile[2];

  for (int i = threadIdx.x; i < ncell; i += kInterpThreads) {
    const int cx = i % P0;
    const int r = i / P0;
    const int cy = r % P1;
    const int cz = r / P1;
    i64 gx = o0 + cx;
    while (gx >= g.nf[0]) gx -= g.nf[0];
    i64 gidx = gx;
    if (DIM > 1) {
      i64 gy = o1 + cy;
      while (gy >= g.nf[1]) gy -= g.nf[1];
      gidx += gy * g.nf[0];
    }
    if (DIM > 2) {
      i64 gz = o2 + cz;
      while (gz >= g.nf[2]) gz -= g.nf[2];
      gidx += gz * g.nf[0] * g.nf[1];
    }
    tile[i] = a.grid[gidx];
  }
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  constexpr int nwarps = kInterpThreads / 32;
  T* kv = kbuf + warp * (DIM * kKerStride);

  for (u32 p = start + warp; p < end; p += nwarps) {
    for (int j = lane; j < DIM * W; j += 32) {
      const int d = j / W;
      const int k = j - d * W;
      kv[d * kKerStride + k] = es_eval<T>(a.pts.frac[d][p] + T(k), a.beta, a.c);
    }
    int lx, ly, lz;
    unpack_local(DIM, a.pts.local[p], lx, ly, lz);
    __syncwarp();
    T sx = 0, sy = 0;
    for (int k = lane; k < Footprint<W, DIM>::cells; k += 32) {
      const int dx = k % W;
      const int r = k / W;
      const int dy = DIM > 1 ? r % W : 0;
      const int dz = DIM > 2 ? r / W : 0;
      T kval = kv[dx];
      if (DIM > 1) kval *= kv[kKerStride + dy];
      if (DIM > 2) kval *= kv[2 * kKerStride + dz];
      const C gv = tile[((lz + dz) * P1 + (ly + dy)) * P0 + (lx + dx)];
      sx += kval * gv.x;
      sy += kval * gv.y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sx += __shfl_xor_sync(0xffffffffu, sx, o);
      sy += __shfl_xor_sync(0xffffffffu, sy, o);
    }
    if (lane == 0) {
      const u32 idx = a.pts.perm[p];
      C res{sx, sy};
      if (a.postphase) res = cmul(res, a.postphase[idx]);
      a.out[idx] = res;
    }
    __syncwarp();
  }
}

template <typename T, int DIM, int W>
void launch_interp_tw(const InterpArgs<T>& a, cudaStream_t stream) {
  const int P0 = a.g.tile[0] + W - 1;
  const int P1 = DIM > 1 ? a.g.tile[1] + W - 1 : 1;
  const int P2 = DIM > 2 ? a.g.tile[2] + W - 1 : 1;
  const size_t smem = size_t(P0) * P1 * P2 * sizeof(cplx_t<T>) +
                      size_t(kInterpThreads / 32) * DIM * kKerStride * sizeof(T);
  if (smem > 227 * 1024) throw_internal("interpolation tile does not fit in shared memory");
  auto kern = interp_tiles_kernel<T, DIM, W>;
  NNB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  kern<<<unsigned(a.g.total_tiles), kInterpThreads, smem, stream>>>(a);
  NNB_LAUNCH_CHECK();
}

template <typename T, int DIM>
void launch_interp_d(const InterpArgs<T>& a, cudaStream_t stream) {
  switch (a.g.w) {
    case 2: return launch_interp_tw<T, DIM, 2>(a, stream);
    case 3: return launch_interp_tw<T, DIM, 3>(a, stream);
    case 4: return launch_interp_tw<T, DIM, 4>(a, stream);
    case 5: return launch_interp_tw<T, DIM, 5>(a, stream);
    case 6: return launch_interp_tw<T, DIM, 6>(a, stream);
    case 7: return launch_interp_tw<T, DIM, 7>(a, stream);
    case 8: return launch_interp_tw<T, DIM, 8>(a, stream);
    case 9: return launch_interp_tw<T, DIM, 9>(a, stream);
    case 10: return launch_interp_tw<T, DIM, 10>(a, stream);
    case 11: return launch_interp_tw<T, DIM, 11>(a, stream);
    case 12: return launch_interp_tw<T, DIM, 12>(a, stream);
    case 13: return launch_interp_tw<T, DIM, 13>(a, stream);
    case 14: return launch_interp_tw<T, DIM, 14>(a, stream);
    case 15: return launch_interp_tw<T, DIM, 15>(a, stream);
    case 16: return launch_interp_tw<T, DIM, 16>(a, stream);
    default: throw_internal("n_spread not in [2, 16]");
  }
}

}  // namespace

template <typename T>
void launch_interp(const InterpArgs<T>& a, cudaStream_t stream) {
  if (a.g.total_tiles <= 0) return;
  switch (a.g.dim) {
    case 1: return launch_interp_d<T, 1>(a, stream);
    case 2: return launch_interp_d<T, 2>(a, stream);
    case 3: return launch_interp_d<T, 3>(a, stream);
    default: throw_internal("invalid dimension");
  }
}

template void launch_interp<float>(const InterpArgs<float>&, cudaStream_t);
template void launch_interp<double>(const InterpArgs<double>&, cudaStream_t);

}  // namespace nnb
