// ES spreading by shared-memory subproblem tiles.
//
// Replaces the reference's atomic spreading (src/neonufft/gpu/kernels/spreading_kernel.cu:477-715),
// which issues 2 * w^d global float atomics per point. Here one CTA owns one tile of the fine
// grid plus its (w-1)-cell halo in shared memory:
//   1. the tile's bin-sorted points are read in order (coalesced SoA records);
//   2. each warp takes one point at a time: lanes evaluate the w*d kernel values once, then the
//      warp's lanes sweep the w^d footprint and accumulate c * kx * ky * kz into shared memory;
//   3. the padded tile is added to the global grid once, coalesced along x, with vector
//      float2/double2 atomics only for cells that received contributions (halos of neighbouring
//      tiles overlap, so the add must be atomic).
// Global atomic traffic is thus O(tile + halo) per tile instead of O(w^d) per point.
#include "kernels.cuh"

namespace nnb {

namespace {

constexpr int kSpreadThreads = 256;
constexpr int kKerStride = 16;  // per-warp kernel value buffer: [DIM][16]

template <int W, int DIM>
struct Footprint {
  static constexpr int cells = (DIM == 1) ? W : (DIM == 2 ? W * W : W * W * W);
};

__device__ __forceinline__ void atomic_add_cplx(float2* p, float2 v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_cplx(double2* p, double2 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
}

template <typename T, int DIM, int W>
__global__ void __launch_bounds__(kSpreadThreads) spread_tiles_kernel(SpreadArgs<T> a) {
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

  C* acc = reinterpret_cast<C*>(smem_raw);
  T* kbuf = reinterpret_cast<T*>(acc + ncell);

  const int batch = blockIdx.y;
  const C* in = a.in + batch * a.in_bdist;
  C* grid = a.grid + batch * a.grid_bdist;

  for (int i = threadIdx.x; i < ncell; i += kSpreadThreads) acc[i] = C{T(0), T(0)};
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  constexpr int nwarps = kSpreadThreads / 32;
  T* kv = kbuf + warp * (DIM * kKerStride);

  for (u32 p = start + warp; p < end; p += nwarps) {
    const u32 idx = a.pts.perm[p];
    for (int j = lane; j < DIM * W; j += 32) {
      const int d = j / W;
      const int k = j - d * W;
      kv[d * kKerStride + k] = es_eval<T>(a.pts.frac[d][p] + T(k), a.beta, a.c);
    }
    C v = in[idx];
    if (a.prephase) v = cmul(v, a.prephase[idx]);
    int lx, ly, lz;
    unpack_local(DIM, a.pts.local[p], lx, ly, lz);
    __syncwarp();
    for (int k = lane; k < Footprint<W, DIM>::cells; k += 32) {
      const int dx = k % W;
      const int r = k / W;
      const int dy = DIM > 1 ? r % W : 0;
      const int dz = DIM > 2 ? r / W : 0;
      T kval = kv[dx];
      if (DIM > 1) kval *= kv[kKerStride + dy];
      if (DIM > 2) kval *= kv[2 * kKerStride + dz];
      const int cell = ((lz + dz) * P1 + (ly + dy)) * P0 + (lx + dx);
      atomicAdd(&acc[cell].x, kval * v.x);
      atomicAdd(&acc[cell].y, kval * v.y);
    }
    __syncwarp();
  }
  __syncthreads();

  // Tile origin and periodic writeback.
  const i64 t0 = bin % g.ntiles[0];
  const i64 t1 = DIM > 1 ? (bin / g.ntiles[0]) % g.ntiles[1] : 0;
  const i64 t2 = DIM > 2 ? bin / (i64(g.ntiles[0]) * g.ntiles[1]) : 0;
  const i64 o0 = t0 * g.tile[0], o1 = t1 * g.tile[1], o2 = t2 * g.tile[2];
  for (int i = threadIdx.x; i < ncell; i += kSpreadThreads) {
    const C val = acc[i];
    if (val.x == T(0) && val.y == T(0)) continue;
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
    atomic_add_cplx(&grid[gidx], val);
  }
}

template <typename T, int DIM, int W>
void launch_spread_tw(const SpreadArgs<T>& a, cudaStream_t stream) {
  const int P0 = a.g.tile[0] + W - 1;
  const int P1 = DIM > 1 ? a.g.tile[1] + W - 1 : 1;
  const int P2 = DIM > 2 ? a.g.tile[2] + W - 1 : 1;
  const size_t smem = size_t(P0) * P1 * P2 * sizeof(cplx_t<T>) +
                      size_t(kSpreadThreads / 32) * DIM * kKerStride * sizeof(T);
  auto kern = spread_tiles_kernel<T, DIM, W>;
  if (smem > 227 * 1024) throw_internal("spread tile does not fit in shared memory");
  // Per device and cheap; set on every launch so that multi-device processes stay correct.
  NNB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  if (a.batch > 65535) throw_input("batch size above 65535");
  dim3 grid(unsigned(a.g.total_tiles), unsigned(a.batch), 1);
  kern<<<grid, kSpreadThreads, smem, stream>>>(a);
  NNB_LAUNCH_CHECK();
}

template <typename T, int DIM>
void launch_spread_d(const SpreadArgs<T>& a, cudaStream_t stream) {
  switch (a.g.w) {
    case 2: return launch_spread_tw<T, DIM, 2>(a, stream);
    case 3: return launch_spread_tw<T, DIM, 3>(a, stream);
    case 4: return launch_spread_tw<T, DIM, 4>(a, stream);
    case 5: return launch_spread_tw<T, DIM, 5>(a, stream);
    case 6: return launch_spread_tw<T, DIM, 6>(a, stream);
    case 7: return launch_spread_tw<T, DIM, 7>(a, stream);
    case 8: return launch_spread_tw<T, DIM, 8>(a, stream);
    case 9: return launch_spread_tw<T, DIM, 9>(a, stream);
    case 10: return launch_spread_tw<T, DIM, 10>(a, stream);
    case 11: return launch_spread_tw<T, DIM, 11>(a, stream);
    case 12: return launch_spread_tw<T, DIM, 12>(a, stream);
    case 13: return launch_spread_tw<T, DIM, 13>(a, stream);
    case 14: return launch_spread_tw<T, DIM, 14>(a, stream);
    case 15: return launch_spread_tw<T, DIM, 15>(a, stream);
    case 16: return launch_spread_tw<T, DIM, 16>(a, stream);
    default: throw_internal("n_spread not in [2, 16]");
  }
}

}  // namespace

template <typename T>
void launch_spread(const SpreadArgs<T>& a, cudaStream_t stream) {
  if (a.g.total_tiles <= 0 || a.batch <= 0) return;
  switch (a.g.dim) {
    case 1: return launch_spread_d<T, 1>(a, stream);
    case 2: return launch_spread_d<T, 2>(a, stream);
    case 3: return launch_spread_d<T, 3>(a, stream);
    default: throw_internal("invalid dimension");
  }
}

template void launch_spread<float>(const SpreadArgs<float>&, cudaStream_t);
template void launch_spread<double>(const SpreadArgs<double>&, cudaStream_t);

}  // namespace nnb
