// Point binning: rescale, tile histogram, exclusive scan, permutation.
//
// Replaces the reference's rescale_and_permut (src/neonufft/gpu/kernels/rescale_loc_kernel.cu:23-126,
// :185-209), which counts with one global atomic per point, assigns bin offsets from a single
// block in atomic (non-deterministic) order and scatters 24-32 byte Point structs with a second
// atomic per point. Here:
//  - the rescaling runs in double precision for every plan precision, and the point is stored
//    as its tile-local first kernel cell (packed integers) plus the fractional kernel argument
//    i0 - loc, so single-precision plans keep the full double-precision position;
//  - pass 1 records each point's rank inside its tile (the only atomic);
//  - a three-kernel device-wide exclusive scan gives tile offsets in tile order;
//  - pass 2 writes one 32-byte record per point (perm, packed cell, fractions), a full sector,
//    with no atomics, as one 256-bit evict-first store where the record array is 32-byte
//    aligned.
#include "kernels.cuh"

namespace nnb {

namespace {

constexpr int kBinBlock = 256;

// First kernel cell of one coordinate: i0 = ceil(loc - w/2) wrapped to [0, nf), and the
// kernel argument frac = i0 - loc in [-w/2, -w/2 + 1]. Returns false for non-finite input.
// The wrap runs on the integral double (exact below 2^53), and the cell index, below nf <= 2^31
// - 1 (make_geom), converts to a 32-bit int: no 64-bit integer arithmetic per point.
__device__ __forceinline__ bool cell_of(const BinGeom& g, int d, double x, int& i0w,
                                        double& frac) {
  const double v = (x - g.offset[d]) * g.scale[d];
  double p = (v + kPi) * kTwoPiInv;
  p = p - floor(p);
  const double nf = double(g.nf[d]);
  const double loc = p * nf;
  double s = ceil(loc - 0.5 * double(g.w));
  frac = s - loc;
  if (!(frac == frac) || !(fabs(frac) <= 16.0)) return false;
  while (s < 0.0) s += nf;
  while (s >= nf) s -= nf;
  i0w = __double2int_rz(s);
  return true;
}

// Quotient and remainder of a cell index by a tile extent (inv_t = 1 / t), from a double
// product and one correction step: for an index under 2^31 the product is off the true quotient
// by far less than one, so the truncated quotient is off by at most one either way. A 64-bit
// integer division here is a long instruction sequence, three per point, and made the binning
// scatter issue-bound.
__device__ __forceinline__ void tile_divmod(int i, int t, double inv_t, int& q, int& r) {
  q = __double2int_rz(double(i) * inv_t);
  r = int(i64(i) - i64(q) * t);
  if (r < 0) {
    --q;
    r += t;
  } else if (r >= t) {
    ++q;
    r -= t;
  }
}

// Points per thread and loop trip: the kernels are bound by memory latency (the coordinate
// loads, the rank atomic, the bin-offset gather), so each thread keeps kBinUnroll independent
// points in flight; point u of a trip is base + u * stride, so every load stays coalesced.
constexpr int kBinUnroll = 4;

// tile_linear with the dimension known at compile time (registers instead of a local array).
template <int DIM>
__device__ __forceinline__ i64 tile_linear_d(const BinGeom& g, const i64 (&t)[3]) {
  if (DIM == 3 && g.zmajor) return t[2] + i64(g.ntiles[2]) * (t[0] + i64(g.ntiles[0]) * t[1]);
  i64 lin = 0, mul = 1;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    lin += t[d] * mul;
    mul *= g.ntiles[d];
  }
  return lin;
}

template <typename T, int DIM>
__global__ void __launch_bounds__(kBinBlock)
    bin_count_kernel(BinGeom g, CoordPtrs<T> x, i64 M, u32* counts, u32* ranks, int* err) {
  const i64 stride = i64(gridDim.x) * kBinBlock;
  double inv_tile[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) inv_tile[d] = 1.0 / double(g.tile[d]);
  for (i64 base = blockIdx.x * i64(kBinBlock) + threadIdx.x; base < M;
       base += stride * kBinUnroll) {
    T v[kBinUnroll][DIM];
#pragma unroll
    for (int u = 0; u < kBinUnroll; ++u) {
      const i64 i = base + u * stride;
#pragma unroll
      for (int d = 0; d < DIM; ++d) v[u][d] = i < M ? x.p[d][i] : T(0);
    }
    i64 tile_lin[kBinUnroll];
#pragma unroll
    for (int u = 0; u < kBinUnroll; ++u) {
      i64 t[3] = {0, 0, 0};
      bool ok = true;
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        int i0 = 0, q, rem;
        double frac;
        ok &= cell_of(g, d, double(v[u][d]), i0, frac);
        tile_divmod(i0, g.tile[d], inv_tile[d], q, rem);
        t[d] = q;
      }
      tile_lin[u] = tile_linear_d<DIM>(g, t);
      if (!ok && base + u * stride < M) {
        atomicOr(err, 1);
        tile_lin[u] = 0;
      }
    }
    u32 r[kBinUnroll];
#pragma unroll
    for (int u = 0; u < kBinUnroll; ++u) {
      if (base + u * stride < M) {
        r[u] = NNB_CHECK_INDEX(tile_lin[u], g.total_tiles) ? atomicAdd(&counts[tile_lin[u]], 1u)
                                                           : 0u;
      }
    }
#pragma unroll
    for (int u = 0; u < kBinUnroll; ++u) {
      if (base + u * stride < M) ranks[base + u * stride] = r[u];
    }
  }
}

template <typename T, int DIM>
__global__ void __launch_bounds__(kBinBlock)
    bin_scatter_kernel(BinGeom g, CoordPtrs<T> x, i64 M, const u32* ranks, const u32* bin_start,
                       PointRec<T>* recs, bool wide) {
  const i64 stride = i64(gridDim.x) * kBinBlock;
  double inv_tile[DIM];
#pragma unroll
  for (int d = 0; d < DIM; ++d) inv_tile[d] = 1.0 / double(g.tile[d]);
  // The tile offsets (4 bytes per tile, read at random by every point) stay in the L2; the
  // records, written once to random slots and read only by the next kernels, leave it first.
  const unsigned long long keep = l2_evict_last_policy();
  const unsigned long long pass = l2_evict_first_policy();
  for (i64 base = blockIdx.x * i64(kBinBlock) + threadIdx.x; base < M;
       base += stride * kBinUnroll) {
    T v[kBinUnroll][DIM];
    u32 rank[kBinUnroll];
#pragma unroll
    for (int u = 0; u < kBinUnroll; ++u) {
      const i64 i = base + u * stride;
#pragma unroll
      for (int d = 0; d < DIM; ++d) v[u][d] = i < M ? x.p[d][i] : T(0);
      rank[u] = i < M ? ranks[i] : 0u;
    }
    PointRec<T> r[kBinUnroll];
    i64 tile_lin[kBinUnroll];
#pragma unroll
    for (int u = 0; u < kBinUnroll; ++u) {
      i64 t[3] = {0, 0, 0};
      int l[3] = {0, 0, 0};
      double fr[3] = {0, 0, 0};
      int i0[3] = {0, 0, 0};
      bool ok = true;
#pragma unroll
      for (int d = 0; d < DIM; ++d) ok &= cell_of(g, d, double(v[u][d]), i0[d], fr[d]);
      // A non-finite point went to tile 0 in pass 1 (the host then rejects the point set); it
      // must land in the same tile here so that its slot stays inside tile 0's range.
#pragma unroll
      for (int d = 0; d < DIM; ++d) {
        if (!ok) {
          i0[d] = 0;
          fr[d] = -0.5 * g.w;
        }
        int q;
        tile_divmod(i0[d], g.tile[d], inv_tile[d], q, l[d]);
        t[d] = q;
      }
      tile_lin[u] = tile_linear_d<DIM>(g, t);
      r[u].perm = u32(base + u * stride);
      r[u].local = (DIM == 3 && g.zmajor) ? pack_local_zmajor(l[0], l[1], i0[2])
                                          : pack_local(DIM, l[0], l[1], l[2]);
      r[u].frac[0] = T(fr[0]);
      r[u].frac[1] = T(fr[1]);
      r[u].frac[2] = T(fr[2]);
    }
    u32 pos[kBinUnroll];
#pragma unroll
    for (int u = 0; u < kBinUnroll; ++u) {
      if (base + u * stride < M) {
        pos[u] = NNB_CHECK_INDEX(tile_lin[u], g.total_tiles)
                     ? load_u32_policy(bin_start + tile_lin[u], keep) + rank[u]
                     : u32(M);
      }
    }
#pragma unroll
    for (int u = 0; u < kBinUnroll; ++u) {
      if (base + u * stride < M && NNB_CHECK_INDEX(pos[u], M)) {
        store_sector_policy(&recs[pos[u]], rec_sector(r[u]), wide, pass);
      }
    }
  }
}

// ---- exclusive scan ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanChunk = kScanThreads * kScanItems;

// Block-wide exclusive scan of one value per thread; returns the block total in *total.
template <int THREADS>
__device__ __forceinline__ u64 block_exclusive_scan(u64 v, u64* total) {
  __shared__ u64 warp_sums[THREADS / 32];
  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  u64 incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const u64 n = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += n;
  }
  if (lane == 31) warp_sums[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    u64 s = lane < THREADS / 32 ? warp_sums[lane] : 0;
    u64 si = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u64 n = __shfl_up_sync(0xffffffffu, si, o);
      if (lane >= o) si += n;
    }
    if (lane < THREADS / 32) warp_sums[lane] = si - s;  // exclusive warp offsets
    if (lane == THREADS / 32 - 1) *total = si;
  }
  __syncthreads();
  const u64 res = warp_sums[warp] + incl - v;
  __syncthreads();
  return res;
}

__global__ void __launch_bounds__(kScanThreads)
    scan_block_sums_kernel(const u32* in, i64 n, u32* block_sums) {
  const i64 base = i64(blockIdx.x) * kScanChunk + threadIdx.x * kScanItems;
  u64 s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) s += in[base + k];
  }
  __shared__ u64 total;
  block_exclusive_scan<kScanThreads>(s, &total);
  if (threadIdx.x == 0) block_sums[blockIdx.x] = u32(total);
}

__global__ void __launch_bounds__(kScanThreads) scan_top_kernel(u32* block_sums, i64 nb) {
  __shared__ u64 total;
  u64 carry = 0;
  for (i64 off = 0; off < nb; off += kScanChunk) {
    const i64 base = off + threadIdx.x * kScanItems;
    u32 v[kScanItems];
    u64 s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      v[k] = (base + k < nb) ? block_sums[base + k] : 0u;
      s += v[k];
    }
    u64 run = block_exclusive_scan<kScanThreads>(s, &total) + carry;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
      if (base + k < nb) block_sums[base + k] = u32(run);
      run += v[k];
    }
    __syncthreads();
    carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) block_sums[nb] = u32(carry);
}

__global__ void __launch_bounds__(kScanThreads)
    scan_apply_kernel(const u32* in, i64 n, const u32* block_offsets, i64 nb, u32* out) {
  const i64 base = i64(blockIdx.x) * kScanChunk + threadIdx.x * kScanItems;
  u32 v[kScanItems];
  u64 s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0u;
    s += v[k];
  }
  __shared__ u64 total;
  u64 run = block_exclusive_scan<kScanThreads>(s, &total) + block_offsets[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = u32(run);
    run += v[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = block_offsets[nb];
}

// Whether a record array starts on a 32-byte boundary (a user allocator may return less), so
// that its records take single 256-bit stores.
bool aligned32(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 31u) == 0; }

int grid_for(i64 n, int block) {
  i64 g = (n + block - 1) / block;
  const i64 cap = 148 * 32;  // grid-stride loops beyond this many blocks
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return int(g);
}

}  // namespace

template <typename T>
void launch_bin_count(const BinGeom& g, CoordPtrs<T> x, i64 M, u32* counts, u32* ranks,
                      int* err_flag, cudaStream_t stream) {
  if (M <= 0) return;
  const int grid = grid_for(M, kBinBlock);
  switch (g.dim) {
    case 1: bin_count_kernel<T, 1><<<grid, kBinBlock, 0, stream>>>(g, x, M, counts, ranks, err_flag); break;
    case 2: bin_count_kernel<T, 2><<<grid, kBinBlock, 0, stream>>>(g, x, M, counts, ranks, err_flag); break;
    default: bin_count_kernel<T, 3><<<grid, kBinBlock, 0, stream>>>(g, x, M, counts, ranks, err_flag); break;
  }
  NNB_LAUNCH_CHECK();
}

i64 scan_tmp_words(i64 n) { return (n + kScanChunk - 1) / kScanChunk + 1; }

void launch_exclusive_scan(const u32* counts, u32* out, i64 n, u32* tmp, cudaStream_t stream) {
  const i64 nb = (n + kScanChunk - 1) / kScanChunk;
  if (nb <= 0) return;
  scan_block_sums_kernel<<<unsigned(nb), kScanThreads, 0, stream>>>(counts, n, tmp);
  NNB_LAUNCH_CHECK();
  scan_top_kernel<<<1, kScanThreads, 0, stream>>>(tmp, nb);
  NNB_LAUNCH_CHECK();
  scan_apply_kernel<<<unsigned(nb), kScanThreads, 0, stream>>>(counts, n, tmp, nb, out);
  NNB_LAUNCH_CHECK();
}

template <typename T>
void launch_bin_scatter(const BinGeom& g, CoordPtrs<T> x, i64 M, const u32* ranks,
                        const u32* bin_start, PointRec<T>* rec, cudaStream_t stream) {
  if (M <= 0) return;
  const int grid = grid_for(M, kBinBlock);
  switch (g.dim) {
    case 1: bin_scatter_kernel<T, 1><<<grid, kBinBlock, 0, stream>>>(g, x, M, ranks, bin_start, rec, aligned32(rec)); break;
    case 2: bin_scatter_kernel<T, 2><<<grid, kBinBlock, 0, stream>>>(g, x, M, ranks, bin_start, rec, aligned32(rec)); break;
    default: bin_scatter_kernel<T, 3><<<grid, kBinBlock, 0, stream>>>(g, x, M, ranks, bin_start, rec, aligned32(rec)); break;
  }
  NNB_LAUNCH_CHECK();
}

template void launch_bin_count<float>(const BinGeom&, CoordPtrs<float>, i64, u32*, u32*, int*, cudaStream_t);
template void launch_bin_count<double>(const BinGeom&, CoordPtrs<double>, i64, u32*, u32*, int*, cudaStream_t);
// Permutation checksum of the bin-sorted records (checked build): sums of perm and perm^2
// (wrapping 64-bit) into sums[0], sums[1], to compare with those of 0 .. M - 1.
template <typename T>
__global__ void __launch_bounds__(kBinBlock)
    perm_checksum_kernel(const PointRec<T>* rec, i64 M, unsigned long long* sums) {
  unsigned long long s1 = 0, s2 = 0;
  for (i64 i = blockIdx.x * i64(kBinBlock) + threadIdx.x; i < M;
       i += i64(gridDim.x) * kBinBlock) {
    const unsigned long long p = rec[i].perm;
    s1 += p;
    s2 += p * p;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&sums[0], s1);
    atomicAdd(&sums[1], s2);
  }
}

template <typename T>
void launch_perm_checksum(const PointRec<T>* rec, i64 M, unsigned long long* sums,
                          cudaStream_t stream) {
  NNB_CUDA(cudaMemsetAsync(sums, 0, 2 * sizeof(unsigned long long), stream));
  if (M <= 0) return;
  i64 grid = (M + kBinBlock - 1) / kBinBlock;
  if (grid > 148 * 8) grid = 148 * 8;
  perm_checksum_kernel<T><<<unsigned(grid), kBinBlock, 0, stream>>>(rec, M, sums);
  NNB_LAUNCH_CHECK();
}
template void launch_perm_checksum<float>(const PointRec<float>*, i64, unsigned long long*,
                                          cudaStream_t);
template void launch_perm_checksum<double>(const PointRec<double>*, i64, unsigned long long*,
                                           cudaStream_t);

template void launch_bin_scatter<float>(const BinGeom&, CoordPtrs<float>, i64, const u32*, const u32*, PointRec<float>*, cudaStream_t);
template void launch_bin_scatter<double>(const BinGeom&, CoordPtrs<double>, i64, const u32*, const u32*, PointRec<double>*, cudaStream_t);

}  // namespace nnb
