// ES spreading by shared-memory subproblem slabs.
//
// Replaces the reference's atomic spreading (src/neonufft/gpu/kernels/spreading_kernel.cu:477-715),
// which issues 2 w^d global float atomics per point.
//
// Method 1 (default), warp-private slabs:
//  * A CTA of up to 4 warps covers as many consecutive tiles (bins) along the last dimension;
//    each warp owns one tile and a private shared-memory slab holding that tile plus its
//    (w-1)-cell halo (padded strides chosen to spread lanes over the banks, tile_layout.cuh).
//  * The warp walks its tile's bin-sorted points in batches of 32: lane j loads point j's
//    record and strength and evaluates its w*d kernel values into a per-warp buffer (all lanes
//    in parallel, one memory latency per batch); then, one point at a time, lane r takes
//    footprint row r (3D: (dy, dz), 2D: cell (dx, dy)) and adds c * ky * kz * kx[dx] along the
//    row with plain shared-memory read-modify-write (all loads of a point first, then the
//    FMAs, then the stores). Lanes of one warp never touch the same cell for one point and no
//    other warp touches the slab, so no atomics are needed (shared-memory float atomics are a
//    compare-and-swap loop on this GPU, ~10x slower than plain read-modify-write).
//  * After a block barrier, slab w's upper halo is added into slab w+1 (in order), and the CTA
//    region is added to the global grid once, coalesced along x, with float2/double2 atomics
//    (regions of neighbouring CTAs overlap by the halo).
// Method 2, thread per point with shared-memory atomics, is kept as an alternative.
#include <type_traits>

#include "kernels.cuh"
#include "tile_layout.cuh"

namespace nnb {

namespace {

constexpr int kMaxSlabWarps = 4;  // warps (tiles) per CTA; fewer when the slabs do not fit
constexpr int kTppThreads = 256;

__device__ __forceinline__ void atomic_add_cplx(float2* p, float2 v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_cplx(double2* p, double2 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
}

template <typename T>
__device__ __forceinline__ void zero_cells(cplx_t<T>* p, int n, int tid, int nthreads) {
  // n is even and p 16-byte aligned: 16-byte stores
  float4* q = reinterpret_cast<float4*>(p);
  const int n16 = n * int(sizeof(cplx_t<T>)) / 16;
  for (int i = tid; i < n16; i += nthreads) q[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

// Adds the first `nrows` rows (x < P0) of a padded slab region to the global grid.
template <typename T, int DIM>
__device__ __forceinline__ void writeback_rows(const BinGeom& g, const TileLayout& L,
                                               const cplx_t<T>* slab, int nrows, i64 o0, i64 o1,
                                               i64 o2, cplx_t<T>* grid, int warp, int nwarps,
                                               int lane) {
  for (int row = warp; row < nrows; row += nwarps) {
    int cy = 0, cz = 0;
    if (DIM == 3) {
      cz = row / L.P1;
      cy = row - cz * L.P1;
    } else {
      cy = row;
    }
    const cplx_t<T>* src = slab + cz * L.PS + cy * L.RS;
    i64 rbase = wrap_index(o1 + cy, g.nf[1]) * g.nf[0];
    if (DIM > 2) rbase += wrap_index(o2 + cz, g.nf[2]) * g.nf[0] * g.nf[1];
    for (int cx = lane; cx < L.P0; cx += 32) {
      const cplx_t<T> val = src[cx];
      if (val.x == T(0) && val.y == T(0)) continue;
      const i64 gi = rbase + wrap_index(o0 + cx, g.nf[0]);
      if (NNB_CHECK_INDEX(gi, g.nf[0] * g.nf[1] * g.nf[2])) atomic_add_cplx(&grid[gi], val);
    }
  }
}

template <typename T, int DIM, int W>
__global__ void __launch_bounds__(kMaxSlabWarps * 32) spread_slab_kernel(SpreadArgs<T> a,
                                                                         TileLayout L,
                                                                         WorkList wl) {
  using C = cplx_t<T>;
  const int nwarps = blockDim.x >> 5;
  constexpr int KS = (DIM * W) | 1;  // odd stride: lanes write their rows without conflicts
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* slabs = reinterpret_cast<C*>(smem_raw);
  T* kbuf = reinterpret_cast<T*>(slabs + nwarps * L.cells);  // [warps][32][KS]

  const BinGeom& g = a.g;
  constexpr int LD = DIM - 1;  // slabs are stacked along the last dimension
  const int n_last = g.ntiles[LD];
  const int groups = (n_last + nwarps - 1) / nwarps;
  u32 unit, slice;
  if (!work_item(wl, unit, slice)) return;
  const i64 rest = unit / groups;
  const int grp = int(unit - rest * groups);
  int tc[3] = {0, 0, 0};  // tile coordinates of warp 0
  {
    i64 r = rest;
    for (int d = 0; d < LD; ++d) {
      tc[d] = int(r % g.ntiles[d]);
      r /= g.ntiles[d];
    }
    tc[LD] = grp * nwarps;
  }
  int nvalid = n_last - tc[LD];
  if (nvalid > nwarps) nvalid = nwarps;

  const int batch = blockIdx.y;
  const C* in = a.in + batch * a.in_bdist;
  C* grid = a.grid + batch * a.grid_bdist;

  auto bin_of = [&](int t_last) -> i64 {
    if (DIM == 1) return t_last;
    if (DIM == 2) return tc[0] + i64(g.ntiles[0]) * t_last;
    return tc[0] + i64(g.ntiles[0]) * (tc[1] + i64(g.ntiles[1]) * t_last);
  };
  // This CTA's slice of each tile's points; CTAs without points contribute nothing.
  bool any = false;
  for (int w = 0; w < nvalid; ++w) {
    const i64 b = bin_of(tc[LD] + w);
    u32 s0, s1;
    work_slice(a.pts.bin_start[b], a.pts.bin_start[b + 1], slice, wl.cap, s0, s1);
    any |= s1 > s0;
  }
  if (!any) return;

  zero_cells<T>(slabs, nwarps * L.cells, threadIdx.x, blockDim.x);
  __syncthreads();

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  if (warp < nvalid) {
    const i64 bin = bin_of(tc[LD] + warp);
    u32 start, end;
    work_slice(a.pts.bin_start[bin], a.pts.bin_start[bin + 1], slice, wl.cap, start, end);
    C* slab = slabs + warp * L.cells;
    T* kvb = kbuf + warp * 32 * KS;

    // Lane-constant footprint rows: 3D rows r = dy + W dz, 2D cells r = dx + W dy.
    constexpr int NR = (DIM == 1) ? W : W * W;
    constexpr int PASSES = (NR + 31) / 32;
    int roff[PASSES], ra[PASSES], rb[PASSES];
#pragma unroll
    for (int k = 0; k < PASSES; ++k) {
      const int r = lane + 32 * k;
      ra[k] = r % W;
      rb[k] = r / W;
      if (DIM == 3) roff[k] = rb[k] * L.PS + ra[k] * L.RS;
      else if (DIM == 2) roff[k] = rb[k] * L.RS + ra[k];
      else roff[k] = r;
    }

    for (u32 b = start; b < end; b += 32) {
      const u32 nb = (end - b) < 32u ? (end - b) : 32u;
      int my_base = 0;
      C my_v{T(0), T(0)};
      if (lane < nb && NNB_CHECK_INDEX(i64(b) + lane, a.pts.M)) {
        const PointRec<T> rec = a.pts.rec[b + lane];
        const u32 idx = rec.perm;
        if (NNB_CHECK_INDEX(idx, a.pts.M)) {
          my_v = in[idx];
          if (a.prephase) my_v = cmul(my_v, a.prephase[idx]);
        }
        int lx, ly, lz;
        unpack_local(DIM, rec.local, lx, ly, lz);
        my_base = lz * L.PS + ly * L.RS + lx;
        T* kr = kvb + lane * KS;
#pragma unroll
        for (int d = 0; d < DIM; ++d) {
          const T f = rec.frac[d];
#pragma unroll
          for (int k = 0; k < W; ++k) kr[d * W + k] = es_eval_fast<T>(f + T(k), a.beta, a.c);
        }
      }
      __syncwarp();
      for (u32 j = 0; j < nb; ++j) {
        const int base = __shfl_sync(0xffffffffu, my_base, int(j));
        const T vx0 = __shfl_sync(0xffffffffu, my_v.x, int(j));
        const T vy0 = __shfl_sync(0xffffffffu, my_v.y, int(j));
        const T* kj = kvb + j * KS;
        if (DIM == 3) {
          T kx[W];
#pragma unroll
          for (int k = 0; k < W; ++k) kx[k] = kj[k];
          constexpr bool kAllRows = PASSES * W <= 32;  // whole footprint share in registers
          if (kAllRows) {
            C cell[PASSES][W];
            T vx[PASSES], vy[PASSES];
#pragma unroll
            for (int k = 0; k < PASSES; ++k) {
              if (lane + 32 * k < NR) {
                const C* row = slab + base + roff[k];
#pragma unroll
                for (int dx = 0; dx < W; ++dx) cell[k][dx] = row[dx];
                const T kyz = kj[W + ra[k]] * kj[2 * W + rb[k]];
                vx[k] = vx0 * kyz;
                vy[k] = vy0 * kyz;
              }
            }
#pragma unroll
            for (int k = 0; k < PASSES; ++k) {
              if (lane + 32 * k < NR) {
                C* row = slab + base + roff[k];
#pragma unroll
                for (int dx = 0; dx < W; ++dx) {
                  cell[k][dx].x += kx[dx] * vx[k];
                  cell[k][dx].y += kx[dx] * vy[k];
                  row[dx] = cell[k][dx];
                }
              }
            }
          } else {
#pragma unroll
            for (int k = 0; k < PASSES; ++k) {
              if (lane + 32 * k < NR) {
                const T kyz = kj[W + ra[k]] * kj[2 * W + rb[k]];
                const T vx = vx0 * kyz, vy = vy0 * kyz;
                C* row = slab + base + roff[k];
                C cell[W];
#pragma unroll
                for (int dx = 0; dx < W; ++dx) cell[dx] = row[dx];
#pragma unroll
                for (int dx = 0; dx < W; ++dx) {
                  cell[dx].x += kx[dx] * vx;
                  cell[dx].y += kx[dx] * vy;
                  row[dx] = cell[dx];
                }
              }
            }
          }
        } else if (DIM == 2) {
          C cell[PASSES];
          T kk[PASSES];
#pragma unroll
          for (int k = 0; k < PASSES; ++k) {
            if (lane + 32 * k < NR) {
              cell[k] = slab[base + roff[k]];
              kk[k] = kj[ra[k]] * kj[W + rb[k]];
            }
          }
#pragma unroll
          for (int k = 0; k < PASSES; ++k) {
            if (lane + 32 * k < NR) {
              cell[k].x += kk[k] * vx0;
              cell[k].y += kk[k] * vy0;
              slab[base + roff[k]] = cell[k];
            }
          }
        } else {
          if (lane < W) {
            const T kk = kj[lane];
            C* cell = slab + base + lane;
            C c = *cell;
            c.x += kk * vx0;
            c.y += kk * vy0;
            *cell = c;
          }
        }
        __syncwarp();
      }
    }
  }
  __syncthreads();

  // Fold each slab's upper halo (last-dim index >= T_last) into the next slab, in order.
  const int T_last = g.tile[LD];
  constexpr int H = W - 1;
  const int plane_cells = (DIM == 3) ? L.PS : (DIM == 2 ? L.RS : 1);
  const int plane_count = (DIM == 3) ? L.RS * L.P1 : (DIM == 2 ? L.P0 : 1);
  for (int w = 1; w < nvalid; ++w) {
    C* dst = slabs + w * L.cells;
    const C* src = slabs + (w - 1) * L.cells + T_last * plane_cells;
    for (int pl = 0; pl < H; ++pl) {
      for (int q = threadIdx.x; q < plane_count; q += blockDim.x) {
        const C s = src[pl * plane_cells + q];
        C d = dst[pl * plane_cells + q];
        d.x += s.x;
        d.y += s.y;
        dst[pl * plane_cells + q] = d;
      }
    }
    __syncthreads();
  }

  // Write back: slab w adds its owned planes [0, T_last); the last valid slab also its halo.
  const i64 o0 = i64(tc[0]) * g.tile[0];
  const i64 o1 = DIM > 1 ? i64(tc[1]) * g.tile[1] : 0;
  const i64 o2 = DIM > 2 ? i64(tc[2]) * g.tile[2] : 0;
  for (int w = 0; w < nvalid; ++w) {
    const C* slab = slabs + w * L.cells;
    const int planes = (w == nvalid - 1) ? T_last + H : T_last;
    if (DIM == 3) {
      writeback_rows<T, 3>(g, L, slab, planes * L.P1, o0, o1, o2 + i64(w) * T_last, grid, warp,
                           nwarps, lane);
    } else if (DIM == 2) {
      writeback_rows<T, 2>(g, L, slab, planes, o0, o1 + i64(w) * T_last, 0, grid, warp, nwarps,
                           lane);
    } else {
      const i64 ox = o0 + i64(w) * T_last;
      for (int cx = threadIdx.x; cx < planes; cx += blockDim.x) {
        const C val = slab[cx];
        if (val.x == T(0) && val.y == T(0)) continue;
        const i64 gi = wrap_index(ox + cx, g.nf[0]);
        if (NNB_CHECK_INDEX(gi, g.nf[0])) atomic_add_cplx(&grid[gi], val);
      }
    }
  }
}

// Thread-per-point variant with shared-memory atomics on one padded tile per CTA.
template <typename T, int DIM, int W>
__global__ void __launch_bounds__(kTppThreads) spread_tpp_kernel(SpreadArgs<T> a, TileLayout L,
                                                                  WorkList wl) {
  using C = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const BinGeom& g = a.g;
  u32 unit, slice;
  if (!work_item(wl, unit, slice)) return;
  const i64 bin = unit;
  u32 start, end;
  work_slice(a.pts.bin_start[bin], a.pts.bin_start[bin + 1], slice, wl.cap, start, end);
  if (start == end) return;
  C* acc = reinterpret_cast<C*>(smem_raw);
  T* accf = reinterpret_cast<T*>(smem_raw);
  const int batch = blockIdx.y;
  const C* in = a.in + batch * a.in_bdist;
  C* grid = a.grid + batch * a.grid_bdist;
  zero_cells<T>(acc, L.cells, threadIdx.x, kTppThreads);
  __syncthreads();

  for (u32 p = start + threadIdx.x; p < end; p += kTppThreads) {
    if (!NNB_CHECK_INDEX(p, a.pts.M)) break;
    const PointRec<T> rec = a.pts.rec[p];
    const u32 idx = rec.perm;
    if (!NNB_CHECK_INDEX(idx, a.pts.M)) continue;
    C v = in[idx];
    if (a.prephase) v = cmul(v, a.prephase[idx]);
    int lx, ly, lz;
    unpack_local(DIM, rec.local, lx, ly, lz);
    T kx[W];
    const T fx = rec.frac[0];
#pragma unroll
    for (int k = 0; k < W; ++k) kx[k] = es_eval_fast<T>(fx + T(k), a.beta, a.c);
    const T fy = DIM > 1 ? rec.frac[1] : T(0);
    const T fz = DIM > 2 ? rec.frac[2] : T(0);
    const int nz = DIM > 2 ? W : 1;
    const int ny = DIM > 1 ? W : 1;
#pragma unroll 1
    for (int dz = 0; dz < nz; ++dz) {
      const T kz = DIM > 2 ? es_eval_fast<T>(fz + T(dz), a.beta, a.c) : T(1);
#pragma unroll 1
      for (int dy = 0; dy < ny; ++dy) {
        const T ky = (DIM > 1 ? es_eval_fast<T>(fy + T(dy), a.beta, a.c) : T(1)) * kz;
        const T vx = v.x * ky, vy = v.y * ky;
        const int row = (lz + dz) * L.PS + (ly + dy) * L.RS + lx;
#pragma unroll
        for (int dx = 0; dx < W; ++dx) {
          atomicAdd(&accf[2 * (row + dx)], kx[dx] * vx);
          atomicAdd(&accf[2 * (row + dx) + 1], kx[dx] * vy);
        }
      }
    }
  }
  __syncthreads();

  const i64 t0 = bin % g.ntiles[0];
  const i64 t1 = DIM > 1 ? (bin / g.ntiles[0]) % g.ntiles[1] : 0;
  const i64 t2 = DIM > 2 ? bin / (i64(g.ntiles[0]) * g.ntiles[1]) : 0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (DIM == 1) {
    for (int cx = threadIdx.x; cx < L.P0; cx += kTppThreads) {
      const C val = acc[cx];
      if (val.x == T(0) && val.y == T(0)) continue;
      const i64 gi = wrap_index(t0 * g.tile[0] + cx, g.nf[0]);
      if (NNB_CHECK_INDEX(gi, g.nf[0])) atomic_add_cplx(&grid[gi], val);
    }
  } else {
    writeback_rows<T, DIM>(g, L, acc, L.P1 * L.P2, t0 * g.tile[0], t1 * g.tile[1],
                           t2 * g.tile[2], grid, warp, kTppThreads / 32, lane);
  }
}

template <typename T, int DIM, int W>
void launch_spread_tw(const SpreadArgs<T>& a, cudaStream_t stream) {
  if (a.batch > 65535) throw_input("batch size above 65535");
  const TileLayout L = make_tile_layout(DIM, W, a.g.tile[0], a.g.tile[1], a.g.tile[2],
                                        int(sizeof(cplx_t<T>)));
  if (a.method == 2) {
    const size_t smem = size_t(L.cells) * sizeof(cplx_t<T>);
    if (smem > 227 * 1024) throw_internal("spread tile does not fit in shared memory");
    auto kern = spread_tpp_kernel<T, DIM, W>;
    NNB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    UnitMap m{};
    m.kind = UnitMap::kTile;
    m.units = a.g.total_tiles;
    const WorkList wl = build_work_list(m, a.g, a.pts.bin_start, a.pts.M, a.pts.work, stream);
    if (wl.grid > 0x7fffffffll) throw_input("grid too large");
    dim3 grid(unsigned(wl.grid), unsigned(a.batch), 1);
    kern<<<grid, kTppThreads, smem, stream>>>(a, L, wl);
    NNB_LAUNCH_CHECK();
    return;
  }
  int nw = kMaxSlabWarps;
  auto smem_for = [&](int n) {
    return size_t(n) * L.cells * sizeof(cplx_t<T>) + size_t(n) * 32 * ((DIM * W) | 1) * sizeof(T);
  };
  while (nw > 1 && smem_for(nw) > 227 * 1024) nw /= 2;
  const size_t smem = smem_for(nw);
  if (smem > 227 * 1024) throw_internal("spread slabs do not fit in shared memory");
  auto kern = spread_slab_kernel<T, DIM, W>;
  // Per device and cheap; set on every launch so that multi-device processes stay correct.
  NNB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  const int LD = DIM - 1;
  UnitMap m{};
  m.kind = UnitMap::kSlab;
  m.nw = nw;
  m.groups = (a.g.ntiles[LD] + nw - 1) / nw;
  m.units = a.g.total_tiles / a.g.ntiles[LD] * m.groups;
  const WorkList wl = build_work_list(m, a.g, a.pts.bin_start, a.pts.M, a.pts.work, stream);
  if (wl.grid > 0x7fffffffll) throw_input("grid too large");
  dim3 grid(unsigned(wl.grid), unsigned(a.batch), 1);
  kern<<<grid, nw * 32, smem, stream>>>(a, L, wl);
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

size_t spread_smem_bytes(int dim, int w, const int* tile, size_t complex_bytes, int warps) {
  const TileLayout L = make_tile_layout(dim, w, tile[0], dim > 1 ? tile[1] : 1,
                                        dim > 2 ? tile[2] : 1, int(complex_bytes));
  return size_t(warps) * L.cells * complex_bytes +
         size_t(warps) * 32 * ((dim * w) | 1) * (complex_bytes / 2);
}

template <typename T>
void launch_spread(const SpreadArgs<T>& a, cudaStream_t stream) {
  if (a.g.total_tiles <= 0 || a.batch <= 0) return;
  if (a.method == 3 || a.method == 4) return launch_spread_zwin<T>(a, stream);
  if (a.method == 5) {
    if constexpr (std::is_same<T, float>::value) return launch_spread_tc(a, stream);
    throw_internal("tensor-core spreading is single precision");
  }
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
