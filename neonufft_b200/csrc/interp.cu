// ES interpolation by shared-memory subproblem tiles.
//
// Replaces the reference's interpolation (src/neonufft/gpu/kernels/interpolation_kernel.cu:27-457),
// where each warp gathers its point's w^d cells straight from global memory in the user's point
// order.
//
// Method 1 (default): a CTA of up to 4 warps covers as many consecutive tiles (bins) along the
// last dimension and stages their union plus the (w-1)-cell halo into shared memory once
// (coalesced along x, periodic wrap, padded strides, tile_layout.cuh). Each warp walks one
// tile's bin-sorted points in batches of 32 (lane j loads point j's record and evaluates its
// w*d kernel values, all in parallel); then, one point at a time, lane r contracts footprint
// row r (3D: (dy, dz); 2D: cell (dx, dy)) against kx, and a shuffle reduction forms the
// point's value, which lane j applies the optional per-point factor to (type-3 postphase) and
// stores at the point's original index.
// Method 2: thread per point on one staged tile per CTA.
#include "kernels.cuh"
#include "tile_layout.cuh"

namespace nnb {

namespace {

constexpr int kMaxInterpWarps = 4;  // warps (tiles) per CTA; fewer when the region does not fit
constexpr int kTppThreads = 256;

// Stages rows [0, nrows) of the padded region starting at (o0, o1, o2) (3D rows are (cy, cz)
// pairs, 2D rows are cy, 1D has one row of ext cells), with periodic wrap.
template <typename T, int DIM>
__device__ __forceinline__ void stage_region(const BinGeom& g, const TileLayout& L, int nrows,
                                             int ext1d, i64 o0, i64 o1, i64 o2,
                                             const cplx_t<T>* grid, cplx_t<T>* tile) {
  if constexpr (DIM == 1) {
    (void)L;
    (void)nrows;
    (void)o1;
    (void)o2;
    for (int cx = threadIdx.x; cx < ext1d; cx += blockDim.x) {
      const i64 gi = wrap_index(o0 + cx, g.nf[0]);
      tile[cx] = NNB_CHECK_INDEX(gi, g.nf[0]) ? grid[gi] : cplx_t<T>{T(0), T(0)};
    }
  } else {
    (void)ext1d;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    for (int row = warp; row < nrows; row += nwarps) {
      int cy = row, cz = 0;
      if (DIM == 3) {
        cz = row / L.P1;
        cy = row - cz * L.P1;
      }
      i64 rbase = wrap_index(o1 + cy, g.nf[1]) * g.nf[0];
      if (DIM == 3) rbase += wrap_index(o2 + cz, g.nf[2]) * g.nf[0] * g.nf[1];
      cplx_t<T>* dst = tile + cz * L.PS + cy * L.RS;
      for (int cx = lane; cx < L.P0; cx += 32) {
        const i64 gi = rbase + wrap_index(o0 + cx, g.nf[0]);
        dst[cx] = NNB_CHECK_INDEX(gi, g.nf[0] * g.nf[1] * g.nf[2]) ? grid[gi]
                                                                   : cplx_t<T>{T(0), T(0)};
      }
    }
  }
}

template <typename T, int DIM, int W>
__global__ void __launch_bounds__(kMaxInterpWarps * 32) interp_slab_kernel(InterpArgs<T> a,
                                                                           TileLayout L,
                                                                           WorkList wl) {
  using C = cplx_t<T>;
  const int nwarps = blockDim.x >> 5;
  constexpr int KS = (DIM * W) | 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tile = reinterpret_cast<C*>(smem_raw);
  T* kbuf = reinterpret_cast<T*>(tile + L.cells);

  const BinGeom& g = a.g;
  constexpr int LD = DIM - 1;
  const int n_last = g.ntiles[LD];
  const int groups = (n_last + nwarps - 1) / nwarps;
  u32 unit, slice;
  if (!work_item(wl, unit, slice)) return;
  const i64 rest = unit / groups;
  const int grp = int(unit - rest * groups);
  int tc[3] = {0, 0, 0};
  {
    i64 r = rest;
    for (int d = 0; d < LD; ++d) {
      tc[d] = int(r % g.ntiles[d]);
      r /= g.ntiles[d];
    }
    tc[LD] = grp * nwarps;
  }
  const int T_last = g.tile[LD];
  int nvalid = n_last - tc[LD];
  if (nvalid > nwarps) nvalid = nwarps;

  const int lane = threadIdx.x & 31;
  const int warp = threadIdx.x >> 5;
  auto bin_of = [&](int t_last) -> i64 {
    if (DIM == 1) return t_last;
    if (DIM == 2) return tc[0] + i64(g.ntiles[0]) * t_last;
    return tc[0] + i64(g.ntiles[0]) * (tc[1] + i64(g.ntiles[1]) * t_last);
  };
  // This CTA's slice of each tile's points; skip CTAs without points (no staging traffic).
  bool any = false;
  for (int w = 0; w < nvalid; ++w) {
    const i64 b = bin_of(tc[LD] + w);
    u32 s0, s1;
    work_slice(a.pts.bin_start[b], a.pts.bin_start[b + 1], slice, wl.cap, s0, s1);
    any |= s1 > s0;
  }
  if (!any) return;

  const i64 o0 = i64(tc[0]) * g.tile[0];
  const i64 o1 = DIM > 1 ? i64(tc[1]) * g.tile[1] : 0;
  const i64 o2 = DIM > 2 ? i64(tc[2]) * g.tile[2] : 0;
  const int p_last = nvalid * T_last + W - 1;  // staged extent along the last dimension
  stage_region<T, DIM>(g, L, DIM == 3 ? p_last * L.P1 : p_last, p_last, o0, o1, o2, a.grid,
                       tile);
  __syncthreads();

  if (warp >= nvalid) return;
  const i64 bin = bin_of(tc[LD] + warp);
  u32 start, end;
  work_slice(a.pts.bin_start[bin], a.pts.bin_start[bin + 1], slice, wl.cap, start, end);
  T* kvb = kbuf + warp * 32 * KS;
  const int shift = warp * T_last * ((DIM == 3) ? L.PS : (DIM == 2 ? L.RS : 1));

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
    u32 my_idx = 0;
    C my_post{T(1), T(0)};
    if (lane < nb && NNB_CHECK_INDEX(i64(b) + lane, a.pts.M)) {
      const PointRec<T> rec = a.pts.rec[b + lane];
      my_idx = rec.perm;
      if (a.postphase && NNB_CHECK_INDEX(my_idx, a.pts.M)) my_post = a.postphase[my_idx];
      int lx, ly, lz;
      unpack_local(DIM, rec.local, lx, ly, lz);
      my_base = shift + lz * L.PS + ly * L.RS + lx;
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
      const T* kj = kvb + j * KS;
      T sx = 0, sy = 0;
      if (DIM == 3) {
        T kx[W];
#pragma unroll
        for (int k = 0; k < W; ++k) kx[k] = kj[k];
#pragma unroll
        for (int k = 0; k < PASSES; ++k) {
          if (lane + 32 * k < NR) {
            const C* row = tile + base + roff[k];
            T rx = 0, ry = 0;
#pragma unroll
            for (int dx = 0; dx < W; ++dx) {
              const C gv = row[dx];
              rx += kx[dx] * gv.x;
              ry += kx[dx] * gv.y;
            }
            const T kyz = kj[W + ra[k]] * kj[2 * W + rb[k]];
            sx += kyz * rx;
            sy += kyz * ry;
          }
        }
      } else if (DIM == 2) {
#pragma unroll
        for (int k = 0; k < PASSES; ++k) {
          if (lane + 32 * k < NR) {
            const T kk = kj[ra[k]] * kj[W + rb[k]];
            const C gv = tile[base + roff[k]];
            sx += kk * gv.x;
            sy += kk * gv.y;
          }
        }
      } else {
        if (lane < W) {
          const C gv = tile[base + lane];
          sx = kj[lane] * gv.x;
          sy = kj[lane] * gv.y;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        sx += __shfl_xor_sync(0xffffffffu, sx, o);
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
      }
      if (lane == int(j)) {
        C res{sx, sy};
        if (a.postphase) res = cmul(res, my_post);
        if (NNB_CHECK_INDEX(my_idx, a.pts.M)) a.out[my_idx] = res;
      }
    }
    __syncwarp();
  }
}

// Thread-per-point variant on one staged tile per CTA.
template <typename T, int DIM, int W>
__global__ void __launch_bounds__(kTppThreads) interp_tpp_kernel(InterpArgs<T> a, TileLayout L,
                                                                  WorkList wl) {
  using C = cplx_t<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* tile = reinterpret_cast<C*>(smem_raw);
  const BinGeom& g = a.g;
  u32 unit, slice;
  if (!work_item(wl, unit, slice)) return;
  const i64 bin = unit;
  u32 start, end;
  work_slice(a.pts.bin_start[bin], a.pts.bin_start[bin + 1], slice, wl.cap, start, end);
  if (start == end) return;
  const i64 t0 = bin % g.ntiles[0];
  const i64 t1 = DIM > 1 ? (bin / g.ntiles[0]) % g.ntiles[1] : 0;
  const i64 t2 = DIM > 2 ? bin / (i64(g.ntiles[0]) * g.ntiles[1]) : 0;
  stage_region<T, DIM>(g, L, DIM == 3 ? L.P1 * L.P2 : L.P1, L.P0, t0 * g.tile[0],
                       t1 * g.tile[1], t2 * g.tile[2], a.grid, tile);
  __syncthreads();
  for (u32 p = start + threadIdx.x; p < end; p += kTppThreads) {
    if (!NNB_CHECK_INDEX(p, a.pts.M)) break;
    const PointRec<T> rec = a.pts.rec[p];
    int lx, ly, lz;
    unpack_local(DIM, rec.local, lx, ly, lz);
    T kx[W];
    const T fx = rec.frac[0];
#pragma unroll
    for (int k = 0; k < W; ++k) kx[k] = es_eval_fast<T>(fx + T(k), a.beta, a.c);
    T sx = 0, sy = 0;
    const int nz = DIM > 2 ? W : 1;
    const int ny = DIM > 1 ? W : 1;
    const T fy = DIM > 1 ? rec.frac[1] : T(0);
    const T fz = DIM > 2 ? rec.frac[2] : T(0);
#pragma unroll 1
    for (int dz = 0; dz < nz; ++dz) {
      const T kz = DIM > 2 ? es_eval_fast<T>(fz + T(dz), a.beta, a.c) : T(1);
#pragma unroll 1
      for (int dy = 0; dy < ny; ++dy) {
        const T ky = (DIM > 1 ? es_eval_fast<T>(fy + T(dy), a.beta, a.c) : T(1)) * kz;
        const C* row = tile + (lz + dz) * L.PS + (ly + dy) * L.RS + lx;
        T rx = 0, ry = 0;
#pragma unroll
        for (int dx = 0; dx < W; ++dx) {
          const C gv = row[dx];
          rx += kx[dx] * gv.x;
          ry += kx[dx] * gv.y;
        }
        sx += ky * rx;
        sy += ky * ry;
      }
    }
    const u32 idx = rec.perm;
    C res{sx, sy};
    if (!NNB_CHECK_INDEX(idx, a.pts.M)) continue;
    if (a.postphase) res = cmul(res, a.postphase[idx]);
    a.out[idx] = res;
  }
}

template <typename T, int DIM, int W>
void launch_interp_tw(const InterpArgs<T>& a, cudaStream_t stream) {
  const int LD = DIM - 1;
  if (a.method == 2) {
    const TileLayout L = make_tile_layout(DIM, W, a.g.tile[0], a.g.tile[1], a.g.tile[2],
                                          int(sizeof(cplx_t<T>)));
    const size_t smem = size_t(L.cells) * sizeof(cplx_t<T>);
    if (smem > 227 * 1024) throw_internal("interpolation tile does not fit in shared memory");
    auto kern = interp_tpp_kernel<T, DIM, W>;
    NNB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    UnitMap m{};
    m.kind = UnitMap::kTile;
    m.units = a.g.total_tiles;
    const WorkList wl = build_work_list(m, a.g, a.pts.bin_start, a.pts.M, a.pts.work, stream);
    if (wl.grid > 0x7fffffffll) throw_input("grid too large");
    kern<<<unsigned(wl.grid), kTppThreads, smem, stream>>>(a, L, wl);
    NNB_LAUNCH_CHECK();
    return;
  }
  int nw = kMaxInterpWarps;
  TileLayout L{};
  size_t smem = 0;
  for (;; nw /= 2) {
    int ext[3] = {a.g.tile[0], a.g.tile[1], a.g.tile[2]};
    ext[LD] = nw * a.g.tile[LD];
    L = make_tile_layout(DIM, W, ext[0], ext[1], ext[2], int(sizeof(cplx_t<T>)));
    smem = size_t(L.cells) * sizeof(cplx_t<T>) + size_t(nw) * 32 * ((DIM * W) | 1) * sizeof(T);
    if (smem <= 227 * 1024 || nw == 1) break;
  }
  if (smem > 227 * 1024) throw_internal("interpolation tile does not fit in shared memory");
  auto kern = interp_slab_kernel<T, DIM, W>;
  NNB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  UnitMap m{};
  m.kind = UnitMap::kSlab;
  m.nw = nw;
  m.groups = (a.g.ntiles[LD] + nw - 1) / nw;
  m.units = a.g.total_tiles / a.g.ntiles[LD] * m.groups;
  const WorkList wl = build_work_list(m, a.g, a.pts.bin_start, a.pts.M, a.pts.work, stream);
  if (wl.grid > 0x7fffffffll) throw_input("grid too large");
  kern<<<unsigned(wl.grid), nw * 32, smem, stream>>>(a, L, wl);
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

size_t interp_smem_bytes(int dim, int w, const int* tile, size_t complex_bytes, int warps) {
  int ext[3] = {tile[0], dim > 1 ? tile[1] : 1, dim > 2 ? tile[2] : 1};
  ext[dim - 1] *= warps;
  const TileLayout L = make_tile_layout(dim, w, ext[0], ext[1], ext[2], int(complex_bytes));
  return size_t(L.cells) * complex_bytes +
         size_t(warps) * 32 * ((dim * w) | 1) * (complex_bytes / 2);
}

template <typename T>
void launch_interp(const InterpArgs<T>& a, cudaStream_t stream) {
  if (a.g.total_tiles <= 0) return;
  // method 5 spreads on the tensor cores; it interpolates with the z-window kernel
  if (a.method == 3 || a.method == 4 || a.method == 5) return launch_interp_zwin<T>(a, stream);
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
