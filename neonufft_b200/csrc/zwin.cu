// 3D ES spreading and interpolation with a sliding z-window held in registers (method 3).
//
// Replaces, for 3D plans with kernel width w <= 8, the reference's spreading
// (src/neonufft/gpu/kernels/spreading_kernel.cu:477-715, one global float atomic per cell and
// point) and interpolation (src/neonufft/gpu/kernels/interpolation_kernel.cu, one thread per
// point reading w^3 cells from global memory).
//
// Points are binned by (x tile of TX cells, y tile of 8 cells, single z plane), and the bins of
// one (x, y) column are consecutive in plane order (BinGeom::zmajor). One CTA walks one column
// over a chunk of planes. Its region is P0 x P1 cells in (x, y), P0 = TX + w - 1 and
// P1 = 8 + w - 1, and RZ >= w consecutive planes in z:
//  * thread (a, b), a = y residue mod 8, b = z residue mod RZ, keeps in registers the region
//    rows y = a, a + 8 (all P0 cells of each) of the one plane p = b (mod RZ) that lies in the
//    current window [t, t + RZ). Each point whose footprint starts at plane t touches, for
//    w = 8, exactly one of those rows in every thread: no two threads share a cell, so there
//    are no atomics and no shared-memory traffic per cell;
//  * the points of plane t are staged once in shared memory (one thread per point: its kernel
//    values placed over the region's x range, zero elsewhere, so that every thread applies
//    them with fixed register indices; strength times ky; kz; y offset);
//  * every thread then adds c * kx[i] * ky * kz to its row cells with packed two-float FMAs
//    (fma.rn.f32x2 on sm_100a), the complex strength being the packed pair;
//  * spreading: after plane t the plane is complete, and the threads holding it add it to the
//    fine grid (float2 / double2 atomics: neighbouring columns and chunks overlap by the halo)
//    and start on plane t + RZ;
//  * interpolation: the threads holding plane t reload their rows with plane t + RZ, fetched
//    with cp.async while plane t's points are processed; per point the row sums of all threads
//    are reduced over the warp for eight points at a time (transposed butterfly), then over
//    the CTA's warps through shared memory.
#include "kernels.cuh"

namespace nnb {

namespace {

// ---- packed complex arithmetic ---------------------------------------------------------------
template <typename T>
struct Packed;

template <>
struct Packed<float> {
  using P = unsigned long long;  // (re, im) in one 64-bit register pair
  static __device__ __forceinline__ P zero() { return 0ull; }
  static __device__ __forceinline__ P pack(float x, float y) {
    P r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
    return r;
  }
  static __device__ __forceinline__ P splat(float x) {
    P r;
    asm("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(x));
    return r;
  }
  static __device__ __forceinline__ float2 unpack(P v) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
  }
  // a * b + c, elementwise
  static __device__ __forceinline__ P fma(P a, P b, P c) {
    P d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
  }
  static __device__ __forceinline__ P mul(P a, P b) {
    P d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
  }
  static __device__ __forceinline__ P add(P a, P b) {
    P d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
  }
  static __device__ __forceinline__ P shfl_xor(P v, int m) {
    return __shfl_xor_sync(0xffffffffu, v, m);
  }
};

template <>
struct Packed<double> {
  using P = double2;
  static __device__ __forceinline__ P zero() { return P{0.0, 0.0}; }
  static __device__ __forceinline__ P pack(double x, double y) { return P{x, y}; }
  static __device__ __forceinline__ P splat(double x) { return P{x, x}; }
  static __device__ __forceinline__ double2 unpack(P v) { return v; }
  static __device__ __forceinline__ P fma(P a, P b, P c) {
    return P{::fma(a.x, b.x, c.x), ::fma(a.y, b.y, c.y)};
  }
  static __device__ __forceinline__ P mul(P a, P b) { return P{a.x * b.x, a.y * b.y}; }
  static __device__ __forceinline__ P add(P a, P b) { return P{a.x + b.x, a.y + b.y}; }
  static __device__ __forceinline__ P shfl_xor(P v, int m) {
    return P{__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m)};
  }
};

__device__ __forceinline__ void atomic_add_cplx(float2* p, float2 v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_cplx(double2* p, double2 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
}

// ---- geometry ----------------------------------------------------------------------------------
template <int W, int TX>
struct ZShape {
  static constexpr int RY = 8;                   // y residues (threads per z residue)
  static constexpr int RZ = W <= 4 ? 4 : 8;      // z residues = window planes (>= W)
  static constexpr int NT = RY * RZ;             // threads per CTA
  static constexpr int TY = 8;                   // tile y
  static constexpr int P0 = TX + W - 1;          // region x extent
  static constexpr int P0R = (P0 + 1) & ~1;      // padded to an even count (16-byte loads)
  static constexpr int P1 = TY + W - 1;          // region y extent
  static constexpr int NYR = (P1 + RY - 1) / RY; // region rows per thread
  static_assert(W <= RZ, "window narrower than the kernel");
};

// Per-point data staged in shared memory (one slot per point of a batch).
template <typename T, int W, int P0R>
struct alignas(16) ZSlot {
  typename Packed<T>::P kx[P0R];  // (k, k) over the region's x range, zero outside the footprint
  typename Packed<T>::P kyv[W];   // spreading: strength * ky[d]; interpolation: (ky, ky)
  T kz[W];
  int ly;                         // first footprint row, tile-local
};

// Stages point p (bin-sorted index) into slot `sl`; v is its strength (spreading only).
template <typename T, int W, int TX, bool SPREAD>
__device__ __forceinline__ void stage_point(ZSlot<T, W, ZShape<W, TX>::P0R>& sl,
                                            const SortedPoints<T>& pts, u32 p,
                                            cplx_t<T> v, T beta, T c) {
  using S = ZShape<W, TX>;
  using Ops = Packed<T>;
  const u32 loc = pts.local[p];
  const int lx = int(loc & 0x7FFu);
  const int ly = int((loc >> 11) & 0x7FFu);
  const T fx = pts.frac[0][p];
  const T fy = pts.frac[1][p];
  const T fz = pts.frac[2][p];
#pragma unroll
  for (int i = 0; i < S::P0R; ++i) sl.kx[i] = Ops::zero();
#pragma unroll
  for (int k = 0; k < W; ++k) sl.kx[lx + k] = Ops::splat(es_eval_fast<T>(fx + T(k), beta, c));
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const T ky = es_eval_fast<T>(fy + T(k), beta, c);
    sl.kyv[k] = SPREAD ? Ops::pack(v.x * ky, v.y * ky) : Ops::splat(ky);
    sl.kz[k] = es_eval_fast<T>(fz + T(k), beta, c);
  }
  sl.ly = ly;
}

// Chunk of planes handled by one CTA.
struct ZChunks {
  int len;      // planes per chunk
  int count;    // chunks per column
};

template <typename T>
__device__ __forceinline__ i64 wrap_add(i64 base, int off, i64 n) {
  i64 i = base + off;
  while (i >= n) i -= n;
  return i;
}

// ---- spreading ---------------------------------------------------------------------------------
template <typename T, int W, int TX>
__global__ void __launch_bounds__(ZShape<W, TX>::NT, sizeof(T) == 4 ? 8 : 5)
    spread_zwin_kernel(SpreadArgs<T> a, ZChunks ch) {
  using S = ZShape<W, TX>;
  using Ops = Packed<T>;
  using P = typename Ops::P;
  using C = cplx_t<T>;
  __shared__ ZSlot<T, W, S::P0R> slots[S::NT];

  const BinGeom& g = a.g;
  const int tid = threadIdx.x;
  const int ra = tid & (S::RY - 1);
  const int rb = tid / S::RY;
  const i64 ncols = i64(g.ntiles[0]) * g.ntiles[1];
  const int chunk = int(blockIdx.x / ncols);
  const i64 col = blockIdx.x - i64(chunk) * ncols;
  const int tx = int(col % g.ntiles[0]);
  const int ty = int(col / g.ntiles[0]);
  const int nz = g.ntiles[2];  // == nf[2]: single-plane tiles
  const int z0 = chunk * ch.len;
  const int z1 = min(z0 + ch.len, nz);
  const u32* bs = a.pts.bin_start + col * nz;
  if (z0 >= z1 || bs[z0] == bs[z1]) return;

  const int batch = blockIdx.y;
  const C* in = a.in + batch * a.in_bdist;
  C* grid = a.grid + batch * a.grid_bdist;
  const i64 nfx = g.nf[0], nfy = g.nf[1], nfz = g.nf[2];
  const i64 gx0 = i64(tx) * TX;
  const i64 gy0 = i64(ty) * S::TY;

  P acc[S::NYR][S::P0];
#pragma unroll
  for (int j = 0; j < S::NYR; ++j) {
#pragma unroll
    for (int i = 0; i < S::P0; ++i) acc[j][i] = Ops::zero();
  }

  // Adds this thread's rows of plane p (absolute, may exceed nfz) to the grid and clears them.
  auto flush = [&](i64 p) {
    const i64 gz = p % nfz;
#pragma unroll
    for (int j = 0; j < S::NYR; ++j) {
      const int y = ra + S::RY * j;
      if (y < S::P1) {
        const i64 row = (gz * nfy + wrap_add<T>(gy0, y, nfy)) * nfx;
#pragma unroll
        for (int i = 0; i < S::P0; ++i) {
          const C v = Ops::unpack(acc[j][i]);
          acc[j][i] = Ops::zero();
          if (v.x != T(0) || v.y != T(0)) atomic_add_cplx(&grid[row + wrap_add<T>(gx0, i, nfx)], v);
        }
      }
    }
  };

  u32 e = bs[z0];
  for (int t = z0; t < z1; ++t) {
    const u32 s = e;
    e = bs[t + 1];
    const int dz = (rb - t) & (S::RZ - 1);  // this thread's plane within the footprint
    for (u32 base = s; base < e; base += S::NT) {
      const int nb = int(min(e - base, u32(S::NT)));
      if (tid < nb) {
        const u32 p = base + tid;
        const u32 idx = a.pts.perm[p];
        C v = in[idx];
        if (a.prephase) v = cmul(v, a.prephase[idx]);
        stage_point<T, W, TX, true>(slots[tid], a.pts, p, v, a.beta, a.c);
      }
      __syncthreads();
      if (dz < W) {
        for (int j = 0; j < nb; ++j) {
          const ZSlot<T, W, S::P0R>& sl = slots[j];
          const P kz = Ops::splat(sl.kz[dz]);
          const int ly = sl.ly;
          P wy[S::NYR];
#pragma unroll
          for (int r = 0; r < S::NYR; ++r) {
            const int dy = ra + S::RY * r - ly;
            const int dyc = dy < 0 ? 0 : (dy >= W ? W - 1 : dy);
            const P kv = sl.kyv[dyc];
            wy[r] = (dy >= 0 && dy < W) ? Ops::mul(kv, kz) : Ops::zero();
          }
          if (sizeof(T) == 4) {
#pragma unroll
            for (int i = 0; i < S::P0; i += 2) {
              const ulonglong2 kk = *reinterpret_cast<const ulonglong2*>(&sl.kx[i]);
              const P k0 = reinterpret_cast<const P&>(kk.x);
              const P k1 = reinterpret_cast<const P&>(kk.y);
#pragma unroll
              for (int r = 0; r < S::NYR; ++r) {
                acc[r][i] = Ops::fma(k0, wy[r], acc[r][i]);
                if (i + 1 < S::P0) acc[r][i + 1] = Ops::fma(k1, wy[r], acc[r][i + 1]);
              }
            }
          } else {
#pragma unroll
            for (int i = 0; i < S::P0; ++i) {
              const P k0 = sl.kx[i];
#pragma unroll
              for (int r = 0; r < S::NYR; ++r) acc[r][i] = Ops::fma(k0, wy[r], acc[r][i]);
            }
          }
        }
      }
      __syncthreads();
    }
    if (rb == (t & (S::RZ - 1))) flush(t);
  }
  // planes [z1, z1 + w - 1) still hold contributions of this chunk's last planes
  flush(z1 + ((rb - z1) & (S::RZ - 1)));
}

// ---- interpolation -----------------------------------------------------------------------------
__device__ __forceinline__ void cp_async_cell(void* smem, const float2* g) {
  const unsigned s = unsigned(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_cell(void* smem, const double2* g) {
  const unsigned s = unsigned(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <typename T, int W, int TX>
__global__ void __launch_bounds__(ZShape<W, TX>::NT, sizeof(T) == 4 ? 8 : 5)
    interp_zwin_kernel(InterpArgs<T> a, ZChunks ch) {
  using S = ZShape<W, TX>;
  using Ops = Packed<T>;
  using P = typename Ops::P;
  using C = cplx_t<T>;
  constexpr int NW = S::NT / 32;
  constexpr int G = 8;  // points reduced together
  __shared__ ZSlot<T, W, S::P0R> slots[S::NT];
  __shared__ P res[NW][S::NT];
  __shared__ C stage[S::RY][S::NYR][S::P0];

  const BinGeom& g = a.g;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int ra = tid & (S::RY - 1);
  const int rb = tid / S::RY;
  const i64 ncols = i64(g.ntiles[0]) * g.ntiles[1];
  const int chunk = int(blockIdx.x / ncols);
  const i64 col = blockIdx.x - i64(chunk) * ncols;
  const int tx = int(col % g.ntiles[0]);
  const int ty = int(col / g.ntiles[0]);
  const int nz = g.ntiles[2];
  const int z0 = chunk * ch.len;
  const int z1 = min(z0 + ch.len, nz);
  const u32* bs = a.pts.bin_start + col * nz;
  if (z0 >= z1 || bs[z0] == bs[z1]) return;

  const C* grid = a.grid;
  const i64 nfx = g.nf[0], nfy = g.nf[1], nfz = g.nf[2];
  const i64 gx0 = i64(tx) * TX;
  const i64 gy0 = i64(ty) * S::TY;

  // Row offsets (in cells) of this thread's region rows within a plane.
  i64 rowoff[S::NYR];
#pragma unroll
  for (int j = 0; j < S::NYR; ++j) {
    const int y = ra + S::RY * j;
    rowoff[j] = y < S::P1 ? wrap_add<T>(gy0, y, nfy) * nfx : -1;
  }
  int xo[S::P0];
#pragma unroll
  for (int i = 0; i < S::P0; ++i) xo[i] = int(wrap_add<T>(gx0, i, nfx));

  P acc[S::NYR][S::P0];
  {
    const i64 p = z0 + ((rb - z0) & (S::RZ - 1));
    const C* plane = grid + (p % nfz) * nfy * nfx;
#pragma unroll
    for (int j = 0; j < S::NYR; ++j) {
#pragma unroll
      for (int i = 0; i < S::P0; ++i) {
        if (rowoff[j] >= 0) {
          const C v = plane[rowoff[j] + xo[i]];
          acc[j][i] = Ops::pack(v.x, v.y);
        } else {
          acc[j][i] = Ops::zero();
        }
      }
    }
  }

  u32 e = bs[z0];
  for (int t = z0; t < z1; ++t) {
    const u32 s = e;
    e = bs[t + 1];
    const int dz = (rb - t) & (S::RZ - 1);
    const bool loader = dz == 0;  // holds plane t; reloads plane t + RZ afterwards
    __syncthreads();  // the previous plane's loaders have read the stage
    if (loader && t + S::RZ < z1 + S::RZ - 1) {
      const C* plane = grid + ((t + S::RZ) % nfz) * nfy * nfx;
#pragma unroll
      for (int j = 0; j < S::NYR; ++j) {
        if (rowoff[j] >= 0) {
#pragma unroll
          for (int i = 0; i < S::P0; ++i) cp_async_cell(&stage[ra][j][i], plane + rowoff[j] + xo[i]);
        }
      }
      cp_async_commit();
    }
    for (u32 base = s; base < e; base += S::NT) {
      const int nb = int(min(e - base, u32(S::NT)));
      u32 my_idx = 0;
      if (tid < nb) {
        const u32 p = base + tid;
        my_idx = a.pts.perm[p];
        stage_point<T, W, TX, false>(slots[tid], a.pts, p, C{T(0), T(0)}, a.beta, a.c);
      }
      __syncthreads();
      for (int j0 = 0; j0 < nb; j0 += G) {
        P part[G];
#pragma unroll
        for (int k = 0; k < G; ++k) {
          part[k] = Ops::zero();
          if (j0 + k < nb && dz < W) {
            const ZSlot<T, W, S::P0R>& sl = slots[j0 + k];
            const P kz = Ops::splat(sl.kz[dz]);
            const int ly = sl.ly;
            P rs[S::NYR];
#pragma unroll
            for (int r = 0; r < S::NYR; ++r) rs[r] = Ops::zero();
            if (sizeof(T) == 4) {
#pragma unroll
              for (int i = 0; i < S::P0; i += 2) {
                const ulonglong2 kk = *reinterpret_cast<const ulonglong2*>(&sl.kx[i]);
                const P k0 = reinterpret_cast<const P&>(kk.x);
                const P k1 = reinterpret_cast<const P&>(kk.y);
#pragma unroll
                for (int r = 0; r < S::NYR; ++r) {
                  rs[r] = Ops::fma(k0, acc[r][i], rs[r]);
                  if (i + 1 < S::P0) rs[r] = Ops::fma(k1, acc[r][i + 1], rs[r]);
                }
              }
            } else {
#pragma unroll
              for (int i = 0; i < S::P0; ++i) {
                const P k0 = sl.kx[i];
#pragma unroll
                for (int r = 0; r < S::NYR; ++r) rs[r] = Ops::fma(k0, acc[r][i], rs[r]);
              }
            }
#pragma unroll
            for (int r = 0; r < S::NYR; ++r) {
              const int dy = ra + S::RY * r - ly;
              const int dyc = dy < 0 ? 0 : (dy >= W ? W - 1 : dy);
              const P kv = sl.kyv[dyc];
              const P wgt = (dy >= 0 && dy < W) ? Ops::mul(kv, kz) : Ops::zero();
              part[k] = Ops::fma(wgt, rs[r], part[k]);
            }
          }
        }
        // Transposed butterfly: after it, lanes with (lane & 3) == 0 hold the warp sum of
        // point j0 + ((lane >> 2) & 7).
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const bool hi = lane & 16;
          const P send = hi ? part[k] : part[k + 4];
          const P keep = hi ? part[k + 4] : part[k];
          part[k] = Ops::add(keep, Ops::shfl_xor(send, 16));
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const bool hi = lane & 8;
          const P send = hi ? part[k] : part[k + 2];
          const P keep = hi ? part[k + 2] : part[k];
          part[k] = Ops::add(keep, Ops::shfl_xor(send, 8));
        }
        {
          const bool hi = lane & 4;
          const P send = hi ? part[0] : part[1];
          const P keep = hi ? part[1] : part[0];
          part[0] = Ops::add(keep, Ops::shfl_xor(send, 4));
        }
        part[0] = Ops::add(part[0], Ops::shfl_xor(part[0], 2));
        part[0] = Ops::add(part[0], Ops::shfl_xor(part[0], 1));
        if ((lane & 3) == 0) res[warp][j0 + ((lane >> 2) & 7)] = part[0];
      }
      __syncthreads();
      if (tid < nb) {
        P sum = res[0][tid];
#pragma unroll
        for (int w = 1; w < NW; ++w) sum = Ops::add(sum, res[w][tid]);
        C r = Ops::unpack(sum);
        if (a.postphase) r = cmul(r, a.postphase[my_idx]);
        a.out[my_idx] = r;
      }
    }
    if (loader && t + S::RZ < z1 + S::RZ - 1) {
      cp_async_wait_all();
#pragma unroll
      for (int j = 0; j < S::NYR; ++j) {
#pragma unroll
        for (int i = 0; i < S::P0; ++i) {
          if (rowoff[j] >= 0) {
            const C v = stage[ra][j][i];
            acc[j][i] = Ops::pack(v.x, v.y);
          }
        }
      }
    }
  }
}

ZChunks make_chunks(i64 ncols, int nz, int w) {
  // About four waves of 8 CTAs per SM; chunks of at least 4 w planes bound the window
  // overhead (w - 1 extra planes flushed, or RZ planes loaded, per chunk).
  const i64 target = 148 * 8 * 4;
  i64 count = (target + ncols - 1) / ncols;
  const int min_len = 4 * w;
  const i64 max_count = (nz + min_len - 1) / min_len;
  if (count > max_count) count = max_count;
  if (count < 1) count = 1;
  ZChunks ch;
  ch.len = int((nz + count - 1) / count);
  ch.count = (nz + ch.len - 1) / ch.len;
  return ch;
}

template <typename T, int W, int TX>
void launch_spread_zwin_tw(const SpreadArgs<T>& a, cudaStream_t stream) {
  using S = ZShape<W, TX>;
  const i64 ncols = i64(a.g.ntiles[0]) * a.g.ntiles[1];
  const ZChunks ch = make_chunks(ncols, a.g.ntiles[2], W);
  const i64 ctas = ncols * ch.count;
  if (ctas > 0x7fffffffll) throw_input("grid too large");
  dim3 grid{unsigned(ctas), unsigned(a.batch), 1u};
  spread_zwin_kernel<T, W, TX><<<grid, S::NT, 0, stream>>>(a, ch);
  NNB_LAUNCH_CHECK();
}

template <typename T, int W, int TX>
void launch_interp_zwin_tw(const InterpArgs<T>& a, cudaStream_t stream) {
  using S = ZShape<W, TX>;
  const i64 ncols = i64(a.g.ntiles[0]) * a.g.ntiles[1];
  const ZChunks ch = make_chunks(ncols, a.g.ntiles[2], W);
  const i64 ctas = ncols * ch.count;
  if (ctas > 0x7fffffffll) throw_input("grid too large");
  interp_zwin_kernel<T, W, TX><<<unsigned(ctas), S::NT, 0, stream>>>(a, ch);
  NNB_LAUNCH_CHECK();
}

template <typename T, int TX>
void spread_zwin_tx(const SpreadArgs<T>& a, cudaStream_t stream) {
  switch (a.g.w) {
    case 2: return launch_spread_zwin_tw<T, 2, TX>(a, stream);
    case 3: return launch_spread_zwin_tw<T, 3, TX>(a, stream);
    case 4: return launch_spread_zwin_tw<T, 4, TX>(a, stream);
    case 5: return launch_spread_zwin_tw<T, 5, TX>(a, stream);
    case 6: return launch_spread_zwin_tw<T, 6, TX>(a, stream);
    case 7: return launch_spread_zwin_tw<T, 7, TX>(a, stream);
    case 8: return launch_spread_zwin_tw<T, 8, TX>(a, stream);
    default: throw_internal("z-window kernels need n_spread <= 8");
  }
}

template <typename T, int TX>
void interp_zwin_tx(const InterpArgs<T>& a, cudaStream_t stream) {
  switch (a.g.w) {
    case 2: return launch_interp_zwin_tw<T, 2, TX>(a, stream);
    case 3: return launch_interp_zwin_tw<T, 3, TX>(a, stream);
    case 4: return launch_interp_zwin_tw<T, 4, TX>(a, stream);
    case 5: return launch_interp_zwin_tw<T, 5, TX>(a, stream);
    case 6: return launch_interp_zwin_tw<T, 6, TX>(a, stream);
    case 7: return launch_interp_zwin_tw<T, 7, TX>(a, stream);
    case 8: return launch_interp_zwin_tw<T, 8, TX>(a, stream);
    default: throw_internal("z-window kernels need n_spread <= 8");
  }
}

void check_zwin_geom(const BinGeom& g) {
  if (g.dim != 3 || !g.zmajor || g.tile[1] != 8 || g.tile[2] != 1 ||
      (g.tile[0] != 4 && g.tile[0] != 8) || g.w > 8) {
    throw_internal("z-window kernels need a 3D plane-major (4|8, 8, 1) tiling and n_spread <= 8");
  }
}

}  // namespace

template <typename T>
void launch_spread_zwin(const SpreadArgs<T>& a, cudaStream_t stream) {
  check_zwin_geom(a.g);
  if (a.batch > 65535) throw_input("batch size above 65535");
  if (a.g.tile[0] == 8) return spread_zwin_tx<T, 8>(a, stream);
  return spread_zwin_tx<T, 4>(a, stream);
}

template <typename T>
void launch_interp_zwin(const InterpArgs<T>& a, cudaStream_t stream) {
  check_zwin_geom(a.g);
  if (a.g.tile[0] == 8) return interp_zwin_tx<T, 8>(a, stream);
  return interp_zwin_tx<T, 4>(a, stream);
}

template void launch_spread_zwin<float>(const SpreadArgs<float>&, cudaStream_t);
template void launch_spread_zwin<double>(const SpreadArgs<double>&, cudaStream_t);
template void launch_interp_zwin<float>(const InterpArgs<float>&, cudaStream_t);
template void launch_interp_zwin<double>(const InterpArgs<double>&, cudaStream_t);

}  // namespace nnb
