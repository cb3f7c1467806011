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
// P1 = 8 + w - 1 <= 15, times a window of RZ >= w consecutive planes:
//  * thread (a, b) keeps in registers the whole region row y = a (P0 cells, as pairs of
//    neighbouring cells) of the one window plane p = b (mod RZ). The 16 rows a are split over
//    the warps, LA = 32 / RZ rows per warp, so for a point whose footprint covers rows
//    [ly, ly + w) a warp either owns some of them or skips the point with a warp-uniform
//    branch; no thread holds a cell that another thread updates, so there are no atomics and
//    no shared-memory traffic per cell;
//  * the points of plane t are staged in shared memory (one thread per point): kx over the
//    region's x range, strength * ky over the 16 rows and kz over the RZ planes, each zero
//    outside the footprint, so that every thread applies them with fixed register indices and
//    no range tests;
//  * each owning thread updates its row with packed two-float FMAs (fma.rn.f32x2 on sm_100a),
//    one for the real and one for the imaginary parts of two neighbouring cells;
//  * spreading: when plane t is complete, the threads holding it add it to the fine grid
//    (float2 / double2 atomics: neighbouring columns and chunks overlap by the halo) and start
//    on plane t + RZ;
//  * interpolation: the threads holding plane t reload their rows with plane t + RZ, fetched
//    with cp.async while plane t's points are processed; per point the row sums are reduced
//    for eight points at a time through a per-warp shared-memory transpose, then over warps.
#include "kernels.cuh"

namespace nnb {

namespace {

// ---- packed arithmetic on pairs of values --------------------------------------------------------
template <typename T>
struct Packed;

template <>
struct Packed<float> {
  using P = unsigned long long;  // two floats in one 64-bit register pair
  static __device__ __forceinline__ P zero() { return 0ull; }
  static __device__ __forceinline__ P pack(float x, float y) {
    P r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(x), "f"(y));
    return r;
  }
  static __device__ __forceinline__ P splat(float x) { return pack(x, x); }
  static __device__ __forceinline__ float lo(P v) {
    float x, y;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(x), "=f"(y) : "l"(v));
    return x;
  }
  static __device__ __forceinline__ float hi(P v) {
    float x, y;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(x), "=f"(y) : "l"(v));
    return y;
  }
  // a * b + c, elementwise
  static __device__ __forceinline__ P fma(P a, P b, P c) {
    P d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
  }
  static __device__ __forceinline__ P add(P a, P b) {
    P d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
  }
};

template <>
struct Packed<double> {
  using P = double2;
  static __device__ __forceinline__ P zero() { return P{0.0, 0.0}; }
  static __device__ __forceinline__ P pack(double x, double y) { return P{x, y}; }
  static __device__ __forceinline__ P splat(double x) { return P{x, x}; }
  static __device__ __forceinline__ double lo(P v) { return v.x; }
  static __device__ __forceinline__ double hi(P v) { return v.y; }
  static __device__ __forceinline__ P fma(P a, P b, P c) {
    return P{::fma(a.x, b.x, c.x), ::fma(a.y, b.y, c.y)};
  }
  static __device__ __forceinline__ P add(P a, P b) { return P{a.x + b.x, a.y + b.y}; }
};

// Four consecutive values of a 16-byte aligned shared-memory array as two pairs.
template <typename T>
__device__ __forceinline__ void load_pairs(const T* p, typename Packed<T>::P* k);
template <>
__device__ __forceinline__ void load_pairs<float>(const float* p, unsigned long long* k) {
  const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(p);
  k[0] = v.x;
  k[1] = v.y;
}
template <>
__device__ __forceinline__ void load_pairs<double>(const double* p, double2* k) {
  k[0] = *reinterpret_cast<const double2*>(p);
  k[1] = *reinterpret_cast<const double2*>(p + 2);
}

__device__ __forceinline__ void atomic_add_cplx(float2* p, float2 v) { atomicAdd(p, v); }
__device__ __forceinline__ void atomic_add_cplx(double2* p, double2 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
}

// ---- geometry ----------------------------------------------------------------------------------
template <int W, int TX>
struct ZShape {
  static constexpr int RZ = W <= 4 ? 4 : 8;   // window planes = z residues (>= W)
  static constexpr int LA = 32 / RZ;          // rows per warp
  static constexpr int RY = 16;               // region rows (>= P1)
  static constexpr int NWARP = RY / LA;
  static constexpr int NT = 32 * NWARP;       // threads per CTA
  static constexpr int TY = 8;                // tile y
  static constexpr int P0 = TX + W - 1;       // region x extent (cells)
  static constexpr int NP = (P0 + 1) / 2;     // cell pairs per row
  static constexpr int KXN = 4 * ((NP + 1) / 2);  // staged kx values (16-byte multiple)
  static constexpr int P1 = TY + W - 1;       // region y extent
  static constexpr int BATCH = 64;            // points staged at a time
  static constexpr int G = 8;                 // points reduced together (interpolation)
  static_assert(W <= RZ && P1 <= RY, "window smaller than the kernel footprint");
};

// Per-point data staged in shared memory (one slot per point of a batch).
template <typename T, int W, int TX, bool SPREAD>
struct alignas(16) ZSlot {
  using S = ZShape<W, TX>;
  using KY = typename std::conditional<SPREAD, cplx_t<T>, T>::type;
  T kx[S::KXN];     // kx over the region's x range, zero outside the footprint
  KY ky[S::RY];     // spreading: strength * ky per region row; interpolation: ky
  T kz[S::RZ];      // kz per window offset, zero beyond w
  int ly;           // first footprint row
};

// Stages bin-sorted point p into slot `sl`; v is its strength (spreading only).
template <typename T, int W, int TX, bool SPREAD>
__device__ __forceinline__ void stage_point(ZSlot<T, W, TX, SPREAD>& sl, const PointRec<T>& rec,
                                            cplx_t<T> v, T beta, T c) {
  using S = ZShape<W, TX>;
  const int lx = int(rec.local & 0x7FFu);
  const int ly = int((rec.local >> 11) & 0x7FFu);
#pragma unroll
  for (int i = 0; i < S::KXN; ++i) sl.kx[i] = T(0);
#pragma unroll
  for (int i = 0; i < S::RY; ++i) {
    if constexpr (SPREAD) {
      sl.ky[i] = cplx_t<T>{T(0), T(0)};
    } else {
      sl.ky[i] = T(0);
    }
  }
#pragma unroll
  for (int k = 0; k < W; ++k) sl.kx[lx + k] = es_eval_fast<T>(rec.frac[0] + T(k), beta, c);
#pragma unroll
  for (int k = 0; k < W; ++k) {
    const T ky = es_eval_fast<T>(rec.frac[1] + T(k), beta, c);
    if constexpr (SPREAD) {
      sl.ky[ly + k] = cplx_t<T>{v.x * ky, v.y * ky};
    } else {
      sl.ky[ly + k] = ky;
    }
  }
#pragma unroll
  for (int k = 0; k < S::RZ; ++k) sl.kz[k] = k < W ? es_eval_fast<T>(rec.frac[2] + T(k), beta, c) : T(0);
  sl.ly = ly;
}

// Chunk of planes handled by one CTA.
struct ZChunks {
  int len;    // planes per chunk
  int count;  // chunks per column
};

__device__ __forceinline__ i64 wrap_add(i64 base, int off, i64 n) {
  i64 i = base + off;
  while (i >= n) i -= n;
  return i;
}

// CTA coordinates: column (tx, ty) and plane range [z0, z1); false if the chunk has no points.
struct ZCta {
  int tx, ty, z0, z1;
  i64 col;
};
__device__ __forceinline__ bool zcta(const BinGeom& g, const u32* bin_start, ZChunks ch,
                                     ZCta& c, const u32*& bs) {
  const i64 ncols = i64(g.ntiles[0]) * g.ntiles[1];
  const int chunk = int(blockIdx.x / ncols);
  c.col = blockIdx.x - i64(chunk) * ncols;
  c.tx = int(c.col % g.ntiles[0]);
  c.ty = int(c.col / g.ntiles[0]);
  const int nz = g.ntiles[2];  // == nf[2]: single-plane tiles
  c.z0 = chunk * ch.len;
  c.z1 = min(c.z0 + ch.len, nz);
  bs = bin_start + c.col * nz;
  return c.z0 < c.z1 && bs[c.z0] != bs[c.z1];
}

// ---- spreading ---------------------------------------------------------------------------------
template <typename T, int W, int TX>
__global__ void __launch_bounds__(ZShape<W, TX>::NT)
    spread_zwin_kernel(SpreadArgs<T> a, ZChunks ch) {
  using S = ZShape<W, TX>;
  using Ops = Packed<T>;
  using P = typename Ops::P;
  using C = cplx_t<T>;
  using Slot = ZSlot<T, W, TX, true>;
  __shared__ Slot slots[S::BATCH];

  const BinGeom& g = a.g;
  ZCta cta;
  const u32* bs;
  if (!zcta(g, a.pts.bin_start, ch, cta, bs)) return;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int ra = warp * S::LA + lane % S::LA;  // region row
  const int rb = lane / S::LA;                  // z residue
  const int a_lo = warp * S::LA;                // first row of this warp

  const int batch = blockIdx.y;
  const C* in = a.in + batch * a.in_bdist;
  C* grid = a.grid + batch * a.grid_bdist;
  const i64 nfx = g.nf[0], nfy = g.nf[1], nfz = g.nf[2];
  const i64 gx0 = i64(cta.tx) * TX;
  const i64 row_y = ra < S::P1 ? wrap_add(i64(cta.ty) * S::TY, ra, nfy) : 0;

  P are[S::NP], aim[S::NP];  // real / imaginary parts of cell pairs (2q, 2q + 1)
#pragma unroll
  for (int q = 0; q < S::NP; ++q) are[q] = aim[q] = Ops::zero();

  // Adds this thread's row of plane p (absolute, may exceed nfz) to the grid and clears it.
  auto flush = [&](i64 p) {
    if (ra < S::P1) {
      C* row = grid + ((p % nfz) * nfy + row_y) * nfx;
#pragma unroll
      for (int q = 0; q < S::NP; ++q) {
        const C v0{Ops::lo(are[q]), Ops::lo(aim[q])};
        const C v1{Ops::hi(are[q]), Ops::hi(aim[q])};
        are[q] = aim[q] = Ops::zero();
        if (v0.x != T(0) || v0.y != T(0)) atomic_add_cplx(&row[wrap_add(gx0, 2 * q, nfx)], v0);
        if (2 * q + 1 < S::P0 && (v1.x != T(0) || v1.y != T(0))) {
          atomic_add_cplx(&row[wrap_add(gx0, 2 * q + 1, nfx)], v1);
        }
      }
    }
  };

  u32 e = bs[cta.z0];
  for (int t = cta.z0; t < cta.z1; ++t) {
    const u32 s = e;
    e = bs[t + 1];
    const int dz = (rb - t) & (S::RZ - 1);  // this thread's plane within the window
    for (u32 base = s; base < e; base += S::BATCH) {
      const int nb = int(min(e - base, u32(S::BATCH)));
      if (tid < nb) {
        const PointRec<T> rec = a.pts.rec[base + tid];
        C v = in[rec.perm];
        if (a.prephase) v = cmul(v, a.prephase[rec.perm]);
        stage_point<T, W, TX, true>(slots[tid], rec, v, a.beta, a.c);
      }
      __syncthreads();
      for (int j = 0; j < nb; ++j) {
        const Slot& sl = slots[j];
        const int ly = sl.ly;
        if (ly < a_lo + S::LA && ly + W > a_lo) {  // warp-uniform: this warp owns footprint rows
          const C kyv = sl.ky[ra];
          const T kzv = sl.kz[dz];
          const P wre = Ops::splat(kyv.x * kzv);
          const P wim = Ops::splat(kyv.y * kzv);
#pragma unroll
          for (int q = 0; q < S::NP; q += 2) {
            P k[2];
            load_pairs<T>(&sl.kx[2 * q], k);
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              if (q + u < S::NP) {
                are[q + u] = Ops::fma(k[u], wre, are[q + u]);
                aim[q + u] = Ops::fma(k[u], wim, aim[q + u]);
              }
            }
          }
        }
      }
      __syncthreads();
    }
    if (dz == 0) flush(t);
  }
  // planes [z1, z1 + w - 1) still hold contributions of this chunk's last planes
  flush(cta.z1 + ((rb - cta.z1) & (S::RZ - 1)));
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
__global__ void __launch_bounds__(ZShape<W, TX>::NT)
    interp_zwin_kernel(InterpArgs<T> a, ZChunks ch) {
  using S = ZShape<W, TX>;
  using Ops = Packed<T>;
  using P = typename Ops::P;
  using C = cplx_t<T>;
  using Slot = ZSlot<T, W, TX, false>;
  constexpr int G = S::G;
  constexpr int RS = 33;  // odd row stride of the transpose buffer: conflict-free reads
  __shared__ Slot slots[S::BATCH];
  __shared__ C red[S::NWARP][G][RS];
  __shared__ C res[S::NWARP][S::BATCH];
  __shared__ C stage[S::RY][2 * S::NP];

  const BinGeom& g = a.g;
  ZCta cta;
  const u32* bs;
  if (!zcta(g, a.pts.bin_start, ch, cta, bs)) return;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int ra = warp * S::LA + lane % S::LA;
  const int rb = lane / S::LA;
  const int a_lo = warp * S::LA;
  const bool has_row = ra < S::P1;

  const C* grid = a.grid;
  const i64 nfx = g.nf[0], nfy = g.nf[1], nfz = g.nf[2];
  const i64 gx0 = i64(cta.tx) * TX;
  const i64 row_y = has_row ? wrap_add(i64(cta.ty) * S::TY, ra, nfy) : 0;
  if (tid < S::RY) {
    for (int i = S::P0; i < 2 * S::NP; ++i) stage[tid][i] = C{T(0), T(0)};  // padding cell
  }

  P gre[S::NP], gim[S::NP];  // real / imaginary parts of cell pairs (2q, 2q + 1) of the row
  {
    const i64 p = cta.z0 + ((rb - cta.z0) & (S::RZ - 1));
    const C* row = grid + ((p % nfz) * nfy + row_y) * nfx;
#pragma unroll
    for (int q = 0; q < S::NP; ++q) {
      C c0{T(0), T(0)}, c1{T(0), T(0)};
      if (has_row) {
        c0 = row[wrap_add(gx0, 2 * q, nfx)];
        if (2 * q + 1 < S::P0) c1 = row[wrap_add(gx0, 2 * q + 1, nfx)];
      }
      gre[q] = Ops::pack(c0.x, c1.x);
      gim[q] = Ops::pack(c0.y, c1.y);
    }
  }

  u32 e = bs[cta.z0];
  for (int t = cta.z0; t < cta.z1; ++t) {
    const u32 s = e;
    e = bs[t + 1];
    const int dz = (rb - t) & (S::RZ - 1);
    const bool loader = dz == 0 && has_row && t + 1 < cta.z1;  // reloads plane t + RZ
    __syncthreads();  // the previous plane's loaders have read the stage
    if (loader) {
      const C* row = grid + (((t + S::RZ) % nfz) * nfy + row_y) * nfx;
#pragma unroll
      for (int i = 0; i < S::P0; ++i) cp_async_cell(&stage[ra][i], row + wrap_add(gx0, i, nfx));
      cp_async_commit();
    }
    for (u32 base = s; base < e; base += S::BATCH) {
      const int nb = int(min(e - base, u32(S::BATCH)));
      u32 my_perm = 0;
      if (tid < nb) {
        const PointRec<T> rec = a.pts.rec[base + tid];
        my_perm = rec.perm;
        stage_point<T, W, TX, false>(slots[tid], rec, C{T(0), T(0)}, a.beta, a.c);
      }
      __syncthreads();
      for (int j0 = 0; j0 < nb; j0 += G) {
#pragma unroll
        for (int k = 0; k < G; ++k) {
          C part{T(0), T(0)};
          const int j = j0 + k;
          if (j < nb) {
            const Slot& sl = slots[j];
            const int ly = sl.ly;
            if (ly < a_lo + S::LA && ly + W > a_lo) {  // warp-uniform
              const T wgt = sl.ky[ra] * sl.kz[dz];
              P sr0 = Ops::zero(), sr1 = Ops::zero(), si0 = Ops::zero(), si1 = Ops::zero();
#pragma unroll
              for (int q = 0; q < S::NP; q += 2) {
                P kk[2];
                load_pairs<T>(&sl.kx[2 * q], kk);
                sr0 = Ops::fma(kk[0], gre[q], sr0);
                si0 = Ops::fma(kk[0], gim[q], si0);
                if (q + 1 < S::NP) {
                  sr1 = Ops::fma(kk[1], gre[q + 1], sr1);
                  si1 = Ops::fma(kk[1], gim[q + 1], si1);
                }
              }
              const P sr = Ops::add(sr0, sr1);
              const P si = Ops::add(si0, si1);
              part = C{wgt * (Ops::lo(sr) + Ops::hi(sr)), wgt * (Ops::lo(si) + Ops::hi(si))};
            }
          }
          red[warp][k][lane] = part;
        }
        __syncwarp();
        {
          // lane (k, quarter): sum of 8 lanes' partials of point j0 + k, then over quarters
          const int k = lane & (G - 1);
          const int q4 = lane / G;
          C sum{T(0), T(0)};
#pragma unroll
          for (int i = 0; i < 32 / 4; ++i) {
            const C v = red[warp][k][q4 * 8 + i];
            sum.x += v.x;
            sum.y += v.y;
          }
#pragma unroll
          for (int o = G; o < 32; o <<= 1) {
            sum.x += __shfl_xor_sync(0xffffffffu, sum.x, o);
            sum.y += __shfl_xor_sync(0xffffffffu, sum.y, o);
          }
          if (q4 == 0) res[warp][j0 + k] = sum;
        }
        __syncwarp();
      }
      __syncthreads();
      if (tid < nb) {
        C r = res[0][tid];
#pragma unroll
        for (int w = 1; w < S::NWARP; ++w) {
          r.x += res[w][tid].x;
          r.y += res[w][tid].y;
        }
        if (a.postphase) r = cmul(r, a.postphase[my_perm]);
        a.out[my_perm] = r;
      }
    }
    if (loader) {
      cp_async_wait_all();
#pragma unroll
      for (int q = 0; q < S::NP; ++q) {
        const C c0 = stage[ra][2 * q];
        const C c1 = stage[ra][2 * q + 1];
        gre[q] = Ops::pack(c0.x, c1.x);
        gim[q] = Ops::pack(c0.y, c1.y);
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
