// 3D ES spreading and interpolation with a sliding z-window held in registers (method 3).
//
// Replaces, for 3D plans with kernel width w <= 8, the reference's spreading
// (src/neonufft/gpu/kernels/spreading_kernel.cu:477-715, one global float atomic per cell and
// point) and interpolation (src/neonufft/gpu/kernels/interpolation_kernel.cu, one thread per
// point reading w^3 cells from global memory).
//
// Points are binned by (x tile of TX cells, y tile of 8 cells, single z plane), and the bins of
// one (x, y) column are consecutive in plane order (BinGeom::zmajor), so the points of a column
// and range of planes are one contiguous run of records. One CTA walks one column over a chunk
// of planes. Its region is P0 x P1 cells in (x, y), P0 = TX + w - 1 and P1 = 8 + w - 1 <= 15,
// times a window of RZ >= w consecutive planes [t, t + RZ):
//  * thread (a, b) keeps in registers the whole region row y = a (P0 cells, as pairs of
//    neighbouring cells) of the window plane p = b (mod RZ). The 16 rows are split over the
//    warps, LA = 32 / RZ rows per warp, so for a point whose footprint covers rows
//    [ly, ly + w) a warp either owns some of them or skips the point with a warp-uniform
//    branch; no thread holds a cell that another thread updates, so there are no atomics and
//    no shared-memory traffic per cell;
//  * the run of points is staged in shared memory 64 at a time (double-buffered, one barrier
//    per batch, spread over all warps): kx over the region's x range, ky over the 16 rows and
//    kz over the RZ planes, each zero outside the footprint, so that every thread applies
//    them with fixed register indices and no range tests;
//  * each owning thread updates its row with packed two-float FMAs (fma.rn.f32x2 on sm_100a),
//    one for the real and one for the imaginary parts of two neighbouring cells;
//  * when the next point starts on a later plane, the window advances: spreading adds each
//    completed plane to the fine grid (float2 / double2 atomics: neighbouring columns and
//    chunks overlap by the halo); interpolation reloads the threads that held it with the
//    plane RZ further on (plain loads: a cp.async prefetch one plane ahead measured no faster);
//  * interpolation reduces the row sums of eight points at a time through a per-warp
//    shared-memory transpose, then over warps.
#include <type_traits>

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
    float x;
    asm("mov.b64 {%0, _}, %1;" : "=f"(x) : "l"(v));
    return x;
  }
  static __device__ __forceinline__ float hi(P v) {
    float y;
    asm("mov.b64 {_, %0}, %1;" : "=f"(y) : "l"(v));
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
template <typename T, int W, int TX, int TY_ = 8>
struct ZShape {
  static constexpr int RZ = W <= 4 ? 4 : 8;         // window planes = z residues (>= W)
  static constexpr int LA = 32 / RZ;                // rows per warp
  static constexpr int TY = TY_;                    // tile y (4, 8 or 16)
  static constexpr int P1 = TY + W - 1;             // region y extent
  // region rows (>= P1, a multiple of the rows per warp)
  static constexpr int RY = TY == 4 ? (P1 + LA - 1) / LA * LA : TY + 8;
  static constexpr int NWARP = RY / LA;
  static constexpr int NT = 32 * NWARP;             // threads per CTA
  static constexpr int P0 = TX + W - 1;             // region x extent (cells)
  static constexpr int NP = (P0 + 1) / 2;           // cell pairs per row
  static constexpr int KXN = 4 * ((NP + 1) / 2);    // staged kx values (16-byte multiple)
  // points staged at a time: a multiple of the warps (each stages its share)
  static constexpr int BATCH =
      sizeof(T) == 4 ? (NWARP == 1 ? 32 : (NWARP % 3 == 0 ? 48 : 64)) : 32;
  static constexpr int G = 8;                       // points reduced together (interpolation)
  // CTAs per SM the interpolation kernel is compiled for: 6 in single precision (78 registers,
  // no spills; 86 uncapped, which allows only 5 CTAs and measured 6 % slower), 5 in double.
  static constexpr int INTERP_CTAS = sizeof(T) == 4 ? 6 : 5;
  // CTAs per SM the two-vector spreading kernel is compiled for: a budget of about 88 registers
  // a thread (7 CTAs of 96 threads; ptxas then allocates 80 registers and spills 24 bytes for
  // w = 8). Uncapped, the allocator takes 158 registers for w = 8, which leaves 2 CTAs per SM.
  static constexpr int SPREAD2_CTAS = 65536 / (NT * 88) > 0 ? 65536 / (NT * 88) : 1;
  static_assert(W <= RZ && P1 <= RY, "window smaller than the kernel footprint");
  static_assert(BATCH % NWARP == 0 && BATCH / NWARP <= 32, "staging threads");
};

// CTAs per SM the persistent kernels are compiled for: without the cap, their loop over items
// lets the register allocator grow far past the per-transform kernels (166 against 72).
template <typename T>
constexpr int kSpreadFusedCtas = sizeof(T) == 4 ? 7 : 4;
template <typename T>
constexpr int kInterpFusedCtas = sizeof(T) == 4 ? 6 : 4;

// Per-point data staged in shared memory (one slot per point of a batch).
template <typename T, int W, int TX, int TY = 8>
struct alignas(16) ZSlotFields {
  using S = ZShape<T, W, TX, TY>;
  T kx[S::KXN];    // kx over the region's x range, zero outside the footprint
  T ky[S::RY];     // ky over the region rows, zero outside the footprint
  T kz[S::RZ];     // kz per window offset, zero beyond w
  cplx_t<T> v;     // strength (spreading)
  int lyp;         // first footprint row | first footprint plane << 4
  u32 perm;        // original point index
};
// 16 bytes of padding when the fields span an even number of 16-byte units: with an odd slot
// stride, consecutive lanes staging consecutive slots store to different banks.
template <bool ODD>
struct ZSlotPad {
  int pad[4];
};
template <>
struct ZSlotPad<true> {};
template <typename T, int W, int TX, int TY = 8>
struct alignas(16) ZSlot
    : ZSlotFields<T, W, TX, TY>, ZSlotPad<(sizeof(ZSlotFields<T, W, TX, TY>) / 16) % 2 == 1> {};

// Stages `count` (<= 16) bin-sorted records `recs` into slots[0 .. count), one warp: lanes
// 0 .. count - 1 load the records (and, for spreading, the strengths; with `v2_out`, also the
// second vector's strengths from `in2`, or zeros where in2 is null, into v2_out[0 .. count), so
// that both gathers are in flight together); then lane pair
// (2p, 2p + 1) fills point p's slot with the same instruction stream: the even lane kx and the
// first half of kz, the odd lane ky and the second half, each zeroing half of the contiguous
// kx / ky arrays first, so all 32 lanes evaluate kernel values.
template <typename T, int W, int TX, bool SPREAD, int TY = 8>
__device__ __forceinline__ void stage_warp(ZSlot<T, W, TX, TY>* slots, const PointRec<T>* recs,
                                           int count, const cplx_t<T>* in,
                                           const cplx_t<T>* prephase, T beta, T c, int lane,
                                           i64 num, const cplx_t<T>* in2 = nullptr,
                                           cplx_t<T>* v2_out = nullptr) {
  using S = ZShape<T, W, TX, TY>;
  using C = cplx_t<T>;
  constexpr unsigned kFull = 0xffffffffu;
  PointRec<T> rec;
  rec.perm = 0;
  rec.local = 0;
  rec.frac[0] = rec.frac[1] = rec.frac[2] = T(0);
  C v{T(0), T(0)};
  if (lane < count) {
    rec = recs[lane];
    if constexpr (SPREAD) {
      C v2{T(0), T(0)};
      if (NNB_CHECK_INDEX(rec.perm, num)) {
        v = in[rec.perm];
        if (in2) v2 = in2[rec.perm];
        if (prephase) {
          const C ph = prephase[rec.perm];
          v = cmul(v, ph);
          v2 = cmul(v2, ph);
        }
      }
      if (v2_out) v2_out[lane] = v2;
    }
  }
  const int p = lane >> 1;
  const int h = lane & 1;
  const u32 loc = __shfl_sync(kFull, rec.local, p);
  const u32 perm = __shfl_sync(kFull, rec.perm, p);
  const T fx = __shfl_sync(kFull, rec.frac[0], p);
  const T fy = __shfl_sync(kFull, rec.frac[1], p);
  const T fz = __shfl_sync(kFull, rec.frac[2], p);
  const T vx = __shfl_sync(kFull, v.x, p);
  const T vy = __shfl_sync(kFull, v.y, p);
  ZSlot<T, W, TX, TY>& sl = slots[p < count ? p : 0];
  constexpr int kZero16 = int((S::KXN + S::RY) * sizeof(T) / 16);  // kx and ky are contiguous
  constexpr int kHalf = (kZero16 + 1) / 2;
  if (p < count) {
    float4* z = reinterpret_cast<float4*>(sl.kx);
#pragma unroll
    for (int i = 0; i < kHalf; ++i) {
      if (h * kHalf + i < kZero16) z[h * kHalf + i] = make_float4(0, 0, 0, 0);
    }
  }
  __syncwarp();
  if (p < count) {
    const int lx = int(loc & 0xFu);
    const int ly = int((loc >> 4) & 0xFu);
    T* dst = h ? sl.ky + ly : sl.kx + lx;
    const T f = h ? fy : fx;
#pragma unroll
    for (int k = 0; k < W; ++k) dst[k] = es_eval_fast<T>(f + T(k), beta, c);
#pragma unroll
    for (int i = 0; i < S::RZ / 2; ++i) {
      const int k = h * (S::RZ / 2) + i;
      sl.kz[k] = k < W ? es_eval_fast<T>(fz + T(k), beta, c) : T(0);
    }
    if (h == 0) {
      sl.v = C{vx, vy};
      sl.lyp = ly | int((loc >> 8) << 4);
      sl.perm = perm;
    }
  }
}

// base + off wrapped to [0, n) for 0 <= base < n, 0 <= off.
__device__ __forceinline__ i64 wrap_add(i64 base, int off, i64 n) {
  i64 i = base + off;
  while (i >= n) i -= n;
  return i;
}

// Column gx0 + i wrapped to the grid; `narrow` when the grid is narrower than the region.
__device__ __forceinline__ i64 wrap_x(i64 gx0, int i, i64 nfx, bool narrow) {
  i64 x = gx0 + i;
  if (narrow) {
    while (x >= nfx) x -= nfx;
  } else if (x >= nfx) {
    x -= nfx;
  }
  return x;
}

// Plane p (p >= 0, below nfz plus a window) wrapped into the grid.
__device__ __forceinline__ i64 wrap_plane(int p, i64 nfz) {
  i64 z = p;
  while (z >= nfz) z -= nfz;
  return z;
}

// Adds two neighbouring cells (re0, im0), (re1, im1) at a 16-byte aligned address.
__device__ __forceinline__ void atomic_add_pair(float2* p, float re0, float im0, float re1,
                                                float im1) {
  atomicAdd(reinterpret_cast<float4*>(p), make_float4(re0, im0, re1, im1));
}
__device__ __forceinline__ void atomic_add_pair(double2* p, double re0, double im0, double re1,
                                                double im1) {
  atomic_add_cplx(p, double2{re0, im0});
  atomic_add_cplx(p + 1, double2{re1, im1});
}

// CTA coordinates: column (tx, ty), plane range [z0, z1) and its run of points [pbeg, pend).
struct ZCta {
  int tx, ty, z0, z1;
  u32 pbeg, pend;
};
__device__ __forceinline__ bool zcta(const BinGeom& g, const u32* bin_start, ZChunks ch,
                                     const WorkList& wl, u32 item, ZCta& c) {
  u32 unit, slice;
  if (!work_item_at(wl, item, unit, slice)) return false;
  const i64 ncols = i64(g.ntiles[0]) * g.ntiles[1];
  const int chunk = int(unit / ncols);
  const i64 col = unit - i64(chunk) * ncols;
  c.tx = int(col % g.ntiles[0]);
  c.ty = int(col / g.ntiles[0]);
  const int nz = g.ntiles[2];  // == nf[2]: single-plane tiles
  c.z0 = chunk * ch.len;
  c.z1 = min(c.z0 + ch.len, nz);
  const u32* bs = bin_start + col * nz;
  work_slice(bs[c.z0], bs[c.z1], slice, wl.cap, c.pbeg, c.pend);
  return c.pbeg < c.pend;
}

// Thread layout shared by both kernels.
template <typename T, int W, int TX, int TY = 8>
struct ZThread {
  using S = ZShape<T, W, TX, TY>;
  int tid, warp, lane, ra, rb, a_lo;
  int stage_j;  // batch slot this thread stages (< BATCH), or -1
  __device__ __forceinline__ ZThread() {
    tid = threadIdx.x;
    warp = tid >> 5;
    lane = tid & 31;
    ra = warp * S::LA + lane % S::LA;  // region row
    rb = lane / S::LA;                  // z residue
    a_lo = warp * S::LA;                // first row of this warp
    // consecutive lanes stage consecutive slots (the slot stride is 4 words times an odd
    // number, so their shared-memory stores fall in different banks)
    stage_j = lane < S::BATCH / S::NWARP ? warp * (S::BATCH / S::NWARP) + lane : -1;
  }
  // Whether this warp owns rows of a footprint starting at row ly.
  __device__ __forceinline__ bool owns(int ly) const { return ly < a_lo + S::LA && ly + W > a_lo; }
};

// ---- spreading ---------------------------------------------------------------------------------
// NV strength vectors on the same points (NV = 2: the second vector's staged strengths).
template <typename T, int W, int TX, int TY = 8, int NV = 1>
struct ZSpreadShared {
  ZSlot<T, W, TX, TY> slots[2][ZShape<T, W, TX, TY>::BATCH];
  cplx_t<T> v2[2][NV > 1 ? ZShape<T, W, TX, TY>::BATCH : 1];
};

// Spreads work item `item` of batch entries batch .. batch + NV - 1 (one CTA; every thread
// calls it). With NV = 2 each staged point, its kernel values and the window's bookkeeping
// serve two strength vectors on the same points (type-3 batches, repeated type-1 transforms):
// the second vector's row sums sit in their own registers and go to the next grid (at
// grid_bdist); a missing second entry (an odd batch) is skipped.
template <typename T, int W, int TX, int TY = 8, int NV = 1>
__device__ __forceinline__ void spread_zwin_item(const SpreadArgs<T>& a, ZChunks ch,
                                                 const WorkList& wl, u32 item, int batch,
                                                 ZSpreadShared<T, W, TX, TY, NV>& sh) {
  static_assert(NV == 1 || NV == 2, "one or two strength vectors per pass");
  using S = ZShape<T, W, TX, TY>;
  using Ops = Packed<T>;
  using P = typename Ops::P;
  using C = cplx_t<T>;
  using Slot = ZSlot<T, W, TX, TY>;
  auto& slots = sh.slots;

  const BinGeom& g = a.g;
  ZCta cta;
  if (!zcta(g, a.pts.bin_start, ch, wl, item, cta)) return;
  const ZThread<T, W, TX, TY> th;
  const C* in = a.in + batch * a.in_bdist;
  C* grid = a.grid + batch * a.grid_bdist;
  const bool has2 = NV > 1 && batch + 1 < a.batch;  // the second vector exists
  const i64 nfx = g.nf[0], nfy = g.nf[1], nfz = g.nf[2];
  [[maybe_unused]] const i64 cells = nfx * nfy * nfz;
  const bool narrow = nfx < S::P0;
  const bool has_row = th.ra < S::P1;
  const i64 row_y = has_row ? wrap_add(i64(cta.ty) * S::TY, th.ra, nfy) : 0;
  const i64 gx0 = i64(cta.tx) * TX;

  // real / imaginary parts of cell pairs (2q, 2q + 1) of the row, per strength vector
  P are[NV][S::NP], aim[NV][S::NP];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
#pragma unroll
    for (int q = 0; q < S::NP; ++q) are[v][q] = aim[v][q] = Ops::zero();
  }
  bool dirty = false;

  // Adds this thread's row of plane p (absolute; may exceed nfz) to the grid(s) and clears it.
  // The region's x range lies inside the grid and its rows start 16-byte aligned (the usual
  // case): whole cell pairs are added with one vector atomic each.
  const bool pairs = !narrow && gx0 + S::P0 <= nfx && (nfx % 2) == 0 &&
                     (reinterpret_cast<size_t>(grid) % 16) == 0 &&
                     (NV == 1 || (a.grid_bdist % 2) == 0);
  auto flush = [&](int p) {
    if (has_row && dirty) {
      const i64 base = (wrap_plane(p, nfz) * nfy + row_y) * nfx;
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        if (v == 1 && !has2) break;
        C* row = grid + v * a.grid_bdist + base;
        if (pairs) {
          C* r = row + gx0;
#pragma unroll
          for (int q = 0; q < S::NP; ++q) {
            if (2 * q + 1 < S::P0) {
              if (NNB_CHECK_INDEX(base + gx0 + 2 * q + 1, cells)) {
                atomic_add_pair(r + 2 * q, Ops::lo(are[v][q]), Ops::lo(aim[v][q]),
                                Ops::hi(are[v][q]), Ops::hi(aim[v][q]));
              }
            } else if (NNB_CHECK_INDEX(base + gx0 + 2 * q, cells)) {
              atomic_add_cplx(r + 2 * q, C{Ops::lo(are[v][q]), Ops::lo(aim[v][q])});
            }
          }
        } else {
#pragma unroll
          for (int q = 0; q < S::NP; ++q) {
            const i64 x0 = wrap_x(gx0, 2 * q, nfx, narrow);
            if (NNB_CHECK_INDEX(base + x0, cells)) {
              atomic_add_cplx(&row[x0], C{Ops::lo(are[v][q]), Ops::lo(aim[v][q])});
            }
            const i64 x1 = wrap_x(gx0, 2 * q + 1, nfx, narrow);
            if (2 * q + 1 < S::P0 && NNB_CHECK_INDEX(base + x1, cells)) {
              atomic_add_cplx(&row[x1], C{Ops::hi(are[v][q]), Ops::hi(aim[v][q])});
            }
          }
        }
      }
#pragma unroll
      for (int v = 0; v < NV; ++v) {
#pragma unroll
        for (int q = 0; q < S::NP; ++q) are[v][q] = aim[v][q] = Ops::zero();
      }
    }
    dirty = false;
  };

  const u32 npts = cta.pend - cta.pbeg;
  const int nbatch = int((npts + S::BATCH - 1) / S::BATCH);
  auto stage = [&](int k) {
    const u32 off = u32(k) * S::BATCH;
    const int nb = int(min(npts - off, u32(S::BATCH)));
    constexpr int PW = S::BATCH / S::NWARP;  // points per warp
    const int count = min(nb - th.warp * PW, PW);
    for (int c0 = 0; c0 < count; c0 += 16) {
      if (!NNB_CHECK_INDEX(i64(cta.pbeg) + off + th.warp * PW + c0 + min(count - c0, 16) - 1,
                           a.pts.M)) {
        break;
      }
      // NV = 2: the second vector's strengths at the same points (zeros when it is missing)
      stage_warp<T, W, TX, true, TY>(slots[k & 1] + th.warp * PW + c0,
                                 a.pts.rec + cta.pbeg + off + th.warp * PW + c0,
                                 min(count - c0, 16), in, a.prephase, a.beta, a.c, th.lane,
                                 a.pts.M, NV > 1 && has2 ? in + a.in_bdist : nullptr,
                                 NV > 1 ? sh.v2[k & 1] + th.warp * PW + c0 : nullptr);
    }
  };

  stage(0);
  __syncthreads();
  int cur = slots[0][0].lyp >> 4;  // window start: the first point's plane
  int dz = (th.rb - cur) & (S::RZ - 1);
  for (int k = 0; k < nbatch; ++k) {
    const int nb = int(min(npts - u32(k) * S::BATCH, u32(S::BATCH)));
    const Slot* sb = slots[k & 1];
    constexpr int NH = (S::BATCH + 31) / 32;
    if constexpr (NV == 1) {
      // The points of this batch whose footprint covers rows of this warp, one bit per slot:
      // the warp visits only those, with a window of its own (no other warp touches its rows).
      u32 own[NH];
#pragma unroll
      for (int h = 0; h < NH; ++h) {
        const int j = h * 32 + th.lane;
        own[h] = __ballot_sync(0xffffffffu, j < nb && th.owns(sb[j < nb ? j : 0].lyp & 15));
      }
#pragma unroll
      for (int h = 0; h < NH; ++h) {
        for (u32 m = own[h]; m != 0u; m &= m - 1u) {
          const int si = h * 32 + __ffs(int(m)) - 1;
          const Slot& sl = sb[si];
          const int tp = sl.lyp >> 4;
          if (tp != cur) {  // advance the window: planes [cur, tp) are complete
            const int n = min(tp - cur, S::RZ);
            for (int i = 0; i < n; ++i) {
              if (th.rb == ((cur + i) & (S::RZ - 1))) flush(cur + i);
            }
            cur = tp;
            dz = (th.rb - cur) & (S::RZ - 1);
          }
          dirty = true;
          const T kw = sl.ky[th.ra] * sl.kz[dz];
          const C v = sl.v;
          const P wre = Ops::splat(v.x * kw);
          const P wim = Ops::splat(v.y * kw);
#pragma unroll
          for (int q = 0; q < S::NP; q += 2) {
            P kk[2];
            load_pairs<T>(&sl.kx[2 * q], kk);
#pragma unroll
            for (int u = 0; u < 2; ++u) {
              if (q + u < S::NP) {
                are[0][q + u] = Ops::fma(kk[u], wre, are[0][q + u]);
                aim[0][q + u] = Ops::fma(kk[u], wim, aim[0][q + u]);
              }
            }
          }
        }
      }
    } else {
      // Two vectors: the owned points are visited one plane at a time (the slots are in plane
      // order), so that the window moves once per plane and the loop over a plane's points
      // holds only the loads and the FMAs. (Measured at 1e8 points on a 512^3 grid, w = 8,
      // tiles 4 x 4 x 1: 28.8 ms per two-vector pass against 32.7 ms with the single-vector
      // loop; that loop stays the faster one for one vector, 17.3 against 17.7 ms.)
      u32 own[NH];
      int pl[NH];  // plane of slot 32 h + lane
#pragma unroll
      for (int h = 0; h < NH; ++h) {
        const int j = h * 32 + th.lane;
        const int lyp = sb[j < nb ? j : 0].lyp;
        pl[h] = lyp >> 4;
        own[h] = __ballot_sync(0xffffffffu, j < nb && th.owns(lyp & 15));
      }
#pragma unroll
      for (int h = 0; h < NH; ++h) {
        u32 m = own[h];
        while (m != 0u) {
          const int tp = __shfl_sync(0xffffffffu, pl[h], __ffs(int(m)) - 1);
          const u32 run = m & __ballot_sync(0xffffffffu, pl[h] == tp);
          m &= ~run;
          if (tp != cur) {  // advance the window: planes [cur, tp) are complete
            const int n = min(tp - cur, S::RZ);
            for (int i = 0; i < n; ++i) {
              if (th.rb == ((cur + i) & (S::RZ - 1))) flush(cur + i);
            }
            cur = tp;
            dz = (th.rb - cur) & (S::RZ - 1);
          }
          dirty = true;
          for (u32 r = run; r != 0u; r &= r - 1u) {
            const int si = h * 32 + __ffs(int(r)) - 1;
            const Slot& sl = sb[si];
            const T kw = sl.ky[th.ra] * sl.kz[dz];
            P wre[NV], wim[NV];
            {
              const C v = sl.v;
              wre[0] = Ops::splat(v.x * kw);
              wim[0] = Ops::splat(v.y * kw);
              const C v2 = sh.v2[k & 1][si];
              wre[1] = Ops::splat(v2.x * kw);
              wim[1] = Ops::splat(v2.y * kw);
            }
#pragma unroll
            for (int q = 0; q < S::NP; q += 2) {
              P kk[2];
              load_pairs<T>(&sl.kx[2 * q], kk);
#pragma unroll
              for (int u = 0; u < 2; ++u) {
                if (q + u < S::NP) {
#pragma unroll
                  for (int v = 0; v < NV; ++v) {
                    are[v][q + u] = Ops::fma(kk[u], wre[v], are[v][q + u]);
                    aim[v][q + u] = Ops::fma(kk[u], wim[v], aim[v][q + u]);
                  }
                }
              }
            }
          }
        }
      }
    }
    if (k + 1 < nbatch) stage(k + 1);
    __syncthreads();
  }
  flush(cur + ((th.rb - cur) & (S::RZ - 1)));  // the rest of the window
}

template <typename T, int W, int TX, int TY>
__global__ void __launch_bounds__(ZShape<T, W, TX, TY>::NT)
    spread_zwin_kernel(const __grid_constant__ SpreadArgs<T> a, ZChunks ch,
                       const __grid_constant__ WorkList wl) {
  __shared__ ZSpreadShared<T, W, TX, TY> sh;
  spread_zwin_item<T, W, TX, TY>(a, ch, wl, blockIdx.x, int(blockIdx.y), sh);
}

// Two strength vectors per CTA: batch entries 2 blockIdx.y and 2 blockIdx.y + 1.
template <typename T, int W, int TX, int TY>
__global__ void __launch_bounds__(ZShape<T, W, TX, TY>::NT, ZShape<T, W, TX, TY>::SPREAD2_CTAS)
    spread_zwin2_kernel(const __grid_constant__ SpreadArgs<T> a, ZChunks ch,
                        const __grid_constant__ WorkList wl) {
  __shared__ ZSpreadShared<T, W, TX, TY, 2> sh;
  spread_zwin_item<T, W, TX, TY, 2>(a, ch, wl, blockIdx.x, 2 * int(blockIdx.y), sh);
}

// Takes the next item of the queue spanning all jobs; every thread returns the same values.
// The job's record is copied to shared memory once per item.
template <typename Job>
__device__ __forceinline__ bool next_fused_item(const Job* jobs, const i64* item_end, int njobs,
                                                i64 total, u32* queue, Job& job, u32& local) {
  __shared__ i64 s_item;
  __shared__ int s_job;
  if (threadIdx.x == 0) {
    const i64 it = i64(atomicAdd(queue, 1u));
    int lo = 0, hi = njobs;  // first job whose cumulative item count exceeds it
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (item_end[mid] > it) {
        hi = mid;
      } else {
        lo = mid + 1;
      }
    }
    s_item = it;
    s_job = lo;
  }
  __syncthreads();
  const i64 it = s_item;
  const int j = s_job;
  if (it >= total || j >= njobs) return false;
  static_assert(sizeof(Job) % 4 == 0, "job records are copied in words");
  const int* src = reinterpret_cast<const int*>(jobs + j);
  int* dst = reinterpret_cast<int*>(&job);
  for (int k = int(threadIdx.x); k < int(sizeof(Job) / 4); k += int(blockDim.x)) dst[k] = src[k];
  local = u32(it - (j > 0 ? item_end[j - 1] : 0));
  __syncthreads();
  return true;
}

template <typename T, int W, int TX>
__global__ void __launch_bounds__(ZShape<T, W, TX>::NT, kSpreadFusedCtas<T>)
    spread_zwin_fused_kernel(const ZSpreadJob<T>* jobs, const i64* item_end, int njobs,
                             i64 total, u32* queue) {
  __shared__ ZSpreadShared<T, W, TX> sh;
  __shared__ ZSpreadJob<T> job;
  u32 local;
  while (next_fused_item(jobs, item_end, njobs, total, queue, job, local)) {
    spread_zwin_item<T, W, TX>(job.a, job.ch, job.wl, local, 0, sh);
    __syncthreads();  // the job record and the slots are rewritten for the next item
  }
}

// ---- spreading on the tensor cores (method 4, single precision, 5 <= w <= 8) ---------------------
//
// The same window, staging and flushes as spread_zwin_kernel, with the per-point row updates
// replaced by TF32 tensor-core products. For a chunk of up to 8 points of the current plane,
//   region[x, (plane, y)] += sum_p kx_p[x] * (v_p ky_p[y] kz_p[plane])
// is, for each tile of one plane and 8 rows, a 16 x 8 x 8 matrix product (mma.sync m16n8k8:
// M = the 16 x cells of the region, K = the points, N = the rows). Both operands are split into
// a TF32 value and a TF32 remainder and the product accumulated as hi*hi + hi*lo + lo*hi in FP32
// (about 2^-21 of each product). Warp w owns window planes 2w, 2w + 1 (mod 8) and both 8-row y
// groups: four tiles, real and imaginary accumulators in registers; in the m16n8k8 fragment
// layout thread (q, t) = (lane / 4, lane % 4) holds x = q, q + 8 and rows 2t, 2t + 1 of a tile.
// A completed plane is added to the grid by its owning warp (all 32 lanes, float2 atomics).

__device__ __forceinline__ unsigned to_tf32(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void tf32_split(float x, unsigned& hi, unsigned& lo) {
  hi = to_tf32(x);
  lo = to_tf32(x - __uint_as_float(hi));
}
// c += a * b for one m16n8k8 TF32 tile (FP32 accumulation)
__device__ __forceinline__ void mma_tf32(float* c, const unsigned* a, unsigned b0, unsigned b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
// c += a * b with both operands split (3 products). The products of one chunk are summed on the
// tensor core into a fresh tile and added to the accumulator with ordinary FP32 adds: chaining
// the accumulator through every MMA of a long run of points loses accuracy.
__device__ __forceinline__ void mma_tf32x3(float* c, const unsigned* ahi, const unsigned* alo,
                                           float b0, float b1) {
  unsigned b0h, b0l, b1h, b1l;
  tf32_split(b0, b0h, b0l);
  tf32_split(b1, b1h, b1l);
  float t[4] = {0.f, 0.f, 0.f, 0.f};
  mma_tf32(t, alo, b0h, b1h);
  mma_tf32(t, ahi, b0l, b1l);
  mma_tf32(t, ahi, b0h, b1h);
#pragma unroll
  for (int e = 0; e < 4; ++e) c[e] += t[e];
}

template <int W>
__global__ void __launch_bounds__(128) spread_zmma_kernel(SpreadArgs<float> a, ZChunks ch,
                                                          WorkList wl) {
  constexpr int TX = 8;
  using S = ZShape<float, W, TX>;
  static_assert(S::RZ == 8 && S::NWARP == 4 && S::P0 <= 16, "tile shapes");
  using C = float2;
  using Slot = ZSlot<float, W, TX>;
  __shared__ Slot slots[2][S::BATCH];

  const BinGeom& g = a.g;
  ZCta cta;
  if (!zcta(g, a.pts.bin_start, ch, wl, blockIdx.x, cta)) return;
  const ZThread<float, W, TX> th;
  const int gq = th.lane >> 2;  // fragment row group
  const int tq = th.lane & 3;   // thread in group
  const bool hi8 = gq + 8 < S::KXN;  // staged kx covers x = gq + 8 (cells beyond it are zero)
  const int batch = blockIdx.y;
  const C* in = a.in + batch * a.in_bdist;
  C* grid = a.grid + batch * a.grid_bdist;
  const i64 nfx = g.nf[0], nfy = g.nf[1], nfz = g.nf[2];
  const bool narrow = nfx < S::P0;
  const i64 gx0 = i64(cta.tx) * TX;
  const i64 gy0 = i64(cta.ty) * S::TY;

  float cre[2][2][4], cim[2][2][4];  // [plane of the warp][y group][fragment element]
#pragma unroll
  for (int pl = 0; pl < 2; ++pl) {
#pragma unroll
    for (int yg = 0; yg < 2; ++yg) {
#pragma unroll
      for (int e = 0; e < 4; ++e) cre[pl][yg][e] = cim[pl][yg][e] = 0.f;
    }
  }
  unsigned dirty = 0;  // plane residues with contributions since their last flush

  // Adds the warp's tiles of window plane p (residue 2 warp + pl) to the grid and clears them.
  auto flush = [&](int pl, int p) {
    const unsigned bit = 1u << (2 * th.warp + pl);
    if (dirty & bit) {
      const i64 plane = wrap_plane(p, nfz);
#pragma unroll
      for (int yg = 0; yg < 2; ++yg) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int x = gq + 8 * (e >> 1);
          const int y = 8 * yg + 2 * tq + (e & 1);
          if (x < S::P0 && y < S::P1) {
            const i64 gy = wrap_add(gy0, y, nfy);
            const i64 idx = (plane * nfy + gy) * nfx + wrap_x(gx0, x, nfx, narrow);
            if (NNB_CHECK_INDEX(idx, nfx * nfy * nfz)) {
              atomic_add_cplx(&grid[idx], C{cre[pl][yg][e], cim[pl][yg][e]});
            }
          }
          cre[pl][yg][e] = cim[pl][yg][e] = 0.f;
        }
      }
      dirty &= ~bit;
    }
  };
  auto flush_plane = [&](int p) {
    const int b = p & 7;
    if ((b >> 1) == th.warp) flush(b & 1, p);
  };

  const u32 npts = cta.pend - cta.pbeg;
  const int nbatch = int((npts + S::BATCH - 1) / S::BATCH);
  auto stage = [&](int k) {
    const u32 off = u32(k) * S::BATCH;
    const int nb = int(min(npts - off, u32(S::BATCH)));
    constexpr int PW = S::BATCH / S::NWARP;
    const int count = min(nb - th.warp * PW, PW);
    for (int c0 = 0; c0 < count; c0 += 16) {
      if (!NNB_CHECK_INDEX(i64(cta.pbeg) + off + th.warp * PW + c0 + min(count - c0, 16) - 1,
                           a.pts.M)) {
        break;
      }
      stage_warp<float, W, TX, true>(slots[k & 1] + th.warp * PW + c0,
                                     a.pts.rec + cta.pbeg + off + th.warp * PW + c0,
                                     min(count - c0, 16), in, a.prephase, a.beta, a.c, th.lane,
                                     a.pts.M);
    }
  };

  stage(0);
  __syncthreads();
  int cur = slots[0][0].lyp >> 4;
  int dz0 = (2 * th.warp - cur) & 7, dz1 = (2 * th.warp + 1 - cur) & 7;
  for (int k = 0; k < nbatch; ++k) {
    const int nb = int(min(npts - u32(k) * S::BATCH, u32(S::BATCH)));
    const Slot* sb = slots[k & 1];
    int j = 0;
    while (j < nb) {
      const int tp = sb[j].lyp >> 4;
      if (tp != cur) {  // advance the window: planes [cur, tp) are complete
        const int n = min(tp - cur, S::RZ);
        for (int i = 0; i < n; ++i) flush_plane(cur + i);
        cur = tp;
        dz0 = (2 * th.warp - cur) & 7;
        dz1 = (2 * th.warp + 1 - cur) & 7;
      }
      // the chunk: points j .. j + n - 1 of plane cur (a prefix, the points are plane-sorted)
      const bool on = th.lane < 8 && j + th.lane < nb && (sb[min(j + th.lane, nb - 1)].lyp >> 4) == cur;
      const int n = __popc(__ballot_sync(0xffffffffu, on));
      const bool h0 = tq < n, h1 = tq + 4 < n;
      const Slot& s0 = sb[h0 ? j + tq : j];
      const Slot& s1 = sb[h1 ? j + tq + 4 : j];
      // A: kx of points tq, tq + 4 at x = gq, gq + 8
      unsigned ahi[4], alo[4];
      tf32_split(h0 ? s0.kx[gq] : 0.f, ahi[0], alo[0]);
      tf32_split(h0 && hi8 ? s0.kx[gq + 8] : 0.f, ahi[1], alo[1]);
      tf32_split(h1 ? s1.kx[gq] : 0.f, ahi[2], alo[2]);
      tf32_split(h1 && hi8 ? s1.kx[gq + 8] : 0.f, ahi[3], alo[3]);
      // B: v ky kz of points tq, tq + 4 at row gq of each tile
      const C v0 = h0 ? s0.v : C{0.f, 0.f};
      const C v1 = h1 ? s1.v : C{0.f, 0.f};
      const float y00 = s0.ky[gq], y01 = s0.ky[gq + 8], z00 = s0.kz[dz0], z01 = s0.kz[dz1];
      const float y10 = s1.ky[gq], y11 = s1.ky[gq + 8], z10 = s1.kz[dz0], z11 = s1.kz[dz1];
#pragma unroll
      for (int pl = 0; pl < 2; ++pl) {
#pragma unroll
        for (int yg = 0; yg < 2; ++yg) {
          const float w0 = (yg ? y01 : y00) * (pl ? z01 : z00);
          const float w1 = (yg ? y11 : y10) * (pl ? z11 : z10);
          mma_tf32x3(cre[pl][yg], ahi, alo, v0.x * w0, v1.x * w1);
          mma_tf32x3(cim[pl][yg], ahi, alo, v0.y * w0, v1.y * w1);
        }
      }
      dirty = 0xffu;
      j += n;
    }
    if (k + 1 < nbatch) stage(k + 1);
    __syncthreads();
  }
  for (int i = 0; i < S::RZ; ++i) flush_plane(cur + i);  // the rest of the window
}

// ---- interpolation -----------------------------------------------------------------------------
template <typename T, int W, int TX, int TY = 8>
struct ZInterpShared {
  using S = ZShape<T, W, TX, TY>;
  static constexpr int RS = 33;  // odd row stride of the transpose buffer: conflict-free reads
  ZSlot<T, W, TX, TY> slots[2][S::BATCH];
  cplx_t<T> red[S::NWARP][S::G][RS];
  cplx_t<T> res[2][S::NWARP][S::BATCH];
};

// Interpolates work item `item` (one CTA; every thread calls it).
template <typename T, int W, int TX, int TY = 8>
__device__ __forceinline__ void interp_zwin_item(const InterpArgs<T>& a, ZChunks ch,
                                                 const WorkList& wl, u32 item,
                                                 ZInterpShared<T, W, TX, TY>& sh) {
  using S = ZShape<T, W, TX, TY>;
  using Ops = Packed<T>;
  using P = typename Ops::P;
  using C = cplx_t<T>;
  using Slot = ZSlot<T, W, TX, TY>;
  constexpr int G = S::G;
  auto& slots = sh.slots;
  auto& red = sh.red;
  auto& res = sh.res;

  const BinGeom& g = a.g;
  ZCta cta;
  if (!zcta(g, a.pts.bin_start, ch, wl, item, cta)) return;
  const ZThread<T, W, TX, TY> th;
  const C* grid = a.grid;
  const i64 nfx = g.nf[0], nfy = g.nf[1], nfz = g.nf[2];
  [[maybe_unused]] const i64 cells = nfx * nfy * nfz;
  const bool narrow = nfx < S::P0;
  const bool has_row = th.ra < S::P1;
  const i64 row_y = has_row ? wrap_add(i64(cta.ty) * S::TY, th.ra, nfy) : 0;
  const i64 gx0 = i64(cta.tx) * TX;

  // Row values of the window plane: real / imaginary parts of cell pairs (2q, 2q + 1); rows
  // outside the region stay zero.
  P gre[S::NP], gim[S::NP];
#pragma unroll
  for (int q = 0; q < S::NP; ++q) gre[q] = gim[q] = Ops::zero();
  // The region's x range lies inside the grid (the usual case): contiguous row segments.
  const bool contiguous = !narrow && gx0 + S::P0 <= nfx;
  // ... and its cell pairs start 16-byte aligned (single precision): one 16-byte load per pair
  const bool pairs16 = sizeof(T) == 4 && contiguous && (nfx % 2) == 0 &&
                       (reinterpret_cast<size_t>(grid) % 16) == 0;
  auto load_row = [&](int p) {
    if (!has_row) return;
    const i64 base = (wrap_plane(p, nfz) * nfy + row_y) * nfx;
    const C* row = grid + base;
    if constexpr (sizeof(T) == 4) {
      if (pairs16) {
#pragma unroll
        for (int q = 0; q < S::NP; ++q) {
          if (2 * q + 1 < S::P0) {
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (NNB_CHECK_INDEX(base + gx0 + 2 * q + 1, cells)) {
              v = *reinterpret_cast<const float4*>(row + gx0 + 2 * q);
            }
            gre[q] = Ops::pack(v.x, v.z);
            gim[q] = Ops::pack(v.y, v.w);
          } else {
            C c0{T(0), T(0)};
            if (NNB_CHECK_INDEX(base + gx0 + 2 * q, cells)) c0 = row[gx0 + 2 * q];
            gre[q] = Ops::pack(c0.x, T(0));
            gim[q] = Ops::pack(c0.y, T(0));
          }
        }
        return;
      }
    }
#pragma unroll
    for (int q = 0; q < S::NP; ++q) {
      C c0{T(0), T(0)}, c1{T(0), T(0)};
      const i64 x0 = contiguous ? gx0 + 2 * q : wrap_x(gx0, 2 * q, nfx, narrow);
      const i64 x1 = contiguous ? gx0 + 2 * q + 1 : wrap_x(gx0, 2 * q + 1, nfx, narrow);
      if (NNB_CHECK_INDEX(base + x0, cells)) c0 = row[x0];
      if (2 * q + 1 < S::P0 && NNB_CHECK_INDEX(base + x1, cells)) c1 = row[x1];
      gre[q] = Ops::pack(c0.x, c1.x);
      gim[q] = Ops::pack(c0.y, c1.y);
    }
  };
  const u32 npts = cta.pend - cta.pbeg;
  const int nbatch = int((npts + S::BATCH - 1) / S::BATCH);
  auto stage = [&](int k) {
    const u32 off = u32(k) * S::BATCH;
    const int nb = int(min(npts - off, u32(S::BATCH)));
    constexpr int PW = S::BATCH / S::NWARP;  // points per warp
    const int count = min(nb - th.warp * PW, PW);
    for (int c0 = 0; c0 < count; c0 += 16) {
      if (!NNB_CHECK_INDEX(i64(cta.pbeg) + off + th.warp * PW + c0 + min(count - c0, 16) - 1,
                           a.pts.M)) {
        break;
      }
      stage_warp<T, W, TX, false, TY>(slots[k & 1] + th.warp * PW + c0,
                                  a.pts.rec + cta.pbeg + off + th.warp * PW + c0,
                                  min(count - c0, 16), nullptr, nullptr, a.beta, a.c, th.lane,
                                  a.pts.M);
    }
  };
  // Writes the outputs of batch k: this thread's staged point, whose slot only this thread's
  // next staging rewrites.
  auto output = [&](int k) {
    const int nb = int(min(npts - u32(k) * S::BATCH, u32(S::BATCH)));
    const int j = th.stage_j;
    if (j >= 0 && j < nb) {
      C r = res[k & 1][0][j];
#pragma unroll
      for (int w = 1; w < S::NWARP; ++w) {
        r.x += res[k & 1][w][j].x;
        r.y += res[k & 1][w][j].y;
      }
      const u32 perm = slots[k & 1][j].perm;
      if (NNB_CHECK_INDEX(perm, a.pts.M)) {
        if (a.postphase) r = cmul(r, a.postphase[perm]);
        a.out[perm] = r;
      }
    }
  };

  stage(0);
  __syncthreads();
  int cur = slots[0][0].lyp >> 4;  // window start: the first point's plane
  int dz = (th.rb - cur) & (S::RZ - 1);
  load_row(cur + dz);

  for (int k = 0; k < nbatch; ++k) {
    const int nb = int(min(npts - u32(k) * S::BATCH, u32(S::BATCH)));
    const Slot* sb = slots[k & 1];
    // The points of this batch whose footprint covers rows of this warp (bit j: slot j).
    unsigned long long own = 0ull;
#pragma unroll
    for (int h = 0; h < (S::BATCH + 31) / 32; ++h) {
      const int j = h * 32 + th.lane;
      const u32 bits = __ballot_sync(0xffffffffu, j < nb && th.owns(sb[j < nb ? j : 0].lyp & 15));
      own |= (unsigned long long)bits << (32 * h);
    }
    // Row sum of an owned point over this thread's row, times ky kz.
    auto partial = [&](const Slot& sl) -> C {
      const T kw = sl.ky[th.ra] * sl.kz[dz];
      P sr0 = Ops::zero(), sr1 = Ops::zero(), si0 = Ops::zero(), si1 = Ops::zero();
#pragma unroll
      for (int q = 0; q < S::NP; q += 2) {
        P kp[2];
        load_pairs<T>(&sl.kx[2 * q], kp);
        sr0 = Ops::fma(kp[0], gre[q], sr0);
        si0 = Ops::fma(kp[0], gim[q], si0);
        if (q + 1 < S::NP) {
          sr1 = Ops::fma(kp[1], gre[q + 1], sr1);
          si1 = Ops::fma(kp[1], gim[q + 1], si1);
        }
      }
      const P sr = Ops::add(sr0, sr1);
      const P si = Ops::add(si0, si1);
      return C{kw * (Ops::lo(sr) + Ops::hi(sr)), kw * (Ops::lo(si) + Ops::hi(si))};
    };
    for (int j0 = 0; j0 < nb; j0 += G) {
      // Points are plane-sorted: if the group's last point is on the window's first plane, so
      // are all of them and the window does not move inside the group.
      // ownership bits of the group (bit kk: slot j0 + kk); zero past the batch's points
      const u32 ob = u32(own >> j0);
      if ((sb[min(j0 + G, nb) - 1].lyp >> 4) == cur) {
        const Slot* g0 = sb + j0;
#pragma unroll
        for (int kk = 0; kk < G; ++kk) {
          red[th.warp][kk][th.lane] = ((ob >> kk) & 1u) ? partial(g0[kk]) : C{T(0), T(0)};
        }
      } else {
#pragma unroll 1
        for (int kk = 0; kk < G; ++kk) {
          C part{T(0), T(0)};
          const int j = j0 + kk;
          if (j < nb) {
            const Slot& sl = sb[j];
            const int lyp = sl.lyp;
            const int tp = lyp >> 4;
            if (tp != cur) {  // advance the window: rows of planes [cur, tp) move on by RZ
              if (tp - cur >= S::RZ) {
                load_row(tp + ((th.rb - tp) & (S::RZ - 1)));
              } else {
                for (int i = 0; i < tp - cur; ++i) {
                  if (th.rb == ((cur + i) & (S::RZ - 1))) load_row(cur + i + S::RZ);
                }
              }
              cur = tp;
              dz = (th.rb - cur) & (S::RZ - 1);
            }
            if ((ob >> kk) & 1u) part = partial(sl);
          }
          red[th.warp][kk][th.lane] = part;
        }
      }
      __syncwarp();
      {
        // lane (k8, quarter): sum of 8 lanes' partials of point j0 + k8, then over quarters
        const int k8 = th.lane & (G - 1);
        const int q4 = th.lane / G;
        C sum{T(0), T(0)};
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const C v = red[th.warp][k8][q4 * 8 + i];
          sum.x += v.x;
          sum.y += v.y;
        }
#pragma unroll
        for (int o = G; o < 32; o <<= 1) {
          sum.x += __shfl_xor_sync(0xffffffffu, sum.x, o);
          sum.y += __shfl_xor_sync(0xffffffffu, sum.y, o);
        }
        if (q4 == 0) res[k & 1][th.warp][j0 + k8] = sum;
      }
      __syncwarp();
    }
    if (k > 0) output(k - 1);
    if (k + 1 < nbatch) stage(k + 1);
    __syncthreads();
  }
  output(nbatch - 1);
}

template <typename T, int W, int TX, int TY>
__global__ void __launch_bounds__(ZShape<T, W, TX, TY>::NT, ZShape<T, W, TX, TY>::INTERP_CTAS)
    interp_zwin_kernel(const __grid_constant__ InterpArgs<T> a, ZChunks ch,
                       const __grid_constant__ WorkList wl) {
  __shared__ ZInterpShared<T, W, TX, TY> sh;
  interp_zwin_item<T, W, TX, TY>(a, ch, wl, blockIdx.x, sh);
}

template <typename T, int W, int TX>
__global__ void __launch_bounds__(ZShape<T, W, TX>::NT, kInterpFusedCtas<T>)
    interp_zwin_fused_kernel(const ZInterpJob<T>* jobs, const i64* item_end, int njobs,
                             i64 total, u32* queue) {
  __shared__ ZInterpShared<T, W, TX> sh;
  __shared__ ZInterpJob<T> job;
  u32 local;
  while (next_fused_item(jobs, item_end, njobs, total, queue, job, local)) {
    interp_zwin_item<T, W, TX>(job.a, job.ch, job.wl, local, sh);
    __syncthreads();  // the job record and the shared buffers are rewritten for the next item
  }
}

}  // namespace

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

// Launch units of a plane-major point set: (column, chunk) pairs.
UnitMap zwin_unit_map(const BinGeom& g, ZChunks ch) {
  UnitMap m{};
  m.kind = UnitMap::kZwin;
  m.ncols = i64(g.ntiles[0]) * g.ntiles[1];
  m.units = m.ncols * ch.count;
  m.nz = g.ntiles[2];
  m.zlen = ch.len;
  return m;
}

ZChunks zwin_chunks(const BinGeom& g) {
  return make_chunks(i64(g.ntiles[0]) * g.ntiles[1], g.ntiles[2], g.w);
}

// Work list of (column, chunk) units split into items of at most kWorkItemPoints points.
template <typename T>
WorkList zwin_work_list(const BinGeom& g, const SortedPoints<T>& pts, ZChunks ch,
                        cudaStream_t stream) {
  const WorkList wl = build_work_list(zwin_unit_map(g, ch), g, pts.bin_start, pts.M, pts.work,
                                      stream);
  if (wl.grid > 0x7fffffffll) throw_input("grid too large");
  return wl;
}
template WorkList zwin_work_list<float>(const BinGeom&, const SortedPoints<float>&, ZChunks,
                                         cudaStream_t);
template WorkList zwin_work_list<double>(const BinGeom&, const SortedPoints<double>&, ZChunks,
                                          cudaStream_t);

namespace {

template <typename T, int W, int TX, int TY>
void launch_spread_zwin_tw(const SpreadArgs<T>& a, cudaStream_t stream) {
  using S = ZShape<T, W, TX, TY>;
  const i64 ncols = i64(a.g.ntiles[0]) * a.g.ntiles[1];
  const ZChunks ch = make_chunks(ncols, a.g.ntiles[2], W);
  const WorkList wl = zwin_work_list(a.g, a.pts, ch, stream);
  // Single precision with the default or 4-row tiles spreads two strength vectors per pass
  // when there are several (the second vector costs its FMAs only).
  constexpr bool kPairs = std::is_same<T, float>::value && TX == 4 && (TY == 8 || TY == 4);
  if constexpr (kPairs) {
    if (a.batch > 1) {
      dim3 grid{unsigned(wl.grid), unsigned((a.batch + 1) / 2), 1u};
      spread_zwin2_kernel<T, W, TX, TY><<<grid, S::NT, 0, stream>>>(a, ch, wl);
      NNB_LAUNCH_CHECK();
      return;
    }
  }
  dim3 grid{unsigned(wl.grid), unsigned(a.batch), 1u};
  spread_zwin_kernel<T, W, TX, TY><<<grid, S::NT, 0, stream>>>(a, ch, wl);
  NNB_LAUNCH_CHECK();
}

template <typename T, int W, int TX, int TY>
void launch_interp_zwin_tw(const InterpArgs<T>& a, cudaStream_t stream) {
  using S = ZShape<T, W, TX, TY>;
  const i64 ncols = i64(a.g.ntiles[0]) * a.g.ntiles[1];
  const ZChunks ch = make_chunks(ncols, a.g.ntiles[2], W);
  const WorkList wl = zwin_work_list(a.g, a.pts, ch, stream);
  interp_zwin_kernel<T, W, TX, TY><<<unsigned(wl.grid), S::NT, 0, stream>>>(a, ch, wl);
  NNB_LAUNCH_CHECK();
}

template <typename T, int TX, int TY>
void spread_zwin_tx(const SpreadArgs<T>& a, cudaStream_t stream) {
  switch (a.g.w) {
    case 2: return launch_spread_zwin_tw<T, 2, TX, TY>(a, stream);
    case 3: return launch_spread_zwin_tw<T, 3, TX, TY>(a, stream);
    case 4: return launch_spread_zwin_tw<T, 4, TX, TY>(a, stream);
    case 5: return launch_spread_zwin_tw<T, 5, TX, TY>(a, stream);
    case 6: return launch_spread_zwin_tw<T, 6, TX, TY>(a, stream);
    case 7: return launch_spread_zwin_tw<T, 7, TX, TY>(a, stream);
    case 8: return launch_spread_zwin_tw<T, 8, TX, TY>(a, stream);
    default: throw_internal("z-window kernels need n_spread <= 8");
  }
}

template <typename T, int TX, int TY>
void interp_zwin_tx(const InterpArgs<T>& a, cudaStream_t stream) {
  switch (a.g.w) {
    case 2: return launch_interp_zwin_tw<T, 2, TX, TY>(a, stream);
    case 3: return launch_interp_zwin_tw<T, 3, TX, TY>(a, stream);
    case 4: return launch_interp_zwin_tw<T, 4, TX, TY>(a, stream);
    case 5: return launch_interp_zwin_tw<T, 5, TX, TY>(a, stream);
    case 6: return launch_interp_zwin_tw<T, 6, TX, TY>(a, stream);
    case 7: return launch_interp_zwin_tw<T, 7, TX, TY>(a, stream);
    case 8: return launch_interp_zwin_tw<T, 8, TX, TY>(a, stream);
    default: throw_internal("z-window kernels need n_spread <= 8");
  }
}

void check_zwin_geom(const BinGeom& g) {
  if (g.dim != 3 || !g.zmajor || (g.tile[1] != 4 && g.tile[1] != 8 && g.tile[1] != 16) ||
      g.tile[2] != 1 ||
      (g.tile[0] != 2 && g.tile[0] != 4 && g.tile[0] != 8) || g.w > 8) {
    throw_internal("z-window kernels need a 3D plane-major (2|4|8, 4|8|16, 1) tiling and n_spread <= 8");
  }
}


// Persistent launches: as many CTAs as fit on the GPU at once, or fewer when there are fewer
// items; each takes items from the shared queue until it is empty.
template <typename K>
unsigned persistent_grid(K kernel, int threads, i64 total) {
  int dev = 0, sms = 0, per_sm = 0;
  NNB_CUDA(cudaGetDevice(&dev));
  NNB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  NNB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0));
  i64 g = i64(sms) * (per_sm > 0 ? per_sm : 1);
  if (g > total) g = total;
  return unsigned(g < 1 ? 1 : g);
}

template <typename T, int W, int TX>
void spread_fused_tw(const ZSpreadJob<T>* jobs, const i64* item_end, int njobs, i64 total,
                     u32* queue, cudaStream_t stream) {
  constexpr int NT = ZShape<T, W, TX>::NT;
  const unsigned grid = persistent_grid(spread_zwin_fused_kernel<T, W, TX>, NT, total);
  spread_zwin_fused_kernel<T, W, TX><<<grid, NT, 0, stream>>>(jobs, item_end, njobs, total,
                                                              queue);
  NNB_LAUNCH_CHECK();
}

template <typename T, int W, int TX>
void interp_fused_tw(const ZInterpJob<T>* jobs, const i64* item_end, int njobs, i64 total,
                     u32* queue, cudaStream_t stream) {
  constexpr int NT = ZShape<T, W, TX>::NT;
  const unsigned grid = persistent_grid(interp_zwin_fused_kernel<T, W, TX>, NT, total);
  interp_zwin_fused_kernel<T, W, TX><<<grid, NT, 0, stream>>>(jobs, item_end, njobs, total,
                                                              queue);
  NNB_LAUNCH_CHECK();
}

// Calls f(std::integral_constant<int, w>) for 2 <= w <= 8.
template <typename F>
void with_width(int w, F&& f) {
  switch (w) {
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 5: return f(std::integral_constant<int, 5>{});
    case 6: return f(std::integral_constant<int, 6>{});
    case 7: return f(std::integral_constant<int, 7>{});
    case 8: return f(std::integral_constant<int, 8>{});
    default: throw_internal("z-window kernels need n_spread <= 8");
  }
}

void check_fused(int njobs, i64 total, int tile_x) {
  if (njobs < 1) throw_internal("a persistent launch needs at least one job");
  if (total < 1 || total > 0x7fffffffll) throw_internal("persistent launch item count out of range");
  if (tile_x != 2 && tile_x != 4 && tile_x != 8) {
    throw_internal("z-window kernels need tiles of 2, 4 or 8 in x");
  }
}
}  // namespace

template <int W>
void launch_spread_zmma_w(const SpreadArgs<float>& a, cudaStream_t stream) {
  const i64 ncols = i64(a.g.ntiles[0]) * a.g.ntiles[1];
  const ZChunks ch = make_chunks(ncols, a.g.ntiles[2], W);
  const WorkList wl = zwin_work_list(a.g, a.pts, ch, stream);
  dim3 grid{unsigned(wl.grid), unsigned(a.batch), 1u};
  spread_zmma_kernel<W><<<grid, 128, 0, stream>>>(a, ch, wl);
  NNB_LAUNCH_CHECK();
}

template <typename T>
void launch_spread_zwin(const SpreadArgs<T>& a, cudaStream_t stream) {
  check_zwin_geom(a.g);
  if (a.batch > 65535) throw_input("batch size above 65535");
  if (a.method == 4) {
    if constexpr (std::is_same<T, float>::value) {
      if (a.g.tile[0] != 8) throw_internal("tensor-core spreading needs tiles of 8 cells in x");
      switch (a.g.w) {
        case 5: return launch_spread_zmma_w<5>(a, stream);
        case 6: return launch_spread_zmma_w<6>(a, stream);
        case 7: return launch_spread_zmma_w<7>(a, stream);
        case 8: return launch_spread_zmma_w<8>(a, stream);
        default: throw_internal("tensor-core spreading needs 5 <= n_spread <= 8");
      }
    }
    throw_internal("tensor-core spreading is single precision");
  }
  if (a.g.tile[1] == 16) {
    if constexpr (std::is_same<T, float>::value) {
      if (a.g.tile[0] == 8) return spread_zwin_tx<T, 8, 16>(a, stream);
      if (a.g.tile[0] == 2) return spread_zwin_tx<T, 2, 16>(a, stream);
      return spread_zwin_tx<T, 4, 16>(a, stream);
    }
    throw_internal("z-window tiles of 16 rows are single precision");
  }
  if (a.g.tile[1] == 4) {
    if constexpr (std::is_same<T, float>::value) {
      if (a.g.tile[0] == 4) return spread_zwin_tx<T, 4, 4>(a, stream);
    }
    throw_internal("z-window tiles of 4 rows are single precision, 4 cells in x");
  }
  if (a.g.tile[0] == 8) return spread_zwin_tx<T, 8, 8>(a, stream);
  if (a.g.tile[0] == 2) return spread_zwin_tx<T, 2, 8>(a, stream);
  return spread_zwin_tx<T, 4, 8>(a, stream);
}

template <typename T>
void launch_interp_zwin(const InterpArgs<T>& a, cudaStream_t stream) {
  check_zwin_geom(a.g);
  if (a.g.tile[1] == 16) {
    if constexpr (std::is_same<T, float>::value) {
      if (a.g.tile[0] == 8) return interp_zwin_tx<T, 8, 16>(a, stream);
      if (a.g.tile[0] == 2) return interp_zwin_tx<T, 2, 16>(a, stream);
      return interp_zwin_tx<T, 4, 16>(a, stream);
    }
    throw_internal("z-window tiles of 16 rows are single precision");
  }
  if (a.g.tile[1] == 4) {
    if constexpr (std::is_same<T, float>::value) {
      if (a.g.tile[0] == 4) return interp_zwin_tx<T, 4, 4>(a, stream);
    }
    throw_internal("z-window tiles of 4 rows are single precision, 4 cells in x");
  }
  if (a.g.tile[0] == 8) return interp_zwin_tx<T, 8, 8>(a, stream);
  if (a.g.tile[0] == 2) return interp_zwin_tx<T, 2, 8>(a, stream);
  return interp_zwin_tx<T, 4, 8>(a, stream);
}

template <typename T>
ZSpreadJob<T> zwin_spread_job(const SpreadArgs<T>& a) {
  check_zwin_geom(a.g);
  if (a.g.tile[1] != 8) throw_internal("persistent z-window kernels use tiles of 8 rows");
  if (a.method != 3 || a.batch != 1) throw_internal("persistent spreading is method 3, batch 1");
  ZSpreadJob<T> j;
  j.a = a;
  j.ch = zwin_chunks(a.g);
  j.wl = describe_work_list(zwin_unit_map(a.g, j.ch), a.pts.M, a.pts.work);
  return j;
}

template <typename T>
ZInterpJob<T> zwin_interp_job(const InterpArgs<T>& a) {
  check_zwin_geom(a.g);
  if (a.g.tile[1] != 8) throw_internal("persistent z-window kernels use tiles of 8 rows");
  if (a.method != 3) throw_internal("persistent interpolation is method 3");
  ZInterpJob<T> j;
  j.a = a;
  j.ch = zwin_chunks(a.g);
  j.wl = describe_work_list(zwin_unit_map(a.g, j.ch), a.pts.M, a.pts.work);
  return j;
}

template <typename T>
void zwin_build_work_list(const BinGeom& g, const SortedPoints<T>& pts, cudaStream_t stream) {
  check_zwin_geom(g);
  (void)zwin_work_list(g, pts, zwin_chunks(g), stream);
}

template <typename T>
void launch_spread_zwin_fused(const ZSpreadJob<T>* jobs, const i64* item_end, int njobs,
                              i64 total, int w, int tile_x, u32* queue, cudaStream_t stream) {
  check_fused(njobs, total, tile_x);
  with_width(w, [&](auto wc) {
    constexpr int W = decltype(wc)::value;
    if (tile_x == 8) {
      spread_fused_tw<T, W, 8>(jobs, item_end, njobs, total, queue, stream);
    } else if (tile_x == 2) {
      spread_fused_tw<T, W, 2>(jobs, item_end, njobs, total, queue, stream);
    } else {
      spread_fused_tw<T, W, 4>(jobs, item_end, njobs, total, queue, stream);
    }
  });
}

template <typename T>
void launch_interp_zwin_fused(const ZInterpJob<T>* jobs, const i64* item_end, int njobs,
                              i64 total, int w, int tile_x, u32* queue, cudaStream_t stream) {
  check_fused(njobs, total, tile_x);
  with_width(w, [&](auto wc) {
    constexpr int W = decltype(wc)::value;
    if (tile_x == 8) {
      interp_fused_tw<T, W, 8>(jobs, item_end, njobs, total, queue, stream);
    } else if (tile_x == 2) {
      interp_fused_tw<T, W, 2>(jobs, item_end, njobs, total, queue, stream);
    } else {
      interp_fused_tw<T, W, 4>(jobs, item_end, njobs, total, queue, stream);
    }
  });
}

template ZSpreadJob<float> zwin_spread_job<float>(const SpreadArgs<float>&);
template ZSpreadJob<double> zwin_spread_job<double>(const SpreadArgs<double>&);
template ZInterpJob<float> zwin_interp_job<float>(const InterpArgs<float>&);
template ZInterpJob<double> zwin_interp_job<double>(const InterpArgs<double>&);
template void zwin_build_work_list<float>(const BinGeom&, const SortedPoints<float>&,
                                          cudaStream_t);
template void zwin_build_work_list<double>(const BinGeom&, const SortedPoints<double>&,
                                           cudaStream_t);
template void launch_spread_zwin_fused<float>(const ZSpreadJob<float>*, const i64*, int, i64,
                                              int, int, u32*, cudaStream_t);
template void launch_spread_zwin_fused<double>(const ZSpreadJob<double>*, const i64*, int, i64,
                                               int, int, u32*, cudaStream_t);
template void launch_interp_zwin_fused<float>(const ZInterpJob<float>*, const i64*, int, i64,
                                              int, int, u32*, cudaStream_t);
template void launch_interp_zwin_fused<double>(const ZInterpJob<double>*, const i64*, int, i64,
                                               int, int, u32*, cudaStream_t);
template void launch_spread_zwin<float>(const SpreadArgs<float>&, cudaStream_t);
template void launch_spread_zwin<double>(const SpreadArgs<double>&, cudaStream_t);
template void launch_interp_zwin<float>(const InterpArgs<float>&, cudaStream_t);
template void launch_interp_zwin<double>(const InterpArgs<double>&, cudaStream_t);

}  // namespace nnb
