// 3D single-precision ES spreading on the 5th-generation tensor cores (tcgen05, sm_100a):
// spreading method 5.
//
// Replaces, for 3D single-precision plans with kernel width w <= 8, the reference's spreading
// (src/neonufft/gpu/kernels/spreading_kernel.cu:477-715: one global float atomic per cell and
// point). Points are binned as for the z-window kernels (zwin.cu) with tiles of 4 x 4 cells in
// (x, y) and single planes in z, bins of one (x, y) column consecutive in plane order, so the
// points of a column and range of planes are one contiguous run of records sorted by their
// first plane. One CTA (4 warps) spreads one work item: a run of a column's points.
//
// The contribution of a group of K = 8 points to the column's region is one matrix product:
//   D[m, n] += sum_k A[m, k] B[n, k],   A[m, k] = kx_k(x) ky_k(y),   B[n, k] = c_k kz_k(plane(n)),
// with m = x + P0 y over the P0 x P1 <= 121 cells of the region (P0 = P1 = 4 + w - 1; rows 121 to
// 127 are zero) and n over the planes of the window times (re, im). D lives in tensor memory
// (TMEM), 128 lanes by 48 fp32 columns: a ring of three blocks of 8 consecutive planes, block b
// at columns 16 (b mod 3) .. + 16, plane 8 b + q, part r at column 16 (b mod 3) + 2 q + r. A
// point whose first plane is z touches planes z .. z + w - 1, so blocks z / 8 and z / 8 + 1; a
// batch of points whose first planes lie in two consecutive blocks fits the three-block ring.
// When a batch starts in a later block, the blocks before it are complete: each thread loads its
// lane's 16 columns of the block (tcgen05.ld), adds them to the fine grid with float2 atomics
// (neighbouring columns and chunks overlap by the halo) and zeroes them (tcgen05.st).
//
// Precision: the operands are split into a TF32 value and its remainder, a = a_hi + a_lo
// (a_hi = cvt.rna.tf32(a)), and each group takes three MMAs, A_hi B_hi + A_hi B_lo + A_lo B_hi,
// with fp32 accumulation in TMEM; the dropped A_lo B_lo term is below 2^-22 of each product.
//
// Per batch of 32 points: stage the points' kernel values in shared memory (the ES kernel is
// evaluated 3 w times per point, as in zwin.cu), build A (128 x 8 per group, K-major, no
// swizzle: 8-row x 16-byte core matrices) and B (48 x 8 per group, same layout) for the hi and
// lo parts, fence the generic-proxy stores for the async proxy, synchronise, and let one thread
// issue the MMAs and commit them to an mbarrier that every thread waits on (a bounded wait:
// after 2 s the CTA records a failure in g_tc_status, waits once more with a bound, frees its
// TMEM and returns; nnb_check_device_status reports it).
//
// A K-major operand without swizzle is described by its shared-memory start address, the byte
// distance between its two 16-byte K chunks (leading byte offset) and between consecutive groups
// of 8 rows (stride byte offset); the instruction descriptor gives the D / A / B formats
// (F32 / TF32 / TF32), both operands K-major, N / 8 and M / 16 (the bit layout of the sm_100
// UMMA descriptors as published in CUTLASS's cute/arch/mma_sm100_desc.hpp).
#include <cstdint>

#include "common.cuh"
#include "kernels.cuh"

namespace nnb {

namespace {

constexpr int kTcThreads = 128;             // 4 warps; thread m owns TMEM lane m (region cell m)
constexpr int kTcBatch = 32;                // points staged at a time
constexpr int kTcGroups = kTcBatch / 8;     // MMA groups of K = 8 points
constexpr int kTcRingBlocks = 3;            // 8-plane blocks held in TMEM
constexpr int kTcRingCols = 16 * kTcRingBlocks;  // 48 fp32 columns in use
constexpr u32 kTcAllocCols = 64;            // TMEM allocation (a power of two >= 32)
constexpr int kTcTile = 4;                  // tile of 4 x 4 cells in (x, y), one plane in z
constexpr int kTcRowPad = 36;               // row stride of the transposed kx / ky arrays
constexpr unsigned long long kTcWaitNs = 2000000000ull;  // bound of every wait (2 s)

__device__ int g_tc_status;  // nonzero once a bounded wait gave up (read by the host)

template <int W>
struct TcShape {
  static constexpr int P0 = kTcTile + W - 1;  // region extent in x and in y
  static constexpr int CELLS = P0 * P0;       // region cells = used accumulator rows
  static constexpr int KW = 12;               // staged kx / ky values per point (>= P0)
  static_assert(CELLS <= 128 && P0 <= KW, "region larger than the 128-row accumulator");
};

// Shared memory of one CTA (dynamic, 16-byte aligned). The operand tiles are in the canonical
// K-major layout without swizzle: element (row r, k) of a tile with R rows sits at float
// (k / 4) * 4 R + 4 r + (k % 4) -- core matrices of 8 rows x 16 bytes, 8-row groups 128 bytes
// apart, the two 16-byte K chunks 16 R bytes apart.
// One staged batch: kx / ky of the points over the region's x / y range, transposed (row =
// cell, column = point; zero outside the footprint and for unstaged points; rows padded to 36
// floats so that the 11 rows a warp reads at once fall in different banks), the B values
// c kz(t) (real and imaginary parts at rows 2 t, 2 t + 1, zero beyond w) split into TF32 value
// and remainder, and the points' first planes.
template <int W>
struct TcStage {
  float kxT[TcShape<W>::KW][kTcRowPad];
  float kyT[TcShape<W>::KW][kTcRowPad];
  float bv_hi[16][kTcBatch];
  float bv_lo[16][kTcBatch];
  int z[kTcBatch];
};

template <int W>
struct TcShared {
  float a_hi[kTcGroups][2 * 128 * 4];
  float a_lo[kTcGroups][2 * 128 * 4];
  float b_hi[kTcGroups][2 * kTcRingCols * 4];
  float b_lo[kTcGroups][2 * kTcRingCols * 4];
  PointRec<float> rec[3][kTcBatch];  // records of three consecutive batches (cp.async ring)
  float2 vin[2][kTcBatch];           // strengths of two consecutive batches (cp.async gather)
  TcStage<W> st;                     // the staged batch
  unsigned long long mbar;           // MMA completion barrier
  u32 tmem_base;                     // TMEM address written by tcgen05.alloc
};

// ---- PTX wrappers ----------------------------------------------------------------------------
__device__ __forceinline__ u32 smem_addr(const void* p) {
  return u32(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Shared-memory matrix descriptor of a K-major operand without swizzle.
__device__ __forceinline__ unsigned long long tc_desc(const float* base, u32 kchunk_bytes,
                                                      u32 group_bytes) {
  const unsigned long long a = smem_addr(base);
  unsigned long long d = (a >> 4) & 0x3FFFull;                   // start address / 16
  d |= (unsigned long long)((kchunk_bytes >> 4) & 0x3FFFu) << 16;  // leading byte offset / 16
  d |= (unsigned long long)((group_bytes >> 4) & 0x3FFFu) << 32;   // stride byte offset / 16
  d |= 1ull << 46;                                               // descriptor version (sm_100)
  return d;  // base offset 0, absolute leading-offset mode, layout "no swizzle" (0)
}

// Instruction descriptor: D fp32, A and B TF32, both K-major, shape M x N (x 8).
__host__ __device__ constexpr u32 tc_idesc(int m, int n) {
  return (1u << 4) | (2u << 7) | (2u << 10) | (u32(n >> 3) << 17) | (u32(m >> 4) << 24);
}

// D (+)= A B^T; accumulate = 0 overwrites D.
__device__ __forceinline__ void tc_mma(u32 d_tmem, unsigned long long a_desc,
                                       unsigned long long b_desc, u32 idesc, u32 accumulate) {
  const u32 zero = 0;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "setp.ne.b32 p, %5, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%4, %4, %4, %4}, p;\n\t"
      "}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(zero), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_commit(unsigned long long* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(mbar))
               : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_smem_for_async_proxy() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_init(unsigned long long* m) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(m)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* m, u32 parity) {
  u32 ok;
  asm volatile(
      "{\n\t"
      ".reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t"
      "}\n"
      : "=r"(ok)
      : "r"(smem_addr(m)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the phase of the given parity to complete, at most kTcWaitNs.
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* m, u32 parity) {
  const unsigned long long t0 = global_ns();
  for (u32 it = 0;; ++it) {
    if (mbar_try_wait(m, parity)) return true;
    if ((it & 63u) == 63u && global_ns() - t0 > kTcWaitNs) return false;
  }
}

// 16 consecutive fp32 columns of this warp's 32 lanes (thread = lane).
__device__ __forceinline__ void tmem_load16(u32 addr, float (&v)[16]) {
  u32 r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_zero16(u32 addr) {
  const u32 z = 0;
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1, %1, %1, %1, "
      "%1, %1, %1, %1, %1};" ::"r"(addr),
      "r"(z)
      : "memory");
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ float to_tf32(float a) {
  u32 r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(a));
  return __uint_as_float(r);
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(smem)), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(smem)), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// ---- the kernel ------------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(kTcThreads)
    spread_tc_kernel(const __grid_constant__ SpreadArgs<float> a, ZChunks ch,
                     const __grid_constant__ WorkList wl) {
  using S = TcShape<W>;
  extern __shared__ __align__(16) unsigned char tc_smem_raw[];
  TcShared<W>& sh = *reinterpret_cast<TcShared<W>*>(tc_smem_raw);

  // work item: column (tx, ty), its run of points [pbeg, pend)
  const BinGeom& g = a.g;
  u32 unit, slice;
  if (!work_item_at(wl, blockIdx.x, unit, slice)) return;
  const i64 ncols = i64(g.ntiles[0]) * g.ntiles[1];
  const int chunk = int(unit / ncols);
  const i64 col = unit - i64(chunk) * ncols;
  const int tx = int(col % g.ntiles[0]);
  const int ty = int(col / g.ntiles[0]);
  const int nz = g.ntiles[2];
  const int cz0 = chunk * ch.len;
  const int cz1 = min(cz0 + ch.len, nz);
  const u32* bs = a.pts.bin_start + col * nz;
  u32 pbeg, pend;
  work_slice(bs[cz0], bs[cz1], slice, wl.cap, pbeg, pend);
  if (pbeg >= pend) return;

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const int batch = blockIdx.y;
  const cplx_t<float>* in = a.in + batch * a.in_bdist;
  float2* grid = a.grid + batch * a.grid_bdist;
  const i64 nfx = g.nf[0], nfy = g.nf[1];
  const int nfz = int(g.nf[2]);
  [[maybe_unused]] const i64 cells = nfx * nfy * g.nf[2];
  const u32 npts = pend - pbeg;
  const int nbatches = int((npts + kTcBatch - 1) / kTcBatch);
  auto batch_size = [&](int bi) { return int(min(npts - u32(bi) * kTcBatch, u32(kTcBatch))); };

  // Warp 3 prefetches with cp.async: the records of a batch (into the ring of three) and its
  // strengths (gathered at the permutation in its records, into the ring of two).
  auto prefetch_rec = [&](int bi) {
    if (bi >= nbatches) return;
    const u32 p0 = u32(bi) * kTcBatch;
    if (lane < batch_size(bi) && NNB_CHECK_INDEX(i64(pbeg) + p0 + lane, a.pts.M)) {
      const PointRec<float>* src = a.pts.rec + pbeg + p0 + lane;
      PointRec<float>* dst = &sh.rec[bi % 3][lane];
      cp_async16(dst, src);
      cp_async16(reinterpret_cast<char*>(dst) + 16, reinterpret_cast<const char*>(src) + 16);
    }
  };
  auto prefetch_v = [&](int bi) {  // the lane reads the record it copied itself
    if (bi >= nbatches) return;
    if (lane < batch_size(bi)) {
      const u32 perm = sh.rec[bi % 3][lane].perm;
      if (NNB_CHECK_INDEX(perm, a.pts.M)) cp_async8(&sh.vin[bi % 2][lane], in + perm);
    }
  };
  // Warps 0 to 2 stage batch bi (its records and strengths have landed): warp 0 kx, warp 1 ky,
  // warp 2 kz, the first planes and the B values.
  auto stage = [&](int bi) {
    TcStage<W>& st = sh.st;
    const int n = batch_size(bi);
    if (warp < 2) {
      float (*dstT)[kTcRowPad] = warp == 0 ? st.kxT : st.kyT;
#pragma unroll
      for (int i = 0; i < S::KW; ++i) dstT[i][lane] = 0.f;
      if (lane < n) {
        const PointRec<float>& rec = sh.rec[bi % 3][lane];
        const int l0 = warp == 0 ? int(rec.local & 0xFu) : int((rec.local >> 4) & 0xFu);
        const float f = rec.frac[warp];
#pragma unroll
        for (int t = 0; t < W; ++t) {
          dstT[l0 + t][lane] = es_eval_fast<float>(f + float(t), a.beta, a.c);
        }
      }
    } else if (warp == 2 && lane < n) {
      const PointRec<float>& rec = sh.rec[bi % 3][lane];
      st.z[lane] = int(rec.local >> 8);
      float2 v = sh.vin[bi % 2][lane];
      if (a.prephase && NNB_CHECK_INDEX(rec.perm, a.pts.M)) v = cmul(v, a.prephase[rec.perm]);
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        const float k = t < W ? es_eval_fast<float>(rec.frac[2] + float(t), a.beta, a.c) : 0.f;
        const float re = v.x * k, im = v.y * k;
        const float re_hi = to_tf32(re), im_hi = to_tf32(im);
        st.bv_hi[2 * t][lane] = re_hi;
        st.bv_hi[2 * t + 1][lane] = im_hi;
        st.bv_lo[2 * t][lane] = re - re_hi;
        st.bv_lo[2 * t + 1][lane] = im - im_hi;
      }
    }
  };

  // TMEM: 64 columns for this CTA (warp 0 allocates), the barrier for MMA completion
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&sh.tmem_base)),
                 "r"(kTcAllocCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) mbar_init(&sh.mbar);
  if (warp == 3) {  // records of batches 0 and 1, then the strengths of batch 0
    prefetch_rec(0);
    prefetch_rec(1);
    cp_async_commit();
    cp_async_wait_all();
    prefetch_v(0);
    cp_async_commit();
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const u32 tmem = sh.tmem_base;
  const u32 lane_addr = tmem + (u32(32 * warp) << 16);  // this warp's 32 lanes
#pragma unroll
  for (int s = 0; s < kTcRingBlocks; ++s) tmem_zero16(lane_addr + u32(16 * s));

  // This thread's region cell (accumulator row m = tid). Rows beyond the region read the
  // always-zero ky rows at or past P0, so their A rows are zero without a test.
  const bool has_cell = tid < S::CELLS;
  const int cx = tid % S::P0;
  const int cy = min(tid / S::P0, S::KW - 1);
  const i64 gx = has_cell ? (i64(tx) * kTcTile + cx) % nfx : 0;
  const i64 gy = has_cell ? (i64(ty) * kTcTile + cy) % nfy : 0;
  const i64 row_base = gy * nfx + gx;
  const i64 plane_stride = nfx * nfy;

  // The lane's running sums of the window's three blocks (acc[i]: block wb + i, 8 planes x
  // (re, im)), in fp32 registers. The tensor-memory accumulator is drained into them after
  // every sub-batch, so that no accumulation chain inside the tensor core runs longer than one
  // sub-batch (longer chains lose precision: with 4 sub-batches per drain, 2.3e-6 relative
  // against the z-window kernel on ~9000 points clustered in one column); tensor-memory
  // columns 16 s .. + 16 hold block wb + s of the current sub-batch and are zeroed when drained.
  float acc[kTcRingBlocks][16];
#pragma unroll
  for (int r = 0; r < kTcRingBlocks; ++r) {
#pragma unroll
    for (int i = 0; i < 16; ++i) acc[r][i] = 0.f;
  }
  // Adds acc[r] (block b) to the grid and clears it.
  auto flush = [&](int r, int b) {
#pragma unroll
    for (int rr = 0; rr < kTcRingBlocks; ++rr) {
      if (rr == r) {
        if (has_cell) {
          int p = 8 * b;
          while (p >= nfz) p -= nfz;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            if (acc[rr][2 * q] != 0.f || acc[rr][2 * q + 1] != 0.f) {
              const i64 idx = i64(p) * plane_stride + row_base;
              if (NNB_CHECK_INDEX(idx, cells)) {
                atomicAdd(&grid[idx], make_float2(acc[rr][2 * q], acc[rr][2 * q + 1]));
              }
            }
            if (++p == nfz) p = 0;
          }
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[rr][i] = 0.f;
      }
    }
  };

  constexpr u32 kAChunk = 128 * 16;         // bytes between the two K chunks of an A tile
  constexpr u32 kBChunk = kTcRingCols * 16;  // ... of a B tile
  int wb = -1;      // first block of the window (acc[0])
  u32 dirty = 0;    // blocks (bit b - wb) with contributions since their last flush
  u32 parity = 0;
  bool failed = false;
  const TcStage<W>& st = sh.st;
  for (int bi = 0; bi < nbatches && !failed; ++bi) {
    const int nstage = batch_size(bi);
    // ---- stage batch bi (warps 0 to 2) while warp 3 prefetches the next two --------------
    if (warp == 3) cp_async_wait_all();  // records of batch bi + 1, strengths of batch bi
    __syncthreads();
    if (warp == 3) {
      prefetch_v(bi + 1);
      prefetch_rec(bi + 2);
      cp_async_commit();
    } else {
      stage(bi);
    }
    __syncthreads();
    // ---- the staged points in sub-batches whose first planes lie in two consecutive blocks --
    for (int k0 = 0; k0 < nstage;) {
      const int b0 = st.z[k0] >> 3;
      const bool in_sub =
          lane >= k0 && lane < nstage && (st.z[lane < nstage ? lane : 0] >> 3) <= b0 + 1;
      const int nb = __popc(__ballot_sync(0xffffffffu, in_sub));  // sorted: a run from k0
      // move the window to start at block b0: flush the complete blocks, shift the rest
      if (wb < 0) {
        wb = b0;
      } else if (b0 > wb) {
        const int d = b0 - wb;
#pragma unroll
        for (int r = 0; r < kTcRingBlocks; ++r) {
          if (r < d && (dirty & (1u << r))) flush(r, wb + r);
        }
        if (d == 1) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            acc[0][i] = acc[1][i];
            acc[1][i] = acc[2][i];
            acc[2][i] = 0.f;
          }
        } else if (d == 2) {
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            acc[0][i] = acc[2][i];
            acc[1][i] = 0.f;
            acc[2][i] = 0.f;
          }
        }  // d >= 3: every block was flushed (and cleared)
        dirty = d < kTcRingBlocks ? dirty >> d : 0u;
        wb = b0;
      }
      // ---- operands: zero B; A = kx (x) ky (hi, lo) ----------------------------------------
#pragma unroll
      for (int i = tid; i < kTcGroups * 2 * kTcRingCols; i += kTcThreads) {
        reinterpret_cast<float4*>(&sh.b_hi[0][0])[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        reinterpret_cast<float4*>(&sh.b_lo[0][0])[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      if (k0 == 0 && nb == nstage) {
        // every staged point (columns past nstage are zero): 16-byte loads of 4 points
#pragma unroll
        for (int gi = 0; gi < kTcGroups; ++gi) {
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            const int k4 = 8 * gi + 4 * c;
            const float4 xv = *reinterpret_cast<const float4*>(&st.kxT[cx][k4]);
            const float4 yv = *reinterpret_cast<const float4*>(&st.kyT[cy][k4]);
            const float av[4] = {xv.x * yv.x, xv.y * yv.y, xv.z * yv.z, xv.w * yv.w};
            float hi[4], lo[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              hi[j] = to_tf32(av[j]);
              lo[j] = av[j] - hi[j];
            }
            *reinterpret_cast<float4*>(&sh.a_hi[gi][c * 512 + 4 * tid]) =
                make_float4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<float4*>(&sh.a_lo[gi][c * 512 + 4 * tid]) =
                make_float4(lo[0], lo[1], lo[2], lo[3]);
          }
        }
      } else {
#pragma unroll
        for (int gi = 0; gi < kTcGroups; ++gi) {
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            float hi[4], lo[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
              const int jj = 8 * gi + 4 * c + j;
              const float av = jj < nb ? st.kxT[cx][k0 + jj] * st.kyT[cy][k0 + jj] : 0.f;
              hi[j] = to_tf32(av);
              lo[j] = av - hi[j];
            }
            *reinterpret_cast<float4*>(&sh.a_hi[gi][c * 512 + 4 * tid]) =
                make_float4(hi[0], hi[1], hi[2], hi[3]);
            *reinterpret_cast<float4*>(&sh.a_lo[gi][c * 512 + 4 * tid]) =
                make_float4(lo[0], lo[1], lo[2], lo[3]);
          }
        }
      }
      __syncthreads();  // B is zero everywhere
      // ---- B: each point's 16 values at rows 2 (z - 8 b0) .. + 16 of its column ------------
      {
        const int jj = lane;  // column of the sub-batch; warp = a quarter of the 16 rows
        if (jj < nb) {
          const int k = k0 + jj;
          const int r0 = 2 * (st.z[k] - 8 * b0);
          const int gi = jj >> 3;
          const int c = (jj & 7) >> 2;
          const int j = jj & 3;
#pragma unroll
          for (int rr = 0; rr < 4; ++rr) {
            const int q = 4 * warp + rr;
            const int n = r0 + q;
            sh.b_hi[gi][c * 4 * kTcRingCols + 4 * n + j] = st.bv_hi[q][k];
            sh.b_lo[gi][c * 4 * kTcRingCols + 4 * n + j] = st.bv_lo[q][k];
          }
        }
      }
      fence_smem_for_async_proxy();
      fence_before_sync();
      __syncthreads();
      // ---- one thread issues the groups' MMAs over the blocks they touch -------------------
      if (tid == 0) {
        fence_after_sync();
        for (int gi = 0; gi * 8 < nb; ++gi) {
          const int last = k0 + min(nb, 8 * gi + 8) - 1;
          const int s0 = (st.z[k0 + 8 * gi] >> 3) - b0;
          const int s1 = ((st.z[last] + W - 1) >> 3) - b0 + 1;
          const u32 idesc = tc_idesc(128, 16 * (s1 - s0));
          const u32 d = tmem + u32(16 * s0);
          const unsigned long long ah = tc_desc(sh.a_hi[gi], kAChunk, 128);
          const unsigned long long al = tc_desc(sh.a_lo[gi], kAChunk, 128);
          const unsigned long long bh = tc_desc(sh.b_hi[gi] + 4 * 16 * s0, kBChunk, 128);
          const unsigned long long bl = tc_desc(sh.b_lo[gi] + 4 * 16 * s0, kBChunk, 128);
          tc_mma(d, ah, bh, idesc, 1u);
          tc_mma(d, ah, bl, idesc, 1u);
          tc_mma(d, al, bh, idesc, 1u);
        }
        tc_commit(&sh.mbar);
      }
      // ---- wait for the MMAs (they read the operand tiles the next sub-batch rewrites) -----
      const bool ok = mbar_wait_bounded(&sh.mbar, parity);
      parity ^= 1u;
      if (__syncthreads_or(!ok)) {
        failed = true;
        break;
      }
      fence_after_sync();
      // ---- drain: tensor-memory block wb + s into acc[s], zeroed for the next sub-batch ---
      const int ns = ((st.z[k0 + nb - 1] + W - 1) >> 3) - b0 + 1;
#pragma unroll
      for (int s = 0; s < kTcRingBlocks; ++s) {
        if (s < ns) {
          float v[16];
          const u32 addr = lane_addr + u32(16 * s);
          tmem_load16(addr, v);
#pragma unroll
          for (int i = 0; i < 16; ++i) acc[s][i] += v[i];
          tmem_zero16(addr);
          dirty |= 1u << s;
        }
      }
      k0 += nb;
    }
  }
  if (warp == 3) cp_async_wait_all();  // no copy outlives the CTA
  if (failed) {
    if (tid == 0) atomicExch(&g_tc_status, 1);
    (void)mbar_wait_bounded(&sh.mbar, parity ^ 1u);  // the MMAs in flight, once more, bounded
  } else if (wb >= 0) {
#pragma unroll
    for (int r = 0; r < kTcRingBlocks; ++r) {
      if (dirty & (1u << r)) flush(r, wb + r);
    }
  }
  fence_before_sync();
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTcAllocCols)
                 : "memory");
  }
}

template <int W>
void launch_spread_tc_w(const SpreadArgs<float>& a, cudaStream_t stream) {
  const i64 ncols = i64(a.g.ntiles[0]) * a.g.ntiles[1];
  const ZChunks ch = make_chunks(ncols, a.g.ntiles[2], W);
  const WorkList wl = zwin_work_list(a.g, a.pts, ch, stream);
  const size_t smem = sizeof(TcShared<W>);
  // the dynamic shared-memory limit is an attribute of the function on the current device; a
  // host-side call per launch, so any device the caller switches to is covered
  NNB_CUDA(cudaFuncSetAttribute(spread_tc_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(smem)));
  const dim3 grid{unsigned(wl.grid), unsigned(a.batch), 1u};
  spread_tc_kernel<W><<<grid, kTcThreads, smem, stream>>>(a, ch, wl);
  NNB_LAUNCH_CHECK();
}

}  // namespace

void launch_spread_tc(const SpreadArgs<float>& a, cudaStream_t stream) {
  const BinGeom& g = a.g;
  if (g.dim != 3 || !g.zmajor || g.tile[0] != kTcTile || g.tile[1] != kTcTile || g.tile[2] != 1) {
    throw_internal("tensor-core spreading needs a 3D plane-major 4 x 4 x 1 tiling");
  }
  if (a.batch > 65535) throw_input("batch size above 65535");
  switch (g.w) {
    case 2: return launch_spread_tc_w<2>(a, stream);
    case 3: return launch_spread_tc_w<3>(a, stream);
    case 4: return launch_spread_tc_w<4>(a, stream);
    case 5: return launch_spread_tc_w<5>(a, stream);
    case 6: return launch_spread_tc_w<6>(a, stream);
    case 7: return launch_spread_tc_w<7>(a, stream);
    case 8: return launch_spread_tc_w<8>(a, stream);
    default: throw_internal("tensor-core spreading needs n_spread <= 8");
  }
}

int read_tc_status(bool clear) {
  int s = 0;
  NNB_CUDA(cudaMemcpyFromSymbol(&s, g_tc_status, sizeof(s)));
  if (clear && s) {
    const int z = 0;
    NNB_CUDA(cudaMemcpyToSymbol(g_tc_status, &z, sizeof(z)));
  }
  return s;
}

}  // namespace nnb
