// Launchers of the engine's device kernels. Every launcher enqueues on `stream` and checks the
// launch status; none synchronises.
#pragma once

#include "common.cuh"

namespace nnb {

template <typename T>
struct CoordPtrs {
  const T* p[3];
};

// ---- binning (binning.cu) -------------------------------------------------------------------
// Pass 1: per point, tile index and rank within the tile (one int atomic per point).
template <typename T>
void launch_bin_count(const BinGeom& g, CoordPtrs<T> x, i64 M, u32* counts, u32* ranks,
                      int* err_flag, cudaStream_t stream);
// Exclusive scan of n counts into out[0..n] (out[n] = total). tmp needs scan_tmp_words(n).
i64 scan_tmp_words(i64 n);
void launch_exclusive_scan(const u32* counts, u32* out, i64 n, u32* tmp, cudaStream_t stream);
// Pass 2: one 32-byte record per point (permutation, packed cell, fractions) in tile order.
template <typename T>
void launch_perm_checksum(const PointRec<T>* rec, i64 M, unsigned long long* sums,
                          cudaStream_t stream);
template <typename T>
void launch_bin_scatter(const BinGeom& g, CoordPtrs<T> x, i64 M, const u32* ranks,
                        const u32* bin_start, PointRec<T>* rec, cudaStream_t stream);

// ---- work lists (worklist.cu) ---------------------------------------------------------------
// Launch units (one CTA each) split into items of at most kWorkItemPoints points.
constexpr u32 kWorkItemPoints = 4096;
struct UnitMap {
  enum { kZwin = 0, kSlab = 1, kTile = 2 };
  int kind;
  i64 units;
  i64 ncols;   // kZwin: columns; unit = chunk * ncols + column
  int nz;      // kZwin: planes
  int zlen;    // kZwin: planes per chunk
  int nw;      // kSlab: tiles per unit along the last dimension
  i64 groups;  // kSlab: units per row of tiles along the last dimension
};
struct WorkList {
  const u32* owner;  // unit of each item
  const u32* start;  // first item of each unit (units + 1)
  i64 units;
  u32 cap;           // points per item
  i64 grid;          // CTAs to launch (an upper bound on the number of items)
};
WorkList build_work_list(const UnitMap& m, const BinGeom& g, const u32* bin_start, i64 M,
                         const WorkScratch& s, cudaStream_t stream);
// The WorkList that build_work_list returns for the same arguments, without launching anything.
WorkList describe_work_list(const UnitMap& m, i64 M, const WorkScratch& s);
// Unit and slice of item i; false if i is past the list's items.
__device__ __forceinline__ bool work_item_at(const WorkList& wl, u32 i, u32& unit, u32& slice) {
  if (i >= wl.start[wl.units]) return false;
  unit = wl.owner[i];
  slice = i - wl.start[unit];
  return true;
}
// Unit and slice of the calling CTA's item (blockIdx.x); false if the CTA has no item.
__device__ __forceinline__ bool work_item(const WorkList& wl, u32& unit, u32& slice) {
  return work_item_at(wl, blockIdx.x, unit, slice);
}
// Points [begin, end) of slice `slice` of a bin's range [b0, b1).
__device__ __forceinline__ void work_slice(u32 b0, u32 b1, u32 slice, u32 cap, u32& begin,
                                           u32& end) {
  const u64 s = u64(b0) + u64(slice) * cap;
  begin = s < b1 ? u32(s) : b1;
  end = (u64(begin) + cap) < b1 ? begin + cap : b1;
}

// ---- spreading (spread.cu) ------------------------------------------------------------------
template <typename T>
struct SpreadArgs {
  BinGeom g;
  SortedPoints<T> pts;
  const cplx_t<T>* in;        // strengths, original point order (batch b at in + b * in_bdist)
  const cplx_t<T>* prephase;  // optional per-point factor, original order
  cplx_t<T>* grid;            // fine grid (batch b at grid + b * grid_bdist), accumulated into
  i64 in_bdist;
  i64 grid_bdist;
  int batch;
  T beta;
  T c;
  int method;  // 1: warp-private slabs, 2: thread per point, 3: z-window, 4: z-window on tensor cores (zwin.cu)
};
template <typename T>
void launch_spread(const SpreadArgs<T>& a, cudaStream_t stream);
template <typename T>
void launch_spread_zwin(const SpreadArgs<T>& a, cudaStream_t stream);
// Method 5: 3D single-precision spreading on the tcgen05 tensor cores (spread_tc.cu).
void launch_spread_tc(const SpreadArgs<float>& a, cudaStream_t stream);
// Status word of the tensor-core spreading: nonzero once one of its bounded waits gave up
// (synchronous read; clear resets it).
int read_tc_status(bool clear);
// Dynamic shared memory of the default spreading / interpolation kernels for a tile shape.
size_t spread_smem_bytes(int dim, int w, const int* tile, size_t complex_bytes, int warps);
size_t interp_smem_bytes(int dim, int w, const int* tile, size_t complex_bytes, int warps);

// ---- interpolation (interp.cu) --------------------------------------------------------------
template <typename T>
struct InterpArgs {
  BinGeom g;
  SortedPoints<T> pts;
  const cplx_t<T>* grid;       // fine grid
  const cplx_t<T>* postphase;  // optional per-point factor, original order
  cplx_t<T>* out;              // original point order
  T beta;
  T c;
  int method;  // 1: warp per point, 2: thread per point, 3: z-window (zwin.cu)
};
template <typename T>
void launch_interp(const InterpArgs<T>& a, cudaStream_t stream);
template <typename T>
void launch_interp_zwin(const InterpArgs<T>& a, cudaStream_t stream);

// ---- z-window kernels over many transforms (zwin.cu) --------------------------------------------
// Plane chunks of the z-window kernels: each (x, y) column is cut into `count` chunks of `len`
// planes, one launch unit each.
struct ZChunks {
  int len;    // planes per chunk
  int count;  // chunks per column
};
// Chunks of `len` planes for ncols columns of nz planes (at least 4 w planes each), and the work
// list of a plane-major point set's (column, chunk) units (zwin.cu; also used by the
// tensor-core spreading, spread_tc.cu).
ZChunks make_chunks(i64 ncols, int nz, int w);
template <typename T>
WorkList zwin_work_list(const BinGeom& g, const SortedPoints<T>& pts, ZChunks ch,
                        cudaStream_t stream);
// One transform's share of a persistent launch: its arguments, chunks and work list.
template <typename T>
struct ZSpreadJob {
  SpreadArgs<T> a;
  ZChunks ch;
  WorkList wl;
};
template <typename T>
struct ZInterpJob {
  InterpArgs<T> a;
  ZChunks ch;
  WorkList wl;
};
// Host-side descriptions (nothing is launched); the work lists they name are built on the
// device by zwin_build_work_list, which must run before the persistent launch.
template <typename T>
ZSpreadJob<T> zwin_spread_job(const SpreadArgs<T>& a);
template <typename T>
ZInterpJob<T> zwin_interp_job(const InterpArgs<T>& a);
template <typename T>
void zwin_build_work_list(const BinGeom& g, const SortedPoints<T>& pts, cudaStream_t stream);
// One persistent launch over the items of njobs transforms that share (T, w, tile x): CTAs take
// items from the counter *queue (zero at launch) until all `total` items are taken; item_end
// holds the jobs' cumulative item counts. Jobs, item_end and queue are device memory.
template <typename T>
void launch_spread_zwin_fused(const ZSpreadJob<T>* jobs, const i64* item_end, int njobs,
                              i64 total, int w, int tile_x, u32* queue, cudaStream_t stream);
template <typename T>
void launch_interp_zwin_fused(const ZInterpJob<T>* jobs, const i64* item_end, int njobs,
                              i64 total, int w, int tile_x, u32* queue, cudaStream_t stream);

// ---- deconvolution (deconv.cu) --------------------------------------------------------------
template <typename T>
struct DeconvArgs {
  int dim;
  int order;        // NeonufftModeOrder
  i64 nf[3];        // fine grid
  i64 modes[3];     // mode box
  i64 stride[3];    // strides (elements) of the user mode array
  const T* corr[3]; // 1 / phi_hat per dim, nf/2 + 1 values
};
// Type 1: out(modes, strided) = fine(k mod nf) * prod corr.
template <typename T>
void launch_downsample(const DeconvArgs<T>& a, const cplx_t<T>* fine, cplx_t<T>* out,
                       cudaStream_t stream);
// Type 2 / type 3 stage 2: fine = zero-padded modes * prod corr (writes every fine cell).
template <typename T>
void launch_upsample(const DeconvArgs<T>& a, const cplx_t<T>* in, cplx_t<T>* fine,
                     cudaStream_t stream);

// ---- type 3 (t3.cu) -------------------------------------------------------------------------
// min / max of each coordinate array into out[2d] (min), out[2d+1] (max), as double.
template <typename T>
void launch_min_max(int dim, CoordPtrs<T> x, i64 M, unsigned long long* enc_out,
                    cudaStream_t stream);
void decode_min_max(const unsigned long long* enc, int n, double* out);
void init_min_max(unsigned long long* enc_host, int n);

template <typename T>
void launch_prephase(int dim, int sign, CoordPtrs<T> x, i64 M, const double* out_offset,
                     cplx_t<T>* pre, cudaStream_t stream);

struct PostphaseQuad {
  int n;
  double z[32];
  double kv[32];
};
template <typename T>
void launch_postphase(int dim, int sign, CoordPtrs<T> s, i64 K, const double* out_offset,
                      const double* in_offset, const double* scale, const PostphaseQuad& q,
                      cplx_t<T>* post, cudaStream_t stream);

// ---- MLP of the learned cost model (mlp.cu) --------------------------------------------------
i64 mlp_param_count(int L, const int* widths);
void mlp_forward(int L, const int* widths, const float* params, const float* x, i64 batch,
                 float* acts, cudaStream_t stream);
void mlp_backward(int L, const int* widths, const float* params, const float* x,
                  const float* acts, float* dacts, i64 batch, float* grads, cudaStream_t stream);
void mlp_mse(const float* y, const float* target, i64 n, float* dy, float* loss,
             cudaStream_t stream);
void mlp_adam(i64 n, float* params, const float* grads, float* m, float* v, float lr,
              float beta1, float beta2, float eps, i64 step, cudaStream_t stream);

// ---- FP64 direct sums (direct.cu) ------------------------------------------------------------
void launch_direct_type1(int dim, int sign, i64 M, const double* const* loc, const double* in,
                         i64 S, const i64* modes_idx, double* out, cudaStream_t stream);
void launch_direct_type2(int dim, int sign, const i64* n_modes, const double* in,
                         const double* const* loc, i64 S, const i64* point_idx, double* out,
                         cudaStream_t stream);
void launch_direct_type3(int dim, int sign, i64 M, const double* const* in_loc, const double* in,
                         const double* const* out_loc, i64 S, const i64* target_idx,
                         double* out, cudaStream_t stream);
// Same sums as launch_direct_type1 through a fixed device scratch array (direct_noalloc.cu).
void launch_direct_type1_noalloc(int dim, int sign, i64 M, const double* const* loc,
                                 const double* in, i64 S, const i64* modes_idx, double* out,
                                 cudaStream_t stream);

}  // namespace nnb
