// Host runtime pieces: allocator adapter, owning device arrays, cuFFT grid, stage timer,
// bin-sorted point sets. Used by the plan implementations (plan.cu).
#pragma once

#include <atomic>
#include <memory>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "common.cuh"
#include "kernels.cuh"
#include "neonufft_gpu.h"
#include "params.hpp"

namespace nnb {

// Number of engine kernels launched by this process (all plans, all devices).
extern std::atomic<i64> g_kernel_launches;

// Adapter over the user's NnbAllocator (or cudaMalloc / cudaFree when none is given).
class DeviceAllocator {
public:
  explicit DeviceAllocator(const NnbAllocator* a);
  void* allocate(size_t bytes);  // throws MemoryAllocError
  void deallocate(void* p, size_t bytes) noexcept;
  u64 in_use() const { return in_use_; }

private:
  NnbAllocator a_{};
  bool custom_ = false;
  u64 in_use_ = 0;
};

// Owning device array allocated through the plan's allocator.
template <typename X>
class DevArray {
public:
  DevArray() = default;
  explicit DevArray(std::shared_ptr<DeviceAllocator> alloc) : alloc_(std::move(alloc)) {}
  DevArray(const DevArray&) = delete;
  DevArray& operator=(const DevArray&) = delete;
  ~DevArray() { release(); }

  void set_allocator(std::shared_ptr<DeviceAllocator> alloc) { alloc_ = std::move(alloc); }

  // Ensures capacity for n elements (reallocates only when growing).
  void reserve(size_t n) {
    if (n <= cap_) {
      n_ = n;
      return;
    }
    release();
    if (n && !alloc_) throw_internal("device array without an allocator");
    if (n) ptr_ = static_cast<X*>(alloc_->allocate(n * sizeof(X)));
    cap_ = n;
    n_ = n;
  }
  void release() {
    if (ptr_) alloc_->deallocate(ptr_, cap_ * sizeof(X));
    ptr_ = nullptr;
    cap_ = n_ = 0;
  }
  X* data() const { return ptr_; }
  size_t size() const { return n_; }

private:
  std::shared_ptr<DeviceAllocator> alloc_;
  X* ptr_ = nullptr;
  size_t cap_ = 0;
  size_t n_ = 0;
};

// Records CUDA events around plan stages when enabled; sums elapsed times on request.
class StageTimer {
public:
  ~StageTimer();
  void enable(bool on) { enabled_ = on; }
  bool enabled() const { return enabled_; }
  void begin(cudaStream_t s, int stage);
  void end(cudaStream_t s, int stage);
  void collect(cudaStream_t s, double* ms, i64* count, bool reset);

private:
  cudaEvent_t get_event();
  struct Pending {
    int stage;
    cudaEvent_t a, b;
  };
  bool enabled_ = false;
  int open_stage_ = -1;
  cudaEvent_t open_event_ = nullptr;
  std::vector<Pending> pending_;
  std::vector<cudaEvent_t> pool_;
  double ms_[NNB_STAGE_COUNT] = {0};
  i64 count_[NNB_STAGE_COUNT] = {0};
};

// One stage of a transform: an NVTX range on the host thread named after the stage ("nnb:bin",
// "nnb:spread", "nnb:fft", "nnb:deconv", "nnb:interp", "nnb:phase"; visible in Nsight Systems and
// as ncu's --nvtx ranges, free when no tool is attached) and, when timing is on, CUDA events
// around the stage's launches.
const char* stage_range_name(int stage);
class ScopedStage {
public:
  ScopedStage(StageTimer& t, cudaStream_t s, int stage) : t_(t), s_(s), stage_(stage) {
    nvtxRangePushA(stage_range_name(stage_));
    t_.begin(s_, stage_);
  }
  ~ScopedStage() {
    t_.end(s_, stage_);
    nvtxRangePop();
  }

private:
  StageTimer& t_;
  cudaStream_t s_;
  int stage_;
};

// Complex fine grid with an in-place cuFFT plan (workspace from the plan's allocator).
// Replaces the reference's FFTGrid (src/neonufft/gpu/util/fft_grid.cpp:19-70).
template <typename T>
class FftGrid {
public:
  FftGrid(std::shared_ptr<DeviceAllocator> alloc, int dim, const i64* nf, int sign,
          cudaStream_t stream);
  ~FftGrid();
  void exec(cudaStream_t stream);
  // The same in-place transform on another buffer of the grid's shape (the plan's work area is
  // shared: executions on one stream are ordered).
  void exec_on(cplx_t<T>* data, cudaStream_t stream);
  // 3D grids that hold (or feed) `modes` modes, stored k mod nf: only the first ceil(n/2) and
  // the last floor(n/2) rows in y (n = modes[1]) carry modes. Type 1 (exec_to_modes) then needs
  // the z transform only on those rows, after the (y, x) transforms of every plane; type 2
  // (exec_from_modes: every other row is zero) needs it before them. Without pruning (other
  // dimensions, or rows that cover most of the grid) both are the full transform.
  void enable_mode_pruning(const i64* modes);
  void exec_to_modes(cplx_t<T>* data, cudaStream_t stream);
  void exec_from_modes(cplx_t<T>* data, cudaStream_t stream);
  cplx_t<T>* data() const { return grid_.data(); }
  i64 cells() const { return cells_; }
  const i64* nf() const { return nf_; }

private:
  void exec_plan(cufftHandle plan, cplx_t<T>* data, cudaStream_t stream);
  DevArray<cplx_t<T>> grid_;
  DevArray<unsigned char> work_;
  cufftHandle plan_ = 0;
  bool has_plan_ = false;
  int dim_;
  int sign_;
  i64 nf_[3] = {1, 1, 1};
  i64 cells_ = 1;
  // pruned form: (y, x) transforms of every z plane, and z transforms of the rows
  // [row0_[k], row0_[k] + rows_[k]) for k < nblocks_
  cufftHandle plan_yx_ = 0, plan_z_[2] = {0, 0};
  bool pruned_ = false;
  int nblocks_ = 0;
  i64 row0_[2] = {0, 0}, rows_[2] = {0, 0};
};

// Bin-sorted point set on one fine grid (see binning.cu).
template <typename T>
class PointSet {
public:
  explicit PointSet(std::shared_ptr<DeviceAllocator> alloc);
  // Bins M points; enqueues work on `stream`, then synchronises it and throws InputError for
  // non-finite coordinates (and, in the checked build, InternalError when the records' point
  // indices are not a permutation of 0 .. M - 1).
  void build(const BinGeom& g, CoordPtrs<T> x, i64 M, cudaStream_t stream);
  SortedPoints<T> view() const;
  i64 size() const { return M_; }
  const BinGeom& geom() const { return g_; }

private:
  BinGeom g_{};
  i64 M_ = 0;
  DevArray<PointRec<T>> rec_;
  DevArray<u32> counts_, bin_start_, ranks_, scan_tmp_, work_start_, work_owner_;
  DevArray<int> err_;
  DevArray<unsigned long long> checksum_;  // checked build: permutation checksum of the records
};

// Spreading / interpolation method for a plan: the requested one (validated), or the default:
// 3 (z-window, zwin.cu) for 3D plans with n_spread <= 8, else 1 (shared-memory slabs). Method 4
// is the z-window with tensor-core spreading (single precision, 5 <= n_spread <= 8).
int choose_method(int dim, int w, int requested, bool single);

// Tile shape for a grid and method: explicit request (validated) or the automatic choice.
// Method 3 uses (tx, 8, 1) tiles, tx in {4, 8}.
void choose_tile(int dim, int w, size_t complex_bytes, const i64* nf, const int* requested,
                 int method, int* tile);

// zmajor: order the bins plane-fastest (method 3).
BinGeom make_geom(int dim, int w, const i64* nf, const int* tile, const double* offset,
                  const double* scale, int zmajor = 0);

}  // namespace nnb
