// Host runtime: errors, allocator adapter, stage timer, cuFFT grid, point sets, tile choice.
#include <cstring>
#include <string>
#include <vector>

#include "runtime.hpp"

namespace nnb {

std::atomic<i64> g_kernel_launches{0};

void count_launch() { g_kernel_launches.fetch_add(1, std::memory_order_relaxed); }

const char* stage_range_name(int stage) {
  static const char* const names[] = {"nnb:bin", "nnb:spread", "nnb:fft", "nnb:deconv",
                                      "nnb:interp", "nnb:phase"};
  return (stage >= 0 && stage < int(sizeof(names) / sizeof(names[0]))) ? names[stage] : "nnb";
}

namespace {
struct CheckUnit {
  CheckReadFn read;
  void (*clear)();
  const char* name;
};
std::vector<CheckUnit>& check_units() {
  static std::vector<CheckUnit> units;  // filled during static initialisation of the library
  return units;
}
}  // namespace

bool register_check_record(CheckReadFn read, void (*clear)(), const char* unit) {
  check_units().push_back(CheckUnit{read, clear, unit});
  return true;
}

void check_device_records() {
#ifdef NNB_CHECKED
  // Never synchronise while a stream capture is open (the checked build is for uncaptured
  // debugging runs): the legacy stream reports one, or refuses the query during it.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(cudaStreamLegacy, &cap) != cudaSuccess) {
    (void)cudaGetLastError();
    return;
  }
  if (cap != cudaStreamCaptureStatusNone) return;
  NNB_CUDA(cudaDeviceSynchronize());
  for (const CheckUnit& u : check_units()) {
    const CheckRecord r = u.read();
    if (r.flag) {
      u.clear();
      throw_internal(std::string("checked build: index ") + std::to_string(r.index) +
                     " outside [0, " + std::to_string(r.bound) + ") at " + u.name + ":" +
                     std::to_string(r.line));
    }
  }
#endif
}

// ---- errors -----------------------------------------------------------------------------------
namespace {
thread_local std::string t_message;
}

const char* store_message(const std::string& msg) {
  t_message = msg;
  return t_message.c_str();
}

void throw_gpu(cudaError_t err, const char* what, const char* file, int line) {
  std::string m = std::string("Neonufft:: GPU error: ") + cudaGetErrorString(err) + " (" + what +
                  " at " + file + ":" + std::to_string(line) + ")";
  if (err == cudaErrorMemoryAllocation) throw neonufft::MemoryAllocError(store_message(m));
  throw neonufft::GPUError(store_message(m));
}

void throw_fft(cufftResult err, const char* what, const char* file, int line) {
  std::string m = std::string("Neonufft:: cuFFT error ") + std::to_string(int(err)) + " (" +
                  what + " at " + file + ":" + std::to_string(line) + ")";
  if (err == CUFFT_ALLOC_FAILED) throw neonufft::MemoryAllocError(store_message(m));
  throw neonufft::GPUFFTError(store_message(m));
}

void throw_input(const std::string& msg) {
  throw neonufft::InputError(store_message("Neonufft:: Input error: " + msg));
}

void throw_internal(const std::string& msg) {
  throw neonufft::InternalError(store_message("Neonufft:: Internal error: " + msg));
}

// ---- allocator ----------------------------------------------------------------------------------
DeviceAllocator::DeviceAllocator(const NnbAllocator* a) {
  if (a && a->allocate && a->deallocate) {
    a_ = *a;
    custom_ = true;
  }
}

void* DeviceAllocator::allocate(size_t bytes) {
  if (bytes == 0) return nullptr;
  void* p = nullptr;
  if (custom_) {
    p = a_.allocate(a_.ctx, bytes);
  } else {
    if (cudaMalloc(&p, bytes) != cudaSuccess) {
      (void)cudaGetLastError();
      p = nullptr;
    }
  }
  if (!p) {
    throw neonufft::MemoryAllocError(store_message(
        "Neonufft:: Memory allocation error: device allocation of " + std::to_string(bytes) +
        " bytes failed"));
  }
  in_use_ += bytes;
  return p;
}

void DeviceAllocator::deallocate(void* p, size_t bytes) noexcept {
  if (!p) return;
  in_use_ -= bytes;
  if (custom_) {
    a_.deallocate(a_.ctx, p);
  } else {
    (void)cudaFree(p);
  }
}

// ---- stage timer ------------------------------------------------------------------------------
StageTimer::~StageTimer() {
  for (auto& p : pending_) {
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  for (auto e : pool_) cudaEventDestroy(e);
  if (open_event_) cudaEventDestroy(open_event_);
}

cudaEvent_t StageTimer::get_event() {
  if (!pool_.empty()) {
    cudaEvent_t e = pool_.back();
    pool_.pop_back();
    return e;
  }
  cudaEvent_t e;
  NNB_CUDA(cudaEventCreate(&e));
  return e;
}

void StageTimer::begin(cudaStream_t s, int stage) {
  if (!enabled_) return;
  open_event_ = get_event();
  open_stage_ = stage;
  NNB_CUDA(cudaEventRecord(open_event_, s));
}

void StageTimer::end(cudaStream_t s, int stage) {
  if (!enabled_ || open_stage_ != stage || !open_event_) return;
  cudaEvent_t b = get_event();
  if (cudaEventRecord(b, s) != cudaSuccess) {
    pool_.push_back(b);
    return;
  }
  pending_.push_back(Pending{stage, open_event_, b});
  open_event_ = nullptr;
  open_stage_ = -1;
}

void StageTimer::collect(cudaStream_t s, double* ms, i64* count, bool reset) {
  NNB_CUDA(cudaStreamSynchronize(s));
  for (auto& p : pending_) {
    float t = 0.f;
    NNB_CUDA(cudaEventElapsedTime(&t, p.a, p.b));
    ms_[p.stage] += t;
    count_[p.stage] += 1;
    pool_.push_back(p.a);
    pool_.push_back(p.b);
  }
  pending_.clear();
  for (int i = 0; i < NNB_STAGE_COUNT; ++i) {
    if (ms) ms[i] = ms_[i];
    if (count) count[i] = count_[i];
  }
  if (reset) {
    for (int i = 0; i < NNB_STAGE_COUNT; ++i) {
      ms_[i] = 0;
      count_[i] = 0;
    }
  }
}

// ---- cuFFT grid -------------------------------------------------------------------------------
template <typename T>
FftGrid<T>::FftGrid(std::shared_ptr<DeviceAllocator> alloc, int dim, const i64* nf, int sign,
                    cudaStream_t stream)
    : grid_(alloc), work_(alloc), dim_(dim), sign_(sign) {
  for (int d = 0; d < dim; ++d) {
    nf_[d] = nf[d];
    cells_ *= nf[d];
  }
  grid_.reserve(size_t(cells_));
  // cuFFT is row-major; the grid is column-major (x fastest), so dims are passed reversed.
  int n[3];
  for (int d = 0; d < dim; ++d) {
    if (nf[d] > i64(0x7fffffff)) throw_input("fine grid dimension too large for cuFFT");
    n[dim - 1 - d] = int(nf[d]);
  }
  NNB_CUFFT(cufftCreate(&plan_));
  has_plan_ = true;
  NNB_CUFFT(cufftSetAutoAllocation(plan_, 0));
  size_t ws = 0;
  const cufftType type = std::is_same<T, float>::value ? CUFFT_C2C : CUFFT_Z2Z;
  NNB_CUFFT(cufftMakePlanMany(plan_, dim, n, nullptr, 1, 0, nullptr, 1, 0, type, 1, &ws));
  work_.reserve(ws);
  NNB_CUFFT(cufftSetWorkArea(plan_, work_.data()));
  NNB_CUFFT(cufftSetStream(plan_, stream));
}

template <typename T>
FftGrid<T>::~FftGrid() {
  if (has_plan_) cufftDestroy(plan_);
  if (plan_yx_) cufftDestroy(plan_yx_);
  for (cufftHandle p : plan_z_) {
    if (p) cufftDestroy(p);
  }
}

template <typename T>
void FftGrid<T>::enable_mode_pruning(const i64* modes) {
  if (dim_ != 3 || pruned_) return;
  const i64 nx = nf_[0], ny = nf_[1], nz = nf_[2];
  const i64 lo = (modes[1] + 1) / 2, hi = modes[1] / 2;  // rows [0, lo) and [ny - hi, ny)
  // (y, x) then z on a fraction f of the rows costs about 1.05 + 0.71 f ms at 480^3 in single
  // precision against 1.67 ms for the 3D transform: worth it up to three quarters of the rows
  if (4 * (lo + hi) > 3 * ny || nx * lo > i64(0x7fffffff) || nx * ny > i64(0x7fffffff)) return;
  const cufftType type = std::is_same<T, float>::value ? CUFFT_C2C : CUFFT_Z2Z;
  size_t ws_max = work_.size(), ws = 0;
  NNB_CUFFT(cufftCreate(&plan_yx_));
  NNB_CUFFT(cufftSetAutoAllocation(plan_yx_, 0));
  int n2[2] = {int(ny), int(nx)};  // row-major: y slow, x fast
  NNB_CUFFT(cufftMakePlanMany(plan_yx_, 2, n2, nullptr, 1, int(nx * ny), nullptr, 1,
                              int(nx * ny), type, int(nz), &ws));
  ws_max = std::max(ws_max, ws);
  const i64 r0[2] = {0, ny - hi}, nr[2] = {lo, hi};
  nblocks_ = 0;
  for (int k = 0; k < 2; ++k) {
    if (nr[k] <= 0) continue;
    // the same shape as the previous block: one plan serves both
    if (nblocks_ == 1 && nr[k] == rows_[0]) {
      row0_[1] = r0[k];
      rows_[1] = nr[k];
      nblocks_ = 2;
      continue;
    }
    cufftHandle& pz = plan_z_[nblocks_];
    NNB_CUFFT(cufftCreate(&pz));
    NNB_CUFFT(cufftSetAutoAllocation(pz, 0));
    int n1[1] = {int(nz)};
    int emb[1] = {int(nz)};
    // lines (x, y) of the block are consecutive elements; their z elements nx ny apart
    NNB_CUFFT(cufftMakePlanMany(pz, 1, n1, emb, int(nx * ny), 1, emb, int(nx * ny), 1, type,
                                int(nx * nr[k]), &ws));
    ws_max = std::max(ws_max, ws);
    row0_[nblocks_] = r0[k];
    rows_[nblocks_] = nr[k];
    ++nblocks_;
  }
  work_.reserve(ws_max);
  NNB_CUFFT(cufftSetWorkArea(plan_, work_.data()));
  NNB_CUFFT(cufftSetWorkArea(plan_yx_, work_.data()));
  for (cufftHandle p : plan_z_) {
    if (p) NNB_CUFFT(cufftSetWorkArea(p, work_.data()));
  }
  pruned_ = true;
}

template <typename T>
void FftGrid<T>::exec_plan(cufftHandle plan, cplx_t<T>* data, cudaStream_t stream) {
  NNB_CUFFT(cufftSetStream(plan, stream));
  const int dir = sign_ < 0 ? CUFFT_FORWARD : CUFFT_INVERSE;
  if constexpr (std::is_same<T, float>::value) {
    NNB_CUFFT(cufftExecC2C(plan, reinterpret_cast<cufftComplex*>(data),
                           reinterpret_cast<cufftComplex*>(data), dir));
  } else {
    NNB_CUFFT(cufftExecZ2Z(plan, reinterpret_cast<cufftDoubleComplex*>(data),
                           reinterpret_cast<cufftDoubleComplex*>(data), dir));
  }
}

template <typename T>
void FftGrid<T>::exec_to_modes(cplx_t<T>* data, cudaStream_t stream) {
  if (!pruned_) return exec_on(data, stream);
  exec_plan(plan_yx_, data, stream);
  for (int k = 0; k < nblocks_; ++k) {
    exec_plan(plan_z_[k < 2 && plan_z_[k] ? k : 0], data + row0_[k] * nf_[0], stream);
  }
}

template <typename T>
void FftGrid<T>::exec_from_modes(cplx_t<T>* data, cudaStream_t stream) {
  if (!pruned_) return exec_on(data, stream);
  for (int k = 0; k < nblocks_; ++k) {
    exec_plan(plan_z_[k < 2 && plan_z_[k] ? k : 0], data + row0_[k] * nf_[0], stream);
  }
  exec_plan(plan_yx_, data, stream);
}

template <typename T>
void FftGrid<T>::exec(cudaStream_t stream) { exec_on(grid_.data(), stream); }

template <typename T>
void FftGrid<T>::exec_on(cplx_t<T>* data, cudaStream_t stream) {
  NNB_CUFFT(cufftSetStream(plan_, stream));
  const int dir = sign_ < 0 ? CUFFT_FORWARD : CUFFT_INVERSE;
  if constexpr (std::is_same<T, float>::value) {
    NNB_CUFFT(cufftExecC2C(plan_, reinterpret_cast<cufftComplex*>(data),
                           reinterpret_cast<cufftComplex*>(data), dir));
  } else {
    NNB_CUFFT(cufftExecZ2Z(plan_, reinterpret_cast<cufftDoubleComplex*>(data),
                           reinterpret_cast<cufftDoubleComplex*>(data), dir));
  }
}

template class FftGrid<float>;
template class FftGrid<double>;

// ---- point sets -------------------------------------------------------------------------------
template <typename T>
PointSet<T>::PointSet(std::shared_ptr<DeviceAllocator> alloc)
    : rec_(alloc), counts_(alloc), bin_start_(alloc), ranks_(alloc), scan_tmp_(alloc),
      work_start_(alloc), work_owner_(alloc), err_(alloc), checksum_(alloc) {}

template <typename T>
void PointSet<T>::build(const BinGeom& g, CoordPtrs<T> x, i64 M, cudaStream_t stream) {
  if (M < 0) throw_input("negative number of points");
  if (M > i64(0xffffffffll)) throw_input("more than 2^32 - 1 points per plan");
  for (int d = 0; d < g.dim && M > 0; ++d) {
    if (!x.p[d]) throw_input("null coordinate pointer");
  }
  g_ = g;
  M_ = M;
  const i64 nt = g.total_tiles;
  counts_.reserve(size_t(nt));
  bin_start_.reserve(size_t(nt + 1));
  scan_tmp_.reserve(size_t(scan_tmp_words(nt)));
  rec_.reserve(size_t(M));
  ranks_.reserve(size_t(M));
  // work lists reuse counts_ and scan_tmp_ after binning (launch units never exceed the tiles)
  work_start_.reserve(size_t(nt + 1));
  work_owner_.reserve(size_t(nt + M / kWorkItemPoints + 2));
  err_.reserve(1);
  NNB_CUDA(cudaMemsetAsync(counts_.data(), 0, sizeof(u32) * nt, stream));
  NNB_CUDA(cudaMemsetAsync(err_.data(), 0, sizeof(int), stream));
  launch_bin_count<T>(g, x, M, counts_.data(), ranks_.data(), err_.data(), stream);
  launch_exclusive_scan(counts_.data(), bin_start_.data(), nt, scan_tmp_.data(), stream);
  launch_bin_scatter<T>(g, x, M, ranks_.data(), bin_start_.data(), rec_.data(), stream);
  int host_err = 0;
  NNB_CUDA(cudaMemcpyAsync(&host_err, err_.data(), sizeof(int), cudaMemcpyDeviceToHost, stream));
#ifdef NNB_CHECKED
  // The records' permutation must be 0 .. M - 1, each once: compare its sum and sum of squares
  // (wrapping 64-bit, as the device adds them) with the closed forms.
  checksum_.reserve(2);
  unsigned long long sums[2] = {0, 0};
  launch_perm_checksum<T>(rec_.data(), M, checksum_.data(), stream);
  NNB_CUDA(cudaMemcpyAsync(sums, checksum_.data(), sizeof(sums), cudaMemcpyDeviceToHost, stream));
#endif
  NNB_CUDA(cudaStreamSynchronize(stream));
  if (host_err) {
    M_ = 0;
    throw_input("non-finite point coordinate");
  }
#ifdef NNB_CHECKED
  const unsigned __int128 m = static_cast<unsigned __int128>(M);
  const unsigned long long want1 = static_cast<unsigned long long>(m * (m - (M > 0)) / 2);
  const unsigned long long want2 =
      M > 0 ? static_cast<unsigned long long>((m - 1) * m * (2 * m - 1) / 6) : 0ull;
  if (sums[0] != want1 || sums[1] != want2) {
    M_ = 0;
    throw_internal("checked build: the bin-sorted records are not a permutation of the points");
  }
#endif
}

template <typename T>
SortedPoints<T> PointSet<T>::view() const {
  SortedPoints<T> v;
  v.rec = rec_.data();
  v.M = M_;
  v.work.cnt = counts_.data();
  v.work.start = work_start_.data();
  v.work.tmp = scan_tmp_.data();
  v.work.owner = work_owner_.data();
  v.work.max_units = g_.total_tiles;
  v.work.max_items = g_.total_tiles + M_ / kWorkItemPoints + 2;
  v.bin_start = bin_start_.data();
  return v;
}

template class PointSet<float>;
template class PointSet<double>;

// ---- tiles ----------------------------------------------------------------------------------------
int choose_method(int dim, int w, int requested, bool single) {
  if (requested == 3 && (dim != 3 || w > 8)) {
    throw_input("spread method 3 needs a 3D plan with kernel width <= 8");
  }
  if (requested == 4 && (dim != 3 || w < 5 || w > 8 || !single)) {
    throw_input("spread method 4 needs a single-precision 3D plan with kernel width in [5, 8]");
  }
  if (requested == 5 && (dim != 3 || w > 8 || !single)) {
    throw_input("spread method 5 needs a single-precision 3D plan with kernel width <= 8");
  }
  if (requested < 0 || requested > 5) throw_input("spread method must be in [0, 5]");
  if (requested > 0) return requested;
  return (dim == 3 && w <= 8) ? 3 : 1;
}

void choose_tile(int dim, int w, size_t complex_bytes, const i64* nf, const int* requested,
                 int method, int* tile) {
  const int max_bits[3] = {dim == 3 ? 11 : (dim == 2 ? 16 : 31), dim == 3 ? 11 : 16, 10};
  bool explicit_tile = requested && requested[0] > 0;
  for (int d = 0; d < 3; ++d) tile[d] = 1;
  if (method == 4) {
    if (explicit_tile && requested[0] != 8) throw_input("spread method 4 uses tiles of 8 x 8 x 1");
    tile[0] = 8;
    tile[1] = 8;
    tile[2] = 1;
    return;
  }
  if (method == 5) {
    // the tensor-core spreading's accumulator rows are the (4 + w - 1)^2 <= 121 region cells
    if (explicit_tile && (requested[0] != 4 || (requested[1] != 0 && requested[1] != 4))) {
      throw_input("spread method 5 uses tiles of 4 x 4 x 1");
    }
    tile[0] = 4;
    tile[1] = 4;
    tile[2] = 1;
    return;
  }
  if (method == 3) {
    // x tile of 4 cells (11-cell register rows at w = 8): measured faster than 8 in both
    // precisions (3D w = 8 FP32 spreading 2.58 against 2.76 ms at M = 1e7, 24.6 against 25.8 ms
    // at M = 1e8, interpolation unchanged).
    tile[0] = 4;
    tile[1] = 8;
    if (explicit_tile) {
      if (requested[0] != 2 && requested[0] != 4 && requested[0] != 8) {
        throw_input("spread method 3 supports tiles of 2, 4 or 8 cells in x");
      }
      tile[0] = requested[0];
      if (requested[1] == 16) {
        // 16-row tiles (6 warps per CTA) are built for single precision only
        if (complex_bytes != 8) throw_input("spread method 3 uses 16-row tiles in single precision only");
        tile[1] = 16;
      } else if (requested[1] == 4) {
        // 4-row tiles (3 warps per CTA): single precision, 4 cells in x
        if (complex_bytes != 8 || tile[0] != 4) {
          throw_input("spread method 3 uses 4-row tiles in single precision with 4 cells in x");
        }
        tile[1] = 4;
      } else if (requested[1] != 0 && requested[1] != 8) {
        throw_input("spread method 3 supports tiles of 4, 8 or 16 rows");
      }
    }
    tile[2] = 1;
    return;
  }
  if (explicit_tile) {
    for (int d = 0; d < dim; ++d) {
      const int t = requested[d];
      if (t < 1 || (max_bits[d] < 31 && t > (1 << max_bits[d]))) throw_input("invalid tile shape");
      tile[d] = t;
    }
  } else {
    // Per-warp tile (bin); the kernels stack 4 of them along the last dimension per CTA.
    if (dim == 1) {
      tile[0] = 512;
    } else if (dim == 2) {
      tile[0] = 64;
      tile[1] = 16;
    } else {
      tile[0] = 8;
      tile[1] = 8;
      tile[2] = 8;
    }
    // Shrink the largest tile dimension until both kernels fit two 4-warp CTAs per SM, but not
    // below 4 cells (wide kernels then run with fewer warps per CTA), unless even one warp's
    // slab would not fit.
    const size_t budget = 113 * 1024;
    for (;;) {
      for (int d = 0; d < dim; ++d) {
        if (tile[d] > nf[d]) tile[d] = int(nf[d]);
      }
      const bool fits4 = spread_smem_bytes(dim, w, tile, complex_bytes, 4) <= budget &&
                         interp_smem_bytes(dim, w, tile, complex_bytes, 4) <= budget;
      const bool fits1 = spread_smem_bytes(dim, w, tile, complex_bytes, 1) <= 200 * 1024 &&
                         interp_smem_bytes(dim, w, tile, complex_bytes, 1) <= 200 * 1024;
      int big = 0;
      for (int d = 1; d < dim; ++d) {
        if (tile[d] > tile[big]) big = d;
      }
      if (fits4 || (fits1 && tile[big] <= 4) || tile[big] <= 1) break;
      tile[big] /= 2;
    }
  }
  for (int d = 0; d < dim; ++d) {
    if (tile[d] > nf[d]) tile[d] = int(nf[d]);
  }
  // the kernels fall back to fewer warps per CTA; one warp must fit
  if (spread_smem_bytes(dim, w, tile, complex_bytes, 1) > 227 * 1024 ||
      interp_smem_bytes(dim, w, tile, complex_bytes, 1) > 227 * 1024) {
    throw_input("tile too large for shared memory");
  }
}

BinGeom make_geom(int dim, int w, const i64* nf, const int* tile, const double* offset,
                  const double* scale, int zmajor) {
  BinGeom g{};
  g.dim = dim;
  g.w = w;
  g.zmajor = (dim == 3 && zmajor) ? 1 : 0;
  g.total_tiles = 1;
  for (int d = 0; d < 3; ++d) {
    if (d < dim) {
      // the binning kernels hold cell indices in 32-bit ints (cuFFT's own limit as well)
      if (nf[d] > i64(0x7fffffff)) throw_input("fine grid dimension too large");
      g.nf[d] = nf[d];
      g.tile[d] = tile[d];
      g.ntiles[d] = int((nf[d] + tile[d] - 1) / tile[d]);
      g.offset[d] = offset ? offset[d] : 0.0;
      g.scale[d] = scale ? scale[d] : 1.0;
    } else {
      g.nf[d] = 1;
      g.tile[d] = 1;
      g.ntiles[d] = 1;
      g.offset[d] = 0.0;
      g.scale[d] = 1.0;
    }
    g.total_tiles *= g.ntiles[d];
  }
  if (g.total_tiles > i64(0x7fffffff)) throw_input("too many tiles");
  if (g.zmajor && (g.tile[0] > 16 || g.tile[1] > 16 || g.tile[2] != 1 || g.nf[2] >= (i64(1) << 24))) {
    throw_input("plane-major binning needs tiles of at most 16 x 16 x 1 and fewer than 2^24 planes");
  }
  return g;
}

}  // namespace nnb
