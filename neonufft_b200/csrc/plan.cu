// Plan implementations (see plan.hpp).
#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "plan.hpp"

namespace nnb {

namespace {

// Placeholder until the constructor resolves the method (choose_method in runtime.cu).
constexpr int kDefaultMethod = 1;

template <typename T>
constexpr bool is_single() {
  return std::is_same<T, float>::value;
}

template <typename T>
void upload(DevArray<T>& dst, const std::vector<double>& src, cudaStream_t stream) {
  std::vector<T> host(src.begin(), src.end());
  dst.reserve(host.size());
  NNB_CUDA(cudaMemcpyAsync(dst.data(), host.data(), sizeof(T) * host.size(),
                           cudaMemcpyHostToDevice, stream));
  // pageable source: the copy has been staged when cudaMemcpyAsync returns, but keep the
  // host vector alive until the stream reaches it to stay independent of that detail.
  NNB_CUDA(cudaStreamSynchronize(stream));
}

template <typename T>
CoordPtrs<T> coords(int dim, const void* const* loc) {
  CoordPtrs<T> c{{nullptr, nullptr, nullptr}};
  if (!loc) return c;
  for (int d = 0; d < dim; ++d) c.p[d] = static_cast<const T*>(loc[d]);
  return c;
}

void check_strides(int dim, const i64* modes, const i64* strides) {
  if (!strides) throw_input("null strides");
  for (int d = 0; d < dim; ++d) {
    if (strides[d] < 1 && modes[d] > 1) throw_input("strides must be positive");
  }
}

}  // namespace

void PlanBase::transform_type_1_many(i64 count, const void* in, i64 in_bdist, void* out,
                                     i64 out_bdist, const i64* out_strides) {
  NnbPlanInfo inf{};
  info(&inf);
  const size_t csz = inf.precision == NNB_FLOAT ? 8 : 16;
  for (i64 v = 0; v < count; ++v) {
    transform_type_1(static_cast<const char*>(in) + size_t(v * in_bdist) * csz,
                     static_cast<char*>(out) + size_t(v * out_bdist) * csz, out_strides);
  }
}

void PlanBase::fused_job(int, const void*, void*, void*) const {
  throw_internal("plan has no persistent z-window step");
}
void PlanBase::fused_pre(int, const void*, const i64*) {
  throw_internal("plan has no persistent z-window step");
}
void PlanBase::fused_post(int, void*, const i64*) {
  throw_internal("plan has no persistent z-window step");
}

void validate_options(const NnbOptions& opt) {
  if (!(opt.tol > 0.0) || !std::isfinite(opt.tol)) throw_input("tol must be positive and finite");
  if (!(opt.upsampfac > 1.0) || !std::isfinite(opt.upsampfac)) {
    throw_input("upsampfac must be greater than 1");
  }
  if (opt.order != NEONUFFT_MODE_ORDER_FFT && opt.order != NEONUFFT_MODE_ORDER_CMCL) {
    throw_input("invalid mode order");
  }
  if (opt.kernel_type != NEONUFFT_ES_KERNEL) throw_input("invalid kernel type");
  if (!std::isfinite(opt.recenter_threshold)) throw_input("invalid recenter threshold");
  for (int d = 0; d < 3; ++d) {
    if (opt.tile[d] < 0) throw_input("invalid tile shape");
  }
  if (opt.spread_method < 0 || opt.spread_method > 5) throw_input("invalid spread method");
  if (opt.n_spread != 0 && (opt.n_spread < 2 || opt.n_spread > 16)) {
    throw_input("kernel width must be in [2, 16]");
  }
}

// An internal stream and events with which transform_type_1_many runs the FFTs and
// deconvolutions of one pair of vectors while the next pair spreads (created on first use).
struct SidePipe {
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  cudaEvent_t spread[2] = {nullptr, nullptr}, done[2] = {nullptr, nullptr};
  SidePipe() = default;
  SidePipe(const SidePipe&) = delete;
  SidePipe& operator=(const SidePipe&) = delete;
  void ensure() {
    if (side) return;
    for (cudaEvent_t* e : {&fork, &join, &spread[0], &spread[1], &done[0], &done[1]}) {
      NNB_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    }
    NNB_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
  }
  ~SidePipe() {  // waits for the stream's work, which reads and writes the plan's arrays
    if (side) cudaStreamSynchronize(side);
    for (cudaEvent_t e : {fork, join, spread[0], spread[1], done[0], done[1]}) {
      if (e) cudaEventDestroy(e);
    }
    if (side) cudaStreamDestroy(side);
  }
};

// =============================================================================================
// Type 1 / type 2.
// =============================================================================================
template <typename T>
class PlanImpl final : public PlanBase {
public:
  PlanImpl(int dim, const NnbOptions& opt, int sign, i64 M, const void* const* loc,
           const i64* modes, cudaStream_t stream, const NnbAllocator* alloc)
      : alloc_(std::make_shared<DeviceAllocator>(alloc)),
        dim_(dim),
        opt_(opt),
        sign_(sign < 0 ? -1 : 1),
        stream_(stream),
        points_(alloc_),
        pair_grid_(alloc_) {
    if (!modes) throw_input("null modes");
    for (int d = 0; d < 3; ++d) {
      modes_[d] = 1;
      nf_[d] = 1;
    }
    for (int d = 0; d < dim; ++d) {
      if (modes[d] < 1) throw_input("number of modes must be positive");
      modes_[d] = modes[d];
    }
    kp_ = kernel_param(opt.tol, opt.upsampfac, is_single<T>(), opt.n_spread);
    if (kp_.w < 2 || kp_.w > 16) throw_internal("n_spread not in [2, 16]");
    method_ = choose_method(dim, kp_.w, opt.spread_method, is_single<T>());
    for (int d = 0; d < dim; ++d) nf_[d] = fine_grid_size(modes_[d], opt.upsampfac, kp_.w);
    fft_ = std::make_unique<FftGrid<T>>(alloc_, dim, nf_, sign_, stream_);
    fft_->enable_mode_pruning(modes_);
    for (int d = 0; d < dim; ++d) {
      corr_[d].set_allocator(alloc_);
      upload(corr_[d], deconv_factors(kp_, nf_[d]), stream_);
    }
    choose_tile(dim, kp_.w, sizeof(cplx_t<T>), nf_, opt.tile, method_, tile_);
    geom_ = make_geom(dim, kp_.w, nf_, tile_, nullptr, nullptr, method_ >= 3);
    set_points(M, loc);
  }

  void set_points(i64 M, const void* const* loc) override {
    if (M < 0) throw_input("negative number of points");
    if (M > 0 && !loc) throw_input("null coordinate pointers");
    ScopedStage st(timer_, stream_, NNB_STAGE_BIN);
    points_.build(geom_, coords<T>(dim_, loc), M, stream_);
  }

  void transform_type_1(const void* in, void* out, const i64* out_strides) override {
    const i64 M = points_.size();
    if (!out) throw_input("null output");
    if (M > 0 && !in) throw_input("null input");
    check_strides(dim_, modes_, out_strides);
    NNB_CUDA(cudaMemsetAsync(fft_->data(), 0, sizeof(cplx_t<T>) * fft_->cells(), stream_));
    {
      ScopedStage st(timer_, stream_, NNB_STAGE_SPREAD);
      if (M > 0) launch_spread<T>(spread_args(in), stream_);
    }
    {
      ScopedStage st(timer_, stream_, NNB_STAGE_FFT);
      fft_->exec_to_modes(fft_->data(), stream_);
    }
    {
      ScopedStage st(timer_, stream_, NNB_STAGE_DECONV);
      launch_downsample<T>(deconv_args(out_strides), fft_->data(), static_cast<cplx_t<T>*>(out),
                           stream_);
    }
  }

  // Single precision on the z-window kernels (default or 4-row tiles) spreads the vectors two
  // at a time: each staged point serves both, into a pair of fine grids; each grid is then
  // transformed and deconvolved into its output.
  void transform_type_1_many(i64 count, const void* in, i64 in_bdist, void* out, i64 out_bdist,
                             const i64* out_strides) override {
    const i64 M = points_.size();
    if (count < 0) throw_input("negative number of transforms");
    if (count == 0) return;
    if (!out) throw_input("null output");
    if (M > 0 && !in) throw_input("null input");
    check_strides(dim_, modes_, out_strides);
    i64 extent = 1;
    for (int d = 0; d < dim_; ++d) extent += (modes_[d] - 1) * out_strides[d];
    if (count > 1 && (in_bdist < M || out_bdist < extent)) {
      throw_input("input / output distances smaller than one vector");
    }
    const bool pairs = is_single<T>() && method_ == 3 && tile_[0] == 4 &&
                       (tile_[1] == 8 || tile_[1] == 4) && count > 1 && M > 0;
    if (!pairs) {
      PlanBase::transform_type_1_many(count, in, in_bdist, out, out_bdist, out_strides);
      return;
    }
    const auto* iv = static_cast<const cplx_t<T>*>(in);
    auto* ov = static_cast<cplx_t<T>*>(out);
    const i64 cells = fft_->cells();
    // Pairs alternate between two sets of two fine grids: pair p spreads on the plan's stream
    // while the FFTs and deconvolutions of pair p - 1 run on the internal stream (the FFTs are
    // bound by memory, the spreading by instruction issue); pair p + 2 reuses pair p's grids
    // once their FFTs are done. The caller's stream then waits for the last pair. (Measured at
    // 1e8 points, 480^3 grids, 8 vectors: 121.2 ms against 122.8 ms on one stream; with the
    // internal stream at the highest priority, 122.6 ms; clearing the grids on the internal
    // stream, 121.4 ms.)
    const i64 npairs = (count + 1) / 2;
    const i64 set_cells = 2 * cells;
    pair_grid_.reserve(size_t((npairs > 1 ? 2 : 1) * set_cells));
    pipe_.ensure();
    NNB_CUDA(cudaEventRecord(pipe_.fork, stream_));
    NNB_CUDA(cudaStreamWaitEvent(pipe_.side, pipe_.fork, 0));
    for (i64 p = 0; p < npairs; ++p) {
      const i64 v = 2 * p;
      const i64 nv = std::min<i64>(2, count - v);
      const int b = int(p % 2);
      cplx_t<T>* grids = pair_grid_.data() + b * set_cells;
      if (p >= 2) NNB_CUDA(cudaStreamWaitEvent(stream_, pipe_.done[b], 0));
      NNB_CUDA(cudaMemsetAsync(grids, 0, sizeof(cplx_t<T>) * size_t(nv * cells), stream_));
      {
        ScopedStage st(timer_, stream_, NNB_STAGE_SPREAD);
        SpreadArgs<T> a = spread_args(iv + v * in_bdist);
        a.grid = grids;
        a.in_bdist = in_bdist;
        a.grid_bdist = cells;
        a.batch = int(nv);
        launch_spread<T>(a, stream_);
      }
      NNB_CUDA(cudaEventRecord(pipe_.spread[b], stream_));
      NNB_CUDA(cudaStreamWaitEvent(pipe_.side, pipe_.spread[b], 0));
      for (i64 j = 0; j < nv; ++j) {
        cplx_t<T>* gj = grids + j * cells;
        {
          ScopedStage st(timer_, pipe_.side, NNB_STAGE_FFT);
          fft_->exec_to_modes(gj, pipe_.side);
        }
        ScopedStage st(timer_, pipe_.side, NNB_STAGE_DECONV);
        launch_downsample<T>(deconv_args(out_strides), gj, ov + (v + j) * out_bdist,
                             pipe_.side);
      }
      NNB_CUDA(cudaEventRecord(pipe_.done[b], pipe_.side));
    }
    NNB_CUDA(cudaEventRecord(pipe_.join, pipe_.side));
    NNB_CUDA(cudaStreamWaitEvent(stream_, pipe_.join, 0));
  }

  void transform_type_2(const void* in, const i64* in_strides, void* out) override {
    const i64 M = points_.size();
    if (!in) throw_input("null input");
    if (M > 0 && !out) throw_input("null output");
    check_strides(dim_, modes_, in_strides);
    {
      ScopedStage st(timer_, stream_, NNB_STAGE_DECONV);
      launch_upsample<T>(deconv_args(in_strides), static_cast<const cplx_t<T>*>(in),
                         fft_->data(), stream_);
    }
    {
      ScopedStage st(timer_, stream_, NNB_STAGE_FFT);
      fft_->exec_from_modes(fft_->data(), stream_);
    }
    if (M > 0) {
      ScopedStage st(timer_, stream_, NNB_STAGE_INTERP);
      launch_interp<T>(interp_args(out), stream_);
    }
  }

  bool fused_key(int* key) const override {
    if (method_ != 3 || dim_ != 3 || points_.size() == 0 || tile_[1] != 8) return false;
    *key = kp_.w | (tile_[0] << 8);
    return true;
  }

  void fused_job(int type, const void* in, void* out, void* job) const override {
    int key;
    if (!fused_key(&key)) throw_internal("plan has no persistent z-window step");
    if (type == 1) {
      *static_cast<ZSpreadJob<T>*>(job) = zwin_spread_job<T>(spread_args(in));
    } else {
      *static_cast<ZInterpJob<T>*>(job) = zwin_interp_job<T>(interp_args(out));
    }
  }

  void fused_pre(int type, const void* in, const i64* strides) override {
    check_strides(dim_, modes_, strides);
    if (type == 1) {
      NNB_CUDA(cudaMemsetAsync(fft_->data(), 0, sizeof(cplx_t<T>) * fft_->cells(), stream_));
    } else {
      launch_upsample<T>(deconv_args(strides), static_cast<const cplx_t<T>*>(in), fft_->data(),
                         stream_);
      fft_->exec_from_modes(fft_->data(), stream_);
    }
    zwin_build_work_list<T>(geom_, points_.view(), stream_);
  }

  void fused_post(int type, void* out, const i64* strides) override {
    if (type != 1) return;
    check_strides(dim_, modes_, strides);
    fft_->exec_to_modes(fft_->data(), stream_);
    launch_downsample<T>(deconv_args(strides), fft_->data(), static_cast<cplx_t<T>*>(out),
                         stream_);
  }

  void info(NnbPlanInfo* info) const override {
    *info = NnbPlanInfo{};
    info->dim = dim_;
    info->precision = is_single<T>() ? NNB_FLOAT : NNB_DOUBLE;
    info->n_spread = kp_.w;
    info->spread_method = method_;
    info->es_beta = kp_.beta;
    for (int d = 0; d < 3; ++d) {
      info->grid[d] = nf_[d];
      info->spread_grid[d] = nf_[d];
      info->tile[d] = d < dim_ ? tile_[d] : 1;
    }
    info->num_in = points_.size();
    info->num_out = 0;
    info->batch_size = 1;
    info->device_bytes = alloc_->in_use();
  }

  StageTimer& timer() override { return timer_; }
  cudaStream_t stream() const override { return stream_; }

private:
  SpreadArgs<T> spread_args(const void* in) const {
    SpreadArgs<T> a{};
    a.g = geom_;
    a.pts = points_.view();
    a.in = static_cast<const cplx_t<T>*>(in);
    a.prephase = nullptr;
    a.grid = fft_->data();
    a.in_bdist = 0;
    a.grid_bdist = 0;
    a.batch = 1;
    a.beta = T(kp_.beta);
    a.c = T(kp_.c);
    a.method = method_;
    return a;
  }

  InterpArgs<T> interp_args(void* out) const {
    InterpArgs<T> a{};
    a.g = geom_;
    a.pts = points_.view();
    a.grid = fft_->data();
    a.postphase = nullptr;
    a.out = static_cast<cplx_t<T>*>(out);
    a.beta = T(kp_.beta);
    a.c = T(kp_.c);
    a.method = method_;
    return a;
  }

  DeconvArgs<T> deconv_args(const i64* strides) const {
    DeconvArgs<T> a{};
    a.dim = dim_;
    a.order = opt_.order;
    for (int d = 0; d < 3; ++d) {
      a.nf[d] = nf_[d];
      a.modes[d] = modes_[d];
      a.stride[d] = d < dim_ ? strides[d] : 0;
      a.corr[d] = d < dim_ ? corr_[d].data() : nullptr;
    }
    return a;
  }

  std::shared_ptr<DeviceAllocator> alloc_;
  int dim_;
  NnbOptions opt_;
  int sign_;
  cudaStream_t stream_;
  KernelParam kp_;
  i64 modes_[3];
  i64 nf_[3];
  int tile_[3] = {1, 1, 1};
  int method_ = kDefaultMethod;
  BinGeom geom_{};
  std::unique_ptr<FftGrid<T>> fft_;
  DevArray<T> corr_[3];
  PointSet<T> points_;
  DevArray<cplx_t<T>> pair_grid_;  // transform_type_1_many: two sets of two fine grids
  StageTimer timer_;
  SidePipe pipe_;  // declared last: destroyed (its stream drained) before the arrays are freed
};

// =============================================================================================
// Type 3.
// =============================================================================================
template <typename T>
class PlanT3Impl final : public PlanT3Base {
public:
  PlanT3Impl(int dim, const NnbOptions& opt, int sign, i64 batch, cudaStream_t stream,
             const NnbAllocator* alloc)
      : alloc_(std::make_shared<DeviceAllocator>(alloc)),
        dim_(dim),
        opt_(opt),
        sign_(sign < 0 ? -1 : 1),
        batch_(batch),
        stream_(stream),
        spread_grid_(alloc_),
        prephase_(alloc_),
        postphase_(alloc_),
        in_points_(alloc_),
        out_points_(alloc_) {
    if (batch < 1) throw_input("batch size must be positive");
    if (batch > 65535) throw_input("batch size above 65535");
    kp_ = kernel_param(opt.tol, opt.upsampfac, is_single<T>(), opt.n_spread);
    if (kp_.w < 2 || kp_.w > 16) throw_internal("n_spread not in [2, 16]");
    method_ = choose_method(dim, kp_.w, opt.spread_method, is_single<T>());
    for (auto& c : corr_) c.set_allocator(alloc_);
  }

  // Bounds from the point sets, computed on the device (reference
  // src/neonufft/gpu/plan_t3_impl.hpp:88-111), then the bounds constructor path.
  void init_from_points(i64 M, const void* const* in_pts, i64 K, const void* const* out_pts) {
    if (M < 0 || K < 0) throw_input("negative number of points");
    if ((M > 0 && !in_pts) || (K > 0 && !out_pts)) throw_input("null coordinate pointers");
    double in_min[3] = {0, 0, 0}, in_max[3] = {0, 0, 0};
    double out_min[3] = {0, 0, 0}, out_max[3] = {0, 0, 0};
    {
      ScopedStage st(timer_, stream_, NNB_STAGE_PHASE);
      DevArray<unsigned long long> enc(alloc_);
      enc.reserve(4 * dim_);
      unsigned long long host[12];
      init_min_max(host, 4 * dim_);
      NNB_CUDA(cudaMemcpyAsync(enc.data(), host, sizeof(host[0]) * 4 * dim_,
                               cudaMemcpyHostToDevice, stream_));
      if (M > 0) launch_min_max<T>(dim_, coords<T>(dim_, in_pts), M, enc.data(), stream_);
      if (K > 0) {
        launch_min_max<T>(dim_, coords<T>(dim_, out_pts), K, enc.data() + 2 * dim_, stream_);
      }
      NNB_CUDA(cudaMemcpyAsync(host, enc.data(), sizeof(host[0]) * 4 * dim_,
                               cudaMemcpyDeviceToHost, stream_));
      NNB_CUDA(cudaStreamSynchronize(stream_));
      double mm[12];
      decode_min_max(host, 4 * dim_, mm);
      for (int d = 0; d < dim_; ++d) {
        if (M > 0) {
          in_min[d] = mm[2 * d];
          in_max[d] = mm[2 * d + 1];
        }
        if (K > 0) {
          out_min[d] = mm[2 * dim_ + 2 * d];
          out_max[d] = mm[2 * dim_ + 2 * d + 1];
        }
      }
    }
    init(in_min, in_max, out_min, out_max);
    set_input_points(M, in_pts);
    set_output_points(K, out_pts);
  }

  // Geometry, grids, FFT plan and correction factors (reference plan_t3_impl.hpp:255-306).
  void init(const double* in_min, const double* in_max, const double* out_min,
            const double* out_max) {
    for (int d = 0; d < dim_; ++d) {
      if (!(T(in_min[d]) <= T(in_max[d]))) throw_input("Invalid input bounds.");
      if (!(T(out_min[d]) <= T(out_max[d]))) throw_input("Invalid output bounds.");
    }
    i64 spread_cells = 1;
    for (int d = 0; d < 3; ++d) {
      nf1_[d] = 1;
      nfft_[d] = 1;
      C_[d] = D_[d] = 0;
      gamma_[d] = h_[d] = 1;
    }
    for (int d = 0; d < dim_; ++d) {
      const T3Dim<T> g = t3_geometry<T>(kp_.w, opt_.upsampfac, T(opt_.recenter_threshold),
                                        T(in_min[d]), T(in_max[d]), T(out_min[d]),
                                        T(out_max[d]));
      nf1_[d] = g.spread_grid;
      nfft_[d] = g.fft_grid;
      C_[d] = double(g.input_offset);
      D_[d] = double(g.output_offset);
      gamma_[d] = double(g.gamma);
      // The spread grid's spacing is exactly 2 pi / nf1: the inputs land on it through
      // (x - C) / gamma, so the targets must be mapped with the same spacing. The reference's
      // h = T(2) T(pi) / T(nf1) carries T's rounding (2.5e-8 relative in single precision),
      // which scales every target frequency by (1 + delta) and costs |x s| delta of relative
      // error: 1.1e-4 at half-widths 50 and 200 in 2D. C, D and gamma need no such care:
      // each enters both sides of x s = (x - C)(s - D) + x D + C (s - D) with the same value.
      h_[d] = 2.0 * 3.14159265358979323846 / double(nf1_[d]);
      spread_cells *= nf1_[d];
    }
    spread_cells_ = spread_cells;
    spread_grid_.reserve(size_t(spread_cells * batch_));
    NNB_CUDA(cudaMemsetAsync(spread_grid_.data(), 0,
                             sizeof(cplx_t<T>) * size_t(spread_cells * batch_), stream_));
    fft_ = std::make_unique<FftGrid<T>>(alloc_, dim_, nfft_, sign_, stream_);
    fft_->enable_mode_pruning(nf1_);  // the spread grid's nf1 modes feed the FFT grid
    for (int d = 0; d < dim_; ++d) upload(corr_[d], deconv_factors(kp_, nfft_[d]), stream_);
    const PhiHatQuad quad = phi_hat_quadrature(kp_);
    if (quad.z.size() > 32) throw_internal("too many quadrature nodes");
    quad_.n = int(quad.z.size());
    for (int i = 0; i < quad_.n; ++i) {
      quad_.z[i] = quad.z[i];
      quad_.kv[i] = quad.kv[i];
    }
    choose_tile(dim_, kp_.w, sizeof(cplx_t<T>), nf1_, opt_.tile, method_, in_tile_);
    choose_tile(dim_, kp_.w, sizeof(cplx_t<T>), nfft_, opt_.tile, method_, out_tile_);
    NNB_CUDA(cudaStreamSynchronize(stream_));
  }

  void set_input_points(i64 M, const void* const* pts) override {
    if (M < 0) throw_input("negative number of points");
    if (M > 0 && !pts) throw_input("null coordinate pointers");
    const CoordPtrs<T> x = coords<T>(dim_, pts);
    bool need_pre = false;
    for (int d = 0; d < dim_; ++d) need_pre |= (D_[d] != 0.0);
    if (need_pre && M > 0) {
      ScopedStage st(timer_, stream_, NNB_STAGE_PHASE);
      prephase_.reserve(size_t(M));
      launch_prephase<T>(dim_, sign_, x, M, D_, prephase_.data(), stream_);
      has_prephase_ = true;
    } else {
      prephase_.release();
      has_prephase_ = false;
    }
    double scale[3];
    for (int d = 0; d < 3; ++d) scale[d] = d < dim_ ? 1.0 / gamma_[d] : 1.0;
    const BinGeom g = make_geom(dim_, kp_.w, nf1_, in_tile_, C_, scale, method_ >= 3);
    ScopedStage st(timer_, stream_, NNB_STAGE_BIN);
    in_points_.build(g, x, M, stream_);
  }

  void set_output_points(i64 K, const void* const* pts) override {
    if (K < 0) throw_input("negative number of points");
    if (K > 0 && !pts) throw_input("null coordinate pointers");
    const CoordPtrs<T> s = coords<T>(dim_, pts);
    double scale[3];
    for (int d = 0; d < 3; ++d) scale[d] = d < dim_ ? gamma_[d] * h_[d] : 1.0;
    const BinGeom g = make_geom(dim_, kp_.w, nfft_, out_tile_, D_, scale, method_ >= 3);
    {
      ScopedStage st(timer_, stream_, NNB_STAGE_BIN);
      out_points_.build(g, s, K, stream_);
    }
    ScopedStage st(timer_, stream_, NNB_STAGE_PHASE);
    postphase_.reserve(size_t(K));
    if (K > 0) {
      launch_postphase<T>(dim_, sign_, s, K, D_, C_, scale, quad_, postphase_.data(), stream_);
    }
    NNB_CUDA(cudaStreamSynchronize(stream_));
  }

  void add_input(const void* in, i64 bdist) override {
    const i64 M = in_points_.size();
    if (M == 0) return;
    if (!in) throw_input("null input");
    if (bdist <= 0) bdist = M;
    ScopedStage st(timer_, stream_, NNB_STAGE_SPREAD);
    SpreadArgs<T> a{};
    a.g = in_points_.geom();
    a.pts = in_points_.view();
    a.in = static_cast<const cplx_t<T>*>(in);
    a.prephase = has_prephase_ ? prephase_.data() : nullptr;
    a.grid = spread_grid_.data();
    a.in_bdist = bdist;
    a.grid_bdist = spread_cells_;
    a.batch = int(batch_);
    a.beta = T(kp_.beta);
    a.c = T(kp_.c);
    a.method = method_;
    launch_spread<T>(a, stream_);
  }

  void transform(void* out, i64 bdist) override {
    const i64 K = out_points_.size();
    if (K == 0) return;
    if (!out) throw_input("null output");
    if (bdist <= 0) bdist = K;
    DeconvArgs<T> dc{};
    dc.dim = dim_;
    dc.order = NEONUFFT_MODE_ORDER_CMCL;
    i64 stride = 1;
    for (int d = 0; d < 3; ++d) {
      dc.nf[d] = nfft_[d];
      dc.modes[d] = nf1_[d];
      dc.stride[d] = stride;
      stride *= nf1_[d];
      dc.corr[d] = d < dim_ ? corr_[d].data() : nullptr;
    }
    for (i64 b = 0; b < batch_; ++b) {
      {
        ScopedStage st(timer_, stream_, NNB_STAGE_DECONV);
        launch_upsample<T>(dc, spread_grid_.data() + b * spread_cells_, fft_->data(), stream_);
      }
      {
        ScopedStage st(timer_, stream_, NNB_STAGE_FFT);
        fft_->exec_from_modes(fft_->data(), stream_);
      }
      ScopedStage st(timer_, stream_, NNB_STAGE_INTERP);
      InterpArgs<T> a{};
      a.g = out_points_.geom();
      a.pts = out_points_.view();
      a.grid = fft_->data();
      a.postphase = postphase_.data();
      a.out = static_cast<cplx_t<T>*>(out) + b * bdist;
      a.beta = T(kp_.beta);
      a.c = T(kp_.c);
      a.method = method_;
      launch_interp<T>(a, stream_);
    }
  }

  void reset() override {
    NNB_CUDA(cudaMemsetAsync(spread_grid_.data(), 0,
                             sizeof(cplx_t<T>) * size_t(spread_cells_ * batch_), stream_));
  }

  void info(NnbPlanInfo* info) const override {
    *info = NnbPlanInfo{};
    info->dim = dim_;
    info->precision = is_single<T>() ? NNB_FLOAT : NNB_DOUBLE;
    info->n_spread = kp_.w;
    info->spread_method = method_;
    info->es_beta = kp_.beta;
    for (int d = 0; d < 3; ++d) {
      info->grid[d] = nfft_[d];
      info->spread_grid[d] = nf1_[d];
      info->tile[d] = d < dim_ ? in_tile_[d] : 1;
      info->input_offset[d] = C_[d];
      info->output_offset[d] = D_[d];
      info->gamma[d] = gamma_[d];
      info->h[d] = h_[d];
    }
    info->num_in = in_points_.size();
    info->num_out = out_points_.size();
    info->batch_size = batch_;
    info->device_bytes = alloc_->in_use();
  }

  StageTimer& timer() override { return timer_; }
  cudaStream_t stream() const override { return stream_; }

private:
  std::shared_ptr<DeviceAllocator> alloc_;
  int dim_;
  NnbOptions opt_;
  int sign_;
  i64 batch_;
  cudaStream_t stream_;
  KernelParam kp_;
  i64 nf1_[3] = {1, 1, 1};
  i64 nfft_[3] = {1, 1, 1};
  double C_[3] = {0, 0, 0}, D_[3] = {0, 0, 0};
  double gamma_[3] = {1, 1, 1}, h_[3] = {1, 1, 1};
  int in_tile_[3] = {1, 1, 1};
  int out_tile_[3] = {1, 1, 1};
  int method_ = kDefaultMethod;
  i64 spread_cells_ = 0;
  DevArray<cplx_t<T>> spread_grid_;
  std::unique_ptr<FftGrid<T>> fft_;
  DevArray<T> corr_[3];
  PostphaseQuad quad_{};
  DevArray<cplx_t<T>> prephase_;
  DevArray<cplx_t<T>> postphase_;
  bool has_prephase_ = false;
  PointSet<T> in_points_;
  PointSet<T> out_points_;
  StageTimer timer_;
};

// =============================================================================================
// Factories.
// =============================================================================================
namespace {
void check_dim_prec(NnbPrecision prec, int dim) {
  if (dim < 1 || dim > 3) throw_input("dimension must be 1, 2 or 3");
  if (prec != NNB_FLOAT && prec != NNB_DOUBLE) throw_input("invalid precision");
}
}  // namespace

std::unique_ptr<PlanBase> make_plan(NnbPrecision prec, int dim, const NnbOptions& opt, int sign,
                                    i64 M, const void* const* loc, const i64* modes,
                                    cudaStream_t stream, const NnbAllocator* alloc) {
  check_dim_prec(prec, dim);
  validate_options(opt);
  if (prec == NNB_FLOAT) {
    return std::make_unique<PlanImpl<float>>(dim, opt, sign, M, loc, modes, stream, alloc);
  }
  return std::make_unique<PlanImpl<double>>(dim, opt, sign, M, loc, modes, stream, alloc);
}

std::unique_ptr<PlanT3Base> make_plan_t3(NnbPrecision prec, int dim, const NnbOptions& opt,
                                         int sign, i64 M, const void* const* in_pts, i64 K,
                                         const void* const* out_pts, cudaStream_t stream,
                                         i64 batch, const NnbAllocator* alloc) {
  check_dim_prec(prec, dim);
  validate_options(opt);
  if (prec == NNB_FLOAT) {
    auto p = std::make_unique<PlanT3Impl<float>>(dim, opt, sign, batch, stream, alloc);
    p->init_from_points(M, in_pts, K, out_pts);
    return p;
  }
  auto p = std::make_unique<PlanT3Impl<double>>(dim, opt, sign, batch, stream, alloc);
  p->init_from_points(M, in_pts, K, out_pts);
  return p;
}

std::unique_ptr<PlanT3Base> make_plan_t3_bounds(NnbPrecision prec, int dim,
                                                const NnbOptions& opt, int sign,
                                                const double* in_min, const double* in_max,
                                                const double* out_min, const double* out_max,
                                                cudaStream_t stream, i64 batch,
                                                const NnbAllocator* alloc) {
  check_dim_prec(prec, dim);
  validate_options(opt);
  if (!in_min || !in_max || !out_min || !out_max) throw_input("null bounds");
  if (prec == NNB_FLOAT) {
    auto p = std::make_unique<PlanT3Impl<float>>(dim, opt, sign, batch, stream, alloc);
    p->init(in_min, in_max, out_min, out_max);
    return p;
  }
  auto p = std::make_unique<PlanT3Impl<double>>(dim, opt, sign, batch, stream, alloc);
  p->init(in_min, in_max, out_min, out_max);
  return p;
}

namespace {
template <typename T>
u64 t3_grid_bytes(int dim, const NnbOptions& opt, const double* in_min, const double* in_max,
                  const double* out_min, const double* out_max) {
  const KernelParam kp = kernel_param(opt.tol, opt.upsampfac, is_single<T>(), opt.n_spread);
  u64 spread = 1, fft = 1;
  for (int d = 0; d < dim; ++d) {
    const T3Dim<T> g = t3_geometry<T>(kp.w, opt.upsampfac, T(opt.recenter_threshold),
                                      T(in_min[d]), T(in_max[d]), T(out_min[d]), T(out_max[d]));
    spread *= u64(g.spread_grid);
    fft *= u64(g.fft_grid);
  }
  // Same accounting as the reference GPU plan (src/neonufft/gpu/plan_t3_impl.hpp:69-71):
  // the FFT grid counts twice for the cuFFT work area.
  return sizeof(cplx_t<T>) * (spread + 2 * fft);
}
}  // namespace

u64 t3_grid_memory_size(NnbPrecision prec, int dim, const NnbOptions& opt, const double* in_min,
                        const double* in_max, const double* out_min, const double* out_max) {
  check_dim_prec(prec, dim);
  validate_options(opt);
  if (!in_min || !in_max || !out_min || !out_max) throw_input("null bounds");
  if (prec == NNB_FLOAT) return t3_grid_bytes<float>(dim, opt, in_min, in_max, out_min, out_max);
  return t3_grid_bytes<double>(dim, opt, in_min, in_max, out_min, out_max);
}

}  // namespace nnb
