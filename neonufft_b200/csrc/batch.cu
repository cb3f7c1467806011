// Batched execution of many independent transforms (see batch.hpp).
#include <algorithm>
#include <cmath>

#include "batch.hpp"
#include "params.hpp"

namespace nnb {

namespace {

cudaEvent_t new_event() {
  cudaEvent_t e = nullptr;
  NNB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  return e;
}

}  // namespace

Batch::Batch(NnbPrecision prec, const NnbOptions& opt, int num_streams, cudaStream_t stream,
             const NnbAllocator* alloc)
    : prec_(prec), opt_(opt), stream_(stream) {
  validate_options(opt);
  if (prec != NNB_FLOAT && prec != NNB_DOUBLE) throw_input("invalid precision");
  if (num_streams < 1 || num_streams > 64) throw_input("number of streams must be in [1, 64]");
  if (alloc) {
    alloc_ = *alloc;
    has_alloc_ = true;
  }
  streams_.assign(size_t(num_streams), nullptr);
  load_.assign(size_t(num_streams), 0.0);
  try {
    for (auto& s : streams_) NNB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    NNB_CUDA(cudaStreamCreateWithFlags(&capture_, cudaStreamNonBlocking));
    events_.push_back(new_event());
    for (int k = 0; k < num_streams; ++k) events_.push_back(new_event());
  } catch (...) {
    for (auto s : streams_) {
      if (s) cudaStreamDestroy(s);
    }
    if (capture_) cudaStreamDestroy(capture_);
    for (auto e : events_) cudaEventDestroy(e);
    throw;
  }
}

Batch::~Batch() {
  for (auto s : streams_) cudaStreamSynchronize(s);
  release_graph();
  items_.clear();  // plans free their memory on their (idle) streams
  for (auto e : events_) cudaEventDestroy(e);
  for (auto s : streams_) cudaStreamDestroy(s);
  cudaStreamDestroy(capture_);
}

void Batch::release_graph() {
  if (graph_) {
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
}

i64 Batch::add(int dim, int type, int sign, i64 M, const void* const* loc, const i64* modes,
               const void* in, void* out, const i64* strides, const NnbOptions* opt) {
  if (type != 1 && type != 2) throw_input("batched transforms are of type 1 or 2");
  if (dim < 1 || dim > 3) throw_input("invalid dimension");
  if (!modes || !strides) throw_input("null modes or strides");
  if (!out || (M > 0 && !in && type == 1) || (type == 2 && !in)) {
    throw_input("null input or output");
  }
  const NnbOptions o = opt ? *opt : opt_;
  validate_options(o);
  // Estimated cost: spreading work M w^d plus an FFT of the fine grid.
  const KernelParam kp = kernel_param(o.tol, o.upsampfac, prec_ == NNB_FLOAT, o.n_spread);
  double cells = 1.0, work = double(M);
  for (int d = 0; d < dim; ++d) {
    cells *= double(fine_grid_size(modes[d], o.upsampfac, kp.w));
    work *= double(kp.w);
  }
  const double cost = work + 5.0 * cells * std::log2(std::max(2.0, cells));
  const int k = int(std::min_element(load_.begin(), load_.end()) - load_.begin());
  load_[size_t(k)] += cost;

  Item it;
  it.plan = make_plan(prec_, dim, o, sign, M, loc, modes, streams_[size_t(k)],
                      has_alloc_ ? &alloc_ : nullptr);
  it.type = type;
  it.in = in;
  it.out = out;
  for (int d = 0; d < 3; ++d) it.strides[d] = d < dim ? strides[d] : 1;
  it.stream = k;
  items_.push_back(std::move(it));
  while (events_.size() < 1 + streams_.size() + items_.size()) events_.push_back(new_event());
  release_graph();
  return i64(items_.size()) - 1;
}

PlanBase& Batch::plan(i64 i) {
  if (i < 0 || i >= size()) throw_input("batch index out of range");
  return *items_[size_t(i)].plan;
}

void Batch::launch_items(bool serial, cudaStream_t origin) {
  const size_t K = streams_.size();
  NNB_CUDA(cudaEventRecord(events_[0], origin));
  if (serial) {
    cudaEvent_t prev = events_[0];
    for (size_t i = 0; i < items_.size(); ++i) {
      Item& it = items_[i];
      cudaStream_t s = streams_[size_t(it.stream)];
      NNB_CUDA(cudaStreamWaitEvent(s, prev, 0));
      if (it.type == 1) {
        it.plan->transform_type_1(it.in, it.out, it.strides);
      } else {
        it.plan->transform_type_2(it.in, it.strides, it.out);
      }
      prev = events_[1 + K + i];
      NNB_CUDA(cudaEventRecord(prev, s));
    }
    NNB_CUDA(cudaStreamWaitEvent(origin, prev, 0));
    return;
  }
  for (size_t k = 0; k < K; ++k) NNB_CUDA(cudaStreamWaitEvent(streams_[k], events_[0], 0));
  for (Item& it : items_) {
    if (it.type == 1) {
      it.plan->transform_type_1(it.in, it.out, it.strides);
    } else {
      it.plan->transform_type_2(it.in, it.strides, it.out);
    }
  }
  for (size_t k = 0; k < K; ++k) {
    NNB_CUDA(cudaEventRecord(events_[1 + k], streams_[k]));
    NNB_CUDA(cudaStreamWaitEvent(origin, events_[1 + k], 0));
  }
}

void Batch::execute(int mode) {
  if (mode < NNB_BATCH_SERIAL || mode > NNB_BATCH_GRAPH) throw_input("invalid batch mode");
  if (items_.empty()) return;
  if (mode != NNB_BATCH_GRAPH) {
    launch_items(mode == NNB_BATCH_SERIAL, stream_);
    return;
  }
  if (!graph_) {
    for (auto& it : items_) {
      if (it.plan->timer().enabled()) throw_input("stage timing cannot be captured in a graph");
    }
    cudaGraph_t g = nullptr;
    // Captured on an internal stream (the caller's stream may be the legacy default stream,
    // which cannot be captured); the graph is then launched on the caller's stream.
    NNB_CUDA(cudaStreamBeginCapture(capture_, cudaStreamCaptureModeThreadLocal));
    try {
      launch_items(false, capture_);
    } catch (...) {
      cudaStreamEndCapture(capture_, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    NNB_CUDA(cudaStreamEndCapture(capture_, &g));
    const cudaError_t err = cudaGraphInstantiate(&graph_, g, 0);
    cudaGraphDestroy(g);
    if (err != cudaSuccess) {
      graph_ = nullptr;
      throw_gpu(err, "cudaGraphInstantiate", __FILE__, __LINE__);
    }
  }
  NNB_CUDA(cudaGraphLaunch(graph_, stream_));
}

}  // namespace nnb
