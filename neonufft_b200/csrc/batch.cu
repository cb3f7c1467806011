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

// Persistent-step job records of precision T (ZSpreadJob<T> for type 1, ZInterpJob<T> for 2).
template <typename T>
size_t job_bytes(int type) {
  return type == 1 ? sizeof(ZSpreadJob<T>) : sizeof(ZInterpJob<T>);
}
template <typename T>
i64 job_items(int type, const unsigned char* job) {
  return type == 1 ? reinterpret_cast<const ZSpreadJob<T>*>(job)->wl.grid
                   : reinterpret_cast<const ZInterpJob<T>*>(job)->wl.grid;
}
template <typename T>
void launch_group(int type, const unsigned char* jobs, const i64* end, int njobs, i64 total,
                  int w, int tile_x, u32* queue, cudaStream_t s) {
  if (type == 1) {
    launch_spread_zwin_fused<T>(reinterpret_cast<const ZSpreadJob<T>*>(jobs), end, njobs, total,
                                w, tile_x, queue, s);
  } else {
    launch_interp_zwin_fused<T>(reinterpret_cast<const ZInterpJob<T>*>(jobs), end, njobs, total,
                                w, tile_x, queue, s);
  }
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
  dev_alloc_ = std::make_shared<DeviceAllocator>(has_alloc_ ? &alloc_ : nullptr);
  fused_jobs_.set_allocator(dev_alloc_);
  fused_end_.set_allocator(dev_alloc_);
  fused_queue_.set_allocator(dev_alloc_);
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
  for (auto s : group_streams_) cudaStreamSynchronize(s);
  release_graph();
  items_.clear();  // plans free their memory on their (idle) streams
  for (auto e : events_) cudaEventDestroy(e);
  for (auto e : pre_events_) cudaEventDestroy(e);
  for (auto e : group_events_) cudaEventDestroy(e);
  for (auto s : streams_) cudaStreamDestroy(s);
  for (auto s : group_streams_) cudaStreamDestroy(s);
  cudaStreamDestroy(capture_);
}

void Batch::release_graph() {
  if (graph_) {
    cudaGraphExecDestroy(graph_);
    graph_ = nullptr;
  }
  if (fused_graph_) {
    cudaGraphExecDestroy(fused_graph_);
    fused_graph_ = nullptr;
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
  cost_.push_back(cost);
  while (events_.size() < 1 + streams_.size() + items_.size()) events_.push_back(new_event());
  release_graph();
  fused_ready_ = false;
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

void Batch::prepare_fused() {
  if (fused_ready_) return;
  // A previous execution may still read the job records about to be rewritten.
  for (auto s : streams_) NNB_CUDA(cudaStreamSynchronize(s));
  for (auto s : group_streams_) NNB_CUDA(cudaStreamSynchronize(s));
  groups_.clear();
  item_group_.assign(items_.size(), -1);
  // Transforms by (type, key), largest first.
  std::vector<Group> keys;
  for (size_t i = 0; i < items_.size(); ++i) {
    int key = 0;
    if (!items_[i].plan->fused_key(&key)) continue;
    int g = -1;
    for (size_t j = 0; j < keys.size(); ++j) {
      if (keys[j].type == items_[i].type && keys[j].key == key) g = int(j);
    }
    if (g < 0) {
      Group grp{};
      grp.type = items_[i].type;
      grp.key = key;
      keys.push_back(grp);
      g = int(keys.size()) - 1;
    }
    keys[size_t(g)].items.push_back(i);
  }
  // Parts of about equal cost: a part closes once it holds its share of the key's cost.
  for (size_t k = 0; k < keys.size(); ++k) {
    Group& kg = keys[k];
    std::stable_sort(kg.items.begin(), kg.items.end(),
                     [&](size_t a, size_t b) { return cost_[a] > cost_[b]; });
    double sum = 0.0;
    for (size_t i : kg.items) sum += cost_[i];
    const int parts = int(std::min<size_t>(
        kFusedParts, (kg.items.size() + kFusedMinPart - 1) / kFusedMinPart));
    const double share = sum / parts;
    Group part{};
    part.type = kg.type;
    part.key = kg.key;
    part.stream = int(k);
    double acc = 0.0;
    int made = 0;
    for (size_t n = 0; n < kg.items.size(); ++n) {
      const size_t i = kg.items[n];
      part.items.push_back(i);
      item_group_[i] = int(groups_.size());
      acc += cost_[i];
      const bool last = n + 1 == kg.items.size();
      if (last || (acc >= share && made + 1 < parts)) {
        groups_.push_back(part);
        part.items.clear();
        acc = 0.0;
        ++made;
      }
    }
  }
  // Job records of every part and the parts' cumulative item counts.
  const bool single = prec_ == NNB_FLOAT;
  std::vector<unsigned char> jobs;
  std::vector<i64> ends;
  for (Group& grp : groups_) {
    const size_t jb = single ? job_bytes<float>(grp.type) : job_bytes<double>(grp.type);
    grp.job_offset = jobs.size();
    grp.end_offset = ends.size();
    grp.total = 0;
    for (size_t i : grp.items) {
      const Item& it = items_[i];
      const size_t off = jobs.size();
      jobs.resize(off + jb);
      it.plan->fused_job(it.type, it.in, it.out, jobs.data() + off);
      grp.total += single ? job_items<float>(grp.type, jobs.data() + off)
                          : job_items<double>(grp.type, jobs.data() + off);
      ends.push_back(grp.total);
    }
    if (grp.total > 0x7fffffffll) throw_input("too many work items for one persistent launch");
  }
  if (!groups_.empty()) {
    fused_jobs_.reserve(jobs.size());
    fused_end_.reserve(ends.size());
    fused_queue_.reserve(groups_.size());
    NNB_CUDA(cudaMemcpy(fused_jobs_.data(), jobs.data(), jobs.size(), cudaMemcpyHostToDevice));
    NNB_CUDA(cudaMemcpy(fused_end_.data(), ends.data(), ends.size() * sizeof(i64),
                        cudaMemcpyHostToDevice));
  }
  while (group_streams_.size() < keys.size()) {
    cudaStream_t s = nullptr;
    NNB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    group_streams_.push_back(s);
  }
  while (group_events_.size() < groups_.size()) group_events_.push_back(new_event());
  while (pre_events_.size() < items_.size()) pre_events_.push_back(new_event());
  fused_ready_ = true;
}

void Batch::launch_fused(cudaStream_t origin) {
  const size_t K = streams_.size();
  NNB_CUDA(cudaEventRecord(events_[0], origin));
  for (size_t k = 0; k < K; ++k) NNB_CUDA(cudaStreamWaitEvent(streams_[k], events_[0], 0));
  // Pre-steps of the grouped transforms, whole transforms for the others.
  for (size_t i = 0; i < items_.size(); ++i) {
    Item& it = items_[i];
    if (item_group_[i] >= 0) {
      it.plan->fused_pre(it.type, it.in, it.strides);
      NNB_CUDA(cudaEventRecord(pre_events_[i], streams_[size_t(it.stream)]));
    } else if (it.type == 1) {
      it.plan->transform_type_1(it.in, it.out, it.strides);
    } else {
      it.plan->transform_type_2(it.in, it.strides, it.out);
    }
  }
  // One persistent launch per group, then the type-1 post-steps on the transforms' streams.
  const bool single = prec_ == NNB_FLOAT;
  for (size_t g = 0; g < groups_.size(); ++g) {
    const Group& grp = groups_[g];
    cudaStream_t gs = group_streams_[size_t(grp.stream)];
    for (size_t i : grp.items) NNB_CUDA(cudaStreamWaitEvent(gs, pre_events_[i], 0));
    u32* queue = fused_queue_.data() + g;
    NNB_CUDA(cudaMemsetAsync(queue, 0, sizeof(u32), gs));
    const unsigned char* jobs = fused_jobs_.data() + grp.job_offset;
    const i64* end = fused_end_.data() + grp.end_offset;
    const int w = grp.key & 0xFF, tile_x = grp.key >> 8;
    if (single) {
      launch_group<float>(grp.type, jobs, end, int(grp.items.size()), grp.total, w, tile_x, queue,
                          gs);
    } else {
      launch_group<double>(grp.type, jobs, end, int(grp.items.size()), grp.total, w, tile_x,
                           queue, gs);
    }
    NNB_CUDA(cudaEventRecord(group_events_[g], gs));
    for (size_t i : grp.items) {
      Item& it = items_[i];
      if (it.type != 1) continue;
      NNB_CUDA(cudaStreamWaitEvent(streams_[size_t(it.stream)], group_events_[g], 0));
      it.plan->fused_post(1, it.out, it.strides);
    }
  }
  for (size_t k = 0; k < K; ++k) {
    NNB_CUDA(cudaEventRecord(events_[1 + k], streams_[k]));
    NNB_CUDA(cudaStreamWaitEvent(origin, events_[1 + k], 0));
  }
  for (size_t g = 0; g < groups_.size(); ++g) {
    NNB_CUDA(cudaStreamWaitEvent(origin, group_events_[g], 0));
  }
}

void Batch::execute(int mode) {
  if (mode < NNB_BATCH_SERIAL || mode > NNB_BATCH_FUSED_GRAPH) throw_input("invalid batch mode");
  if (items_.empty()) return;
  const bool fused = mode == NNB_BATCH_FUSED || mode == NNB_BATCH_FUSED_GRAPH;
  if (fused) prepare_fused();
  if (mode == NNB_BATCH_SERIAL || mode == NNB_BATCH_STREAMS) {
    launch_items(mode == NNB_BATCH_SERIAL, stream_);
    return;
  }
  if (mode == NNB_BATCH_FUSED) {
    launch_fused(stream_);
    return;
  }
  cudaGraphExec_t& exec = fused ? fused_graph_ : graph_;
  if (!exec) {
    for (auto& it : items_) {
      if (it.plan->timer().enabled()) throw_input("stage timing cannot be captured in a graph");
    }
    cudaGraph_t g = nullptr;
    // Captured on an internal stream (the caller's stream may be the legacy default stream,
    // which cannot be captured); the graph is then launched on the caller's stream.
    NNB_CUDA(cudaStreamBeginCapture(capture_, cudaStreamCaptureModeThreadLocal));
    try {
      if (fused) {
        launch_fused(capture_);
      } else {
        launch_items(false, capture_);
      }
    } catch (...) {
      cudaStreamEndCapture(capture_, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    NNB_CUDA(cudaStreamEndCapture(capture_, &g));
    const cudaError_t err = cudaGraphInstantiate(&exec, g, 0);
    cudaGraphDestroy(g);
    if (err != cudaSuccess) {
      exec = nullptr;
      throw_gpu(err, "cudaGraphInstantiate", __FILE__, __LINE__);
    }
  }
  NNB_CUDA(cudaGraphLaunch(exec, stream_));
}

}  // namespace nnb
