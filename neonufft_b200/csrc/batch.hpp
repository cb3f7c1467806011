// Batched execution of many independent type-1 / type-2 transforms of uneven sizes.
//
// No counterpart in the reference, which runs one plan at a time on the caller's stream
// (src/neonufft/gpu/plan_impl.hpp:41-152). A Batch owns one plan per transform, each bound to
// one of K internal streams chosen by estimated cost (longest work to the least loaded stream),
// and runs all of them in one of three ways:
//  * serial: one after the other, each waiting for the previous (the baseline);
//  * streams: the K streams run concurrently, forked from and joined back into the batch stream;
//  * graph: the streams' launch sequence is captured once into a CUDA graph (fork / join
//    edges included) and replayed with one cudaGraphLaunch per execution; adding a transform
//    invalidates the graph, which is captured again at the next execution;
//  * fused (and fused graph): as streams (graph), except that the transforms whose plans run
//    the 3D z-window kernels are grouped by (type, kernel width, tile width), and each group's
//    spreading or interpolation step is one persistent launch: as many CTAs as fit on the GPU
//    take work items (a column chunk of one transform, at most 4096 points) from one atomic
//    queue over all the group's transforms, largest transform first. The steps before it (grid
//    clearing, or deconvolution and FFT) and after it (FFT and deconvolution) stay on the
//    transforms' streams; the other transforms run whole on theirs, concurrently.
// Inputs and outputs are fixed at add time: the graph replays the same device pointers, so a
// caller refills the same input buffers between executions.
#pragma once

#include <memory>
#include <vector>

#include "plan.hpp"

namespace nnb {

class Batch {
public:
  Batch(NnbPrecision prec, const NnbOptions& opt, int num_streams, cudaStream_t stream,
        const NnbAllocator* alloc);
  ~Batch();
  Batch(const Batch&) = delete;
  Batch& operator=(const Batch&) = delete;

  // Adds transform `type` (1 or 2) of M points in `dim` dimensions; `opt` overrides the batch
  // options for this transform (null: the batch's). Points are binned now (synchronising the
  // transform's stream). Returns the transform's index.
  i64 add(int dim, int type, int sign, i64 M, const void* const* loc, const i64* modes,
          const void* in, void* out, const i64* strides, const NnbOptions* opt);
  void execute(int mode);
  i64 size() const { return i64(items_.size()); }
  // Plan of transform i (for info and stage timing).
  PlanBase& plan(i64 i);

private:
  struct Item {
    std::unique_ptr<PlanBase> plan;
    int type;
    const void* in;
    void* out;
    i64 strides[3];
    int stream;
  };
  // A persistent launch: transforms of one type whose plans share a fused key. The transforms
  // of one (type, key) are cut, largest first, into up to kFusedParts launches of about equal
  // estimated cost and at least kFusedMinPart transforms, run one after the other on one
  // stream, so that the FFTs of one part's transforms overlap the next part's spreading.
  struct Group {
    int type;
    int key;                    // kernel width | tile width << 8
    std::vector<size_t> items;  // indices into items_, largest estimated cost first
    size_t job_offset;          // bytes into fused_jobs_
    size_t end_offset;          // elements into fused_end_
    i64 total;                  // queue length (sum of the jobs' work-list bounds)
    int stream;                 // index into group_streams_ (shared by a key's parts)
  };
  static constexpr int kFusedParts = 4;
  static constexpr int kFusedMinPart = 4;
  void launch_items(bool serial, cudaStream_t origin);
  void prepare_fused();
  void launch_fused(cudaStream_t origin);
  void release_graph();

  NnbPrecision prec_;
  NnbOptions opt_;
  NnbAllocator alloc_{};
  bool has_alloc_ = false;
  cudaStream_t stream_;
  std::vector<cudaStream_t> streams_;
  cudaStream_t capture_ = nullptr;  // origin stream of the graph capture
  std::vector<double> load_;
  std::vector<cudaEvent_t> events_;  // [0]: fork, [1 + k]: join of stream k, then serial chain
  std::vector<Item> items_;
  std::vector<double> cost_;  // estimated cost of each transform
  cudaGraphExec_t graph_ = nullptr;

  // Persistent execution (fused modes); rebuilt after add().
  std::shared_ptr<DeviceAllocator> dev_alloc_;
  bool fused_ready_ = false;
  std::vector<Group> groups_;
  std::vector<int> item_group_;             // group of each transform, or -1
  std::vector<cudaStream_t> group_streams_;  // one per group
  std::vector<cudaEvent_t> pre_events_;      // per transform: its pre-step is enqueued
  std::vector<cudaEvent_t> group_events_;    // per group: its persistent launch is enqueued
  DevArray<unsigned char> fused_jobs_;
  DevArray<i64> fused_end_;
  DevArray<u32> fused_queue_;
  cudaGraphExec_t fused_graph_ = nullptr;
};

}  // namespace nnb
