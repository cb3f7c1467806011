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
//    invalidates the graph, which is captured again at the next execution.
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
  void launch_items(bool serial, cudaStream_t origin);
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
  cudaGraphExec_t graph_ = nullptr;
};

}  // namespace nnb
