// Transform options shared by all plans (reference include/neonufft/plan.hpp:19-29).
// The GPU engine ignores num_threads, sort_input, sort_output and kernel_approximation,
// exactly as the reference GPU plan does.
#pragma once

#include <neonufft/enums.h>
#include <neonufft/types.hpp>

namespace neonufft {

struct Options {
  double tol = 0.001;
  double upsampfac = 2.0;
  double recenter_threshold = 0.1;
  int num_threads = 0;
  bool sort_input = true;
  bool sort_output = true;
  bool kernel_approximation = false;
  NeonufftModeOrder order = NEONUFFT_MODE_ORDER_CMCL;
  NeonufftKernelType kernel_type = NEONUFFT_ES_KERNEL;
};

}  // namespace neonufft
