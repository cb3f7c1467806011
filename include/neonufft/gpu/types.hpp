// GPU type aliases (reference include/neonufft/gpu/types.hpp:21-33): complex data is
// cuComplex / cuDoubleComplex, streams are cudaStream_t.
#pragma once

#include <cuComplex.h>
#include <cuda_runtime_api.h>

#include <type_traits>

namespace neonufft {
namespace gpu {

using ComplexDoubleType = cuDoubleComplex;
using ComplexFloatType = cuComplex;
using StreamType = cudaStream_t;

template <typename T>
using ComplexType =
    std::conditional_t<std::is_same_v<T, float>, ComplexFloatType, ComplexDoubleType>;

}  // namespace gpu
}  // namespace neonufft
