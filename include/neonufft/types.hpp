// Integer type used for sizes, counts and strides (reference include/neonufft/types.hpp:9).
#pragma once

#include <cstdint>

namespace neonufft {
using IntType = std::int64_t;
}  // namespace neonufft
