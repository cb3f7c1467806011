// Allocator interface used by the plans for every device buffer they own
// (reference include/neonufft/allocator.hpp:12-21).
#pragma once

#include <cstddef>

namespace neonufft {

class Allocator {
public:
  Allocator() = default;
  virtual ~Allocator() = default;
  virtual void* allocate(std::size_t size) = 0;
  virtual void deallocate(void* ptr) noexcept = 0;
};

}  // namespace neonufft
