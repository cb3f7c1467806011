// Default device allocator (reference include/neonufft/gpu/device_allocator.hpp:14-21).
// Header-only: forwards to the engine's C ABI, so user code needs no CUDA runtime link.
#pragma once

#include <neonufft/allocator.hpp>
#include <neonufft_gpu.h>

#include <cstddef>

namespace neonufft {
namespace gpu {

class DeviceAllocator : public Allocator {
public:
  DeviceAllocator() = default;

  void* allocate(std::size_t size) override {
    void* ptr = nullptr;
    if (size && nnb_device_alloc(&ptr, size) != NEONUFFT_SUCCESS) return nullptr;
    return ptr;
  }

  void deallocate(void* ptr) noexcept override {
    if (ptr) (void)nnb_device_free(ptr);
  }
};

}  // namespace gpu
}  // namespace neonufft
