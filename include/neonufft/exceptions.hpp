// Exception hierarchy of the C++ API (reference include/neonufft/exceptions.hpp:16-103).
// The C++ plan classes are thin shims over the C ABI (neonufft_gpu.h); they translate the
// returned NeonufftError into these types. The message points into thread-local storage of
// the library (valid until the next failing call on the same thread) or to a literal.
#pragma once

#include <neonufft/errors.h>

#include <exception>

namespace neonufft {

class GenericError : public std::exception {
public:
  GenericError() : msg_("Neonufft:: Generic error") {}
  GenericError(const char* msg) : msg_(msg) {}
  const char* what() const noexcept override { return msg_; }
  virtual NeonufftError error_code() const noexcept { return NEONUFFT_GENERIC_ERROR; }

private:
  const char* msg_;
};

class InputError : public GenericError {
public:
  InputError() : GenericError("Neonufft:: Input error") {}
  InputError(const char* msg) : GenericError(msg) {}
  NeonufftError error_code() const noexcept override { return NEONUFFT_INPUT_ERROR; }
};

class InternalError : public GenericError {
public:
  InternalError() : GenericError("Neonufft:: Internal error") {}
  InternalError(const char* msg) : GenericError(msg) {}
  NeonufftError error_code() const noexcept override { return NEONUFFT_INTERNAL_ERROR; }
};

class MemoryAllocError : public GenericError {
public:
  MemoryAllocError() : GenericError("Neonufft:: Memory allocation error") {}
  MemoryAllocError(const char* msg) : GenericError(msg) {}
  NeonufftError error_code() const noexcept override { return NEONUFFT_MEMORY_ALLOC_ERROR; }
};

class NotImplementedError : public GenericError {
public:
  NotImplementedError() : GenericError("Neonufft:: Not implemented") {}
  NotImplementedError(const char* msg) : GenericError(msg) {}
  NeonufftError error_code() const noexcept override { return NEONUFFT_NOT_IMPLEMENTED_ERROR; }
};

class GPUError : public GenericError {
public:
  GPUError() : GenericError("Neonufft:: GPU error") {}
  GPUError(const char* msg) : GenericError(msg) {}
  NeonufftError error_code() const noexcept override { return NEONUFFT_GPU_ERROR; }
};

class GPUFFTError : public GenericError {
public:
  GPUFFTError() : GenericError("Neonufft:: GPU FFT error") {}
  GPUFFTError(const char* msg) : GenericError(msg) {}
  NeonufftError error_code() const noexcept override { return NEONUFFT_GPU_ERROR; }
};

}  // namespace neonufft
