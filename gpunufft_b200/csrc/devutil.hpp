// Small host-side helpers: error propagation and owning device buffers.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

#include <cuda_runtime.h>

namespace gnufft
{

// Thrown inside the library, converted to a gnufft_status at the C ABI.
struct Error : std::runtime_error
{
  int status;
  Error(int s, const std::string &m) : std::runtime_error(m), status(s) {}
};

// Status values mirror gnufft_status in include/gpunufft_b200.h.
enum : int
{
  kOk = 0,
  kInvalidArgument = 1,
  kOutOfMemory = 2,
  kCudaError = 3,
  kCufftError = 4,
  kNotSupported = 5,
  kInternal = 6
};

inline void cuda_check(cudaError_t e, const char *what)
{
  if (e == cudaSuccess)
    return;
  int st = (e == cudaErrorMemoryAllocation) ? kOutOfMemory : kCudaError;
  throw Error(st, std::string(what) + ": " + cudaGetErrorString(e));
}

#define GN_CUDA(call) ::gnufft::cuda_check((call), #call)
#define GN_LAUNCH_CHECK(what) ::gnufft::cuda_check(cudaGetLastError(), what)

// Owning device allocation; move-only.
class DeviceBuffer
{
 public:
  DeviceBuffer() = default;
  explicit DeviceBuffer(size_t bytes) { reset(bytes); }
  ~DeviceBuffer() { release(); }
  DeviceBuffer(const DeviceBuffer &) = delete;
  DeviceBuffer &operator=(const DeviceBuffer &) = delete;
  DeviceBuffer(DeviceBuffer &&o) noexcept : p_(o.p_), n_(o.n_)
  {
    o.p_ = nullptr;
    o.n_ = 0;
  }
  DeviceBuffer &operator=(DeviceBuffer &&o) noexcept
  {
    if (this != &o)
    {
      release();
      p_ = o.p_;
      n_ = o.n_;
      o.p_ = nullptr;
      o.n_ = 0;
    }
    return *this;
  }
  void reset(size_t bytes)
  {
    release();
    if (bytes)
    {
      GN_CUDA(cudaMalloc(&p_, bytes));
      n_ = bytes;
    }
  }
  // grow-only reallocation (contents are not preserved)
  void ensure(size_t bytes)
  {
    if (bytes > n_)
      reset(bytes);
  }
  void release()
  {
    if (p_)
      cudaFree(p_);
    p_ = nullptr;
    n_ = 0;
  }
  template <class T> T *as() const { return static_cast<T *>(p_); }
  void *get() const { return p_; }
  size_t bytes() const { return n_; }

 private:
  void *p_ = nullptr;
  size_t n_ = 0;
};

inline unsigned grid_for(size_t n, unsigned threads, unsigned cap = 1u << 20)
{
  size_t b = (n + threads - 1) / threads;
  if (b == 0)
    b = 1;
  return (unsigned)(b > cap ? cap : b);
}

}  // namespace gnufft
