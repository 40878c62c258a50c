// Helpers of the C entry points: exceptions to statuses, the plan's device
// made current for the duration of a call, cuFFT results to exceptions.
#pragma once

#include <new>
#include <stdexcept>
#include <string>

#include <cufft.h>
#include <cuda_runtime.h>

#include "../../include/gpunufft_b200.h"
#include "devutil.hpp"
#include "planview.hpp"

namespace gnufft
{
inline int fail(int st, const std::string &msg)
{
  set_last_error(msg);
  return st;
}

// Runs f(); an exception becomes the status it carries (and the thread's
// last error message).  Nothing escapes across the C ABI.
template <class F> gnufft_status guarded(F &&f)
{
  try
  {
    f();
    return GNUFFT_SUCCESS;
  }
  catch (const Error &e)
  {
    set_last_error(e.what());
    return (gnufft_status)e.status;
  }
  catch (const std::bad_alloc &)
  {
    set_last_error("host allocation failed");
    return GNUFFT_ERROR_OUT_OF_MEMORY;
  }
  catch (const std::exception &e)
  {
    set_last_error(e.what());
    return GNUFFT_ERROR_INTERNAL;
  }
}

struct DeviceGuard
{
  int prev = -1;
  explicit DeviceGuard(int dev)
  {
    cudaGetDevice(&prev);
    GN_CUDA(cudaSetDevice(dev));
  }
  ~DeviceGuard()
  {
    if (prev >= 0)
      cudaSetDevice(prev);
  }
};

inline void check_cufft(cufftResult r, const char *what)
{
  if (r != CUFFT_SUCCESS)
    throw Error(r == CUFFT_ALLOC_FAILED ? kOutOfMemory : kCufftError,
                std::string(what) + ": cuFFT error " + std::to_string((int)r));
}
}  // namespace gnufft
