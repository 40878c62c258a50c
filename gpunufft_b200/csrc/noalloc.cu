// gnufft_adjoint_convolution_noalloc: the adjoint up to the CONVOLUTION
// stage (raw oversampled grid per coil) without allocating device memory.
//
// Who needs it: callers that must not call cudaMalloc / cudaFree while they
// run -- real-time reconstruction loops and serving workers that reserve all
// device memory up front, code that runs with a fixed memory budget owned by
// another framework, and callers that cannot afford the implicit device
// synchronisation an allocation or free causes.  The regular entry points
// grow the plan's scratch buffers on first use; this one never does.
//
// The only scratch is the sorted, coil-interleaved copy of the k-space
// (samples x coil lanes), which lives in the fixed array below.  Every GPU
// that loads this library holds it until the process exits.
#include <cstdint>
#include <exception>
#include <string>

#include <cuda_runtime.h>

#include "../../include/gpunufft_b200.h"
#include "devutil.hpp"
#include "gridding.cuh"
#include "planview.hpp"

namespace
{
constexpr size_t kScratchBytes = GNUFFT_NOALLOC_SCRATCH_BYTES;
constexpr size_t kScratchElems = kScratchBytes / sizeof(float2);

// Shared by every call on a device; keeps the contents of the last call.
static __device__ __align__(256) float2 g_noalloc_ks[kScratchElems];

// Device address of g_noalloc_ks on the current device.  In host code the
// array's name is only a host-side stand-in; the address comes from
// cudaGetSymbolAddress with the device current, looked up on every call
// (cheap once the module is loaded; a cached address would go stale after
// the context is torn down and recreated).
float2 *scratch_address()
{
  void *ptr = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_ks);
  if (e != cudaSuccess || !ptr)
    throw gnufft::Error(gnufft::kCudaError,
                        std::string("cudaGetSymbolAddress(no-allocation "
                                    "scratch): ") +
                            cudaGetErrorString(e));
  return static_cast<float2 *>(ptr);
}
}  // namespace

extern "C" gnufft_status gnufft_adjoint_convolution_noalloc(gnufft_plan *plan,
                                                            const void *kspace,
                                                            void *grid,
                                                            uint32_t n_coils,
                                                            void *stream)
{
  using namespace gnufft;
  int prev = -1;
  gnufft_status st = GNUFFT_SUCCESS;
  try
  {
    PlanView v;
    if (!plan_view(plan, &v) || !kspace || !grid)
      throw Error(kInvalidArgument, "NULL argument");
    if (n_coils == 0 || (v.sens_coils && n_coils != v.sens_coils))
      throw Error(kInvalidArgument,
                  "n_coils must be positive and match the sensitivity maps");
    const int cg = spmm_coil_group((int)n_coils);
    const size_t CP = ((size_t)n_coils + cg - 1) / cg * cg;
    const size_t need = (size_t)v.M * CP;
    if (need > kScratchElems)
      throw Error(kInvalidArgument,
                  "no-allocation adjoint: samples x coil lanes (" +
                      std::to_string(v.M) + " x " + std::to_string(CP) +
                      " = " + std::to_string(need * sizeof(float2)) +
                      " bytes) exceed the fixed " +
                      std::to_string(kScratchBytes) +
                      "-byte staging area");
    cudaGetDevice(&prev);
    GN_CUDA(cudaSetDevice(v.device));
    float2 *ks = scratch_address();
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // Every one of the M x CP staged entries is written (coil lanes beyond
    // n_coils as zeros), so nothing left from an earlier call is read.
    launch_gather_kspace(static_cast<const float2 *>(kspace), v.data_indices,
                         v.dens_sorted, v.M, (int)n_coils, (int)CP, ks, s);
    launch_adjoint_spmm(v.w_rows, v.w_nz, ks, (int)CP, v.g, (int)n_coils,
                        false, static_cast<float2 *>(grid), s);
  }
  catch (const Error &e)
  {
    set_last_error(e.what());
    st = (gnufft_status)e.status;
  }
  catch (const std::exception &e)
  {
    set_last_error(e.what());
    st = GNUFFT_ERROR_INTERNAL;
  }
  if (prev >= 0)
    cudaSetDevice(prev);
  return st;
}
