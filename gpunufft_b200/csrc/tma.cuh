// Tensor-memory-access (TMA) helpers shared by the kernels that stage
// tiles in shared memory with bulk tensor copies: tensor-map encoding
// through the driver entry point (no link-time dependency on the driver
// library), and the mbarrier operations of a copy (expect-tx arrival,
// bounded completion wait).  Only plain (non-multicast) copies from this
// GPU's own memory are issued.
#pragma once

#include <cstdint>

#include <cuda.h>
#include <cuda_runtime.h>

namespace gnufft
{
namespace tma
{
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType,
                                  cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle,
                                  CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_fn()
{
  static EncodeTiledFn fn = [] {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f,
                                cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (EncodeTiledFn) nullptr;
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  return fn;
}

// Iterations of a bounded wait for a copy; a copy that has not completed
// by then is reported through the caller's error flag.
constexpr long long kMbarSpin = 1LL << 22;

// Error reporting of the tile copies of one launch: `err` (a mapped host
// flag) is set when a block's wait for a copy gives up after `polls` polls
// (kMbarSpin by default); the waits a block makes before returning, for its
// copies still in flight, always use kMbarSpin.
struct CopyWait
{
  int *err = nullptr;
  long long polls = kMbarSpin;
};

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

// One thread: barriers with an arrival count of one, made visible to the
// async proxy.
__device__ __forceinline__ void mbar_init(uint32_t bar)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void mbar_init_fence()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
      "r"(bytes)
      : "memory");
}

// Orders this thread's generic-proxy shared-memory writes before later
// async-proxy (bulk copy) writes to the same locations; used when a buffer
// that was written in place is refilled by a copy.
__device__ __forceinline__ void fence_proxy_async()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Waits (at most `polls` polls) for the phase with the given parity to
// complete; false if it did not.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar,
                                                  uint32_t parity,
                                                  long long polls = kMbarSpin)
{
  uint32_t done = 0;
  for (long long i = 0; i < polls && !done; ++i)
    asm volatile(
        "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, "
        "[%1], %2; selp.u32 %0, 1, 0, p; }"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
  return done != 0;
}

// Bulk tensor copies global -> shared, completion counted on `bar`.  The
// innermost coordinate times the element size must be a multiple of 16
// bytes (callers start tiles on such columns).
__device__ __forceinline__ void copy_2d(uint32_t dst, const void *tmap,
                                        int x, int y, uint32_t bar)
{
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::"
      "complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void copy_3d(uint32_t dst, const void *tmap,
                                        int x, int y, int z, uint32_t bar)
{
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::"
      "complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(z),
      "r"(bar)
      : "memory");
}

__device__ __forceinline__ void copy_4d(uint32_t dst, const void *tmap,
                                        int x, int y, int z, int w,
                                        uint32_t bar)
{
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::"
      "complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(z), "r"(w),
      "r"(bar)
      : "memory");
}

// Untiled bulk copy global -> shared of `bytes` bytes (both addresses
// 16-byte aligned, bytes a multiple of 16), completion counted on `bar`.
__device__ __forceinline__ void copy_bulk(uint32_t dst, const void *src,
                                          uint32_t bytes, uint32_t bar)
{
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
      "[%0], [%1], %2, [%3];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(bar)
      : "memory");
}

}  // namespace tma
}  // namespace gnufft
