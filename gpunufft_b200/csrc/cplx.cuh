// Complex products with a fixed rounding: each part is one rounded product
// and one fused multiply-add, written out with the round-to-nearest
// intrinsics, so that the compiler's choice of which product to fuse
// cannot differ between kernels (or inlined call sites) and every kernel
// that computes the same product gets the same bits.
#pragma once

#include <cuda_runtime.h>

namespace gnufft
{

// a * b
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
  return make_float2(__fmaf_rn(a.x, b.x, -__fmul_rn(a.y, b.y)),
                     __fmaf_rn(a.x, b.y, __fmul_rn(a.y, b.x)));
}

// conj(s) * v
__device__ __forceinline__ float2 cmul_conj(float2 v, float2 s)
{
  return make_float2(__fmaf_rn(v.x, s.x, __fmul_rn(v.y, s.y)),
                     __fmaf_rn(v.y, s.x, -__fmul_rn(v.x, s.y)));
}

}  // namespace gnufft
