// Two-lane FP32 arithmetic: one sm_100 paired instruction per float2
// operation.  Each lane rounds to nearest exactly like the scalar
// operation (add, sub, mul, and fma with a single rounding), so results are
// identical to the scalar code they replace.
#pragma once

#include <cuda_runtime.h>

namespace gnufft
{

#define GNUFFT_F32X2_BINARY(name, op)                                        \
  __device__ __forceinline__ float2 name(float2 a, float2 b)                 \
  {                                                                          \
    float2 r;                                                                \
    asm("{\n\t.reg .b64 pa, pb, pd;\n\t"                                     \
        "mov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t" op              \
        " pd, pa, pb;\n\tmov.b64 {%0, %1}, pd;\n\t}"                         \
        : "=f"(r.x), "=f"(r.y)                                               \
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                           \
    return r;                                                                \
  }

GNUFFT_F32X2_BINARY(add2, "add.rn.f32x2")
GNUFFT_F32X2_BINARY(sub2, "sub.rn.f32x2")
GNUFFT_F32X2_BINARY(mul2, "mul.rn.f32x2")
#undef GNUFFT_F32X2_BINARY

// a * b + c per lane, one rounding.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c)
{
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pc, pd;\n\t"
      "mov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "mov.b64 pc, {%6, %7};\n\t"
      "fma.rn.f32x2 pd, pa, pb, pc;\n\tmov.b64 {%0, %1}, pd;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
  return r;
}

}  // namespace gnufft
