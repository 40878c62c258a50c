// Register-level DFT building blocks shared by the transform passes and the
// adjoint spread's fused x transform (see fftpass.cuh for the scheme): a
// line of L = R1 * R2 points is two register DFT stages with one exchange
// through shared memory.
#pragma once

#include <cstddef>
#include <cstdint>

#include <cuda_runtime.h>

#include "cplx.cuh"
#include "f32x2.cuh"

namespace gnufft
{
namespace fftcore
{
constexpr int kFftThreads = 256;

template <int L> struct Split;
template <> struct Split<16> { static constexpr int R1 = 4, R2 = 4; };
template <> struct Split<32> { static constexpr int R1 = 8, R2 = 4; };
template <> struct Split<64> { static constexpr int R1 = 8, R2 = 8; };
template <> struct Split<128> { static constexpr int R1 = 16, R2 = 8; };
template <> struct Split<256> { static constexpr int R1 = 16, R2 = 16; };
template <> struct Split<512> { static constexpr int R1 = 32, R2 = 16; };
template <> struct Split<1024> { static constexpr int R1 = 32, R2 = 32; };

template <int L> struct Shape
{
  static constexpr int R1 = Split<L>::R1, R2 = Split<L>::R2;
  static constexpr int T = R1 > R2 ? R1 : R2;  // threads per line
  static constexpr int NL = kFftThreads / T;   // lines per block (rows)
  static constexpr int YP = R2 + 1;            // padded exchange row
  static size_t smem() { return (size_t)(L + NL * R1 * YP) * sizeof(float2); }
  // column passes: TC adjacent columns per block, so that every warp moves
  // 32 * 8 bytes (L <= 256) of one row per access
  static constexpr int TC = L <= 256 ? 16 : (L == 512 ? 16 : 8);
  static constexpr int CT = TC * T;            // threads per column block
  static size_t col_smem()
  {
    return (size_t)(L + TC * R1 * YP) * sizeof(float2);
  }
};

// Division of integers 0 <= n < 2^31 by a fixed divisor d >= 1 with one
// wide multiply and a shift: q = (n * m) >> p, m = ceil(2^p / d),
// p = 31 + ceil(log2 d) (the round-up method of Granlund and Montgomery,
// "Division by invariant integers using multiplication", PLDI 1994; exact
// because (m d - 2^p) n < d 2^31 <= 2^p).
struct FastDiv
{
  uint32_t d = 1, m = 1u << 31, p = 31;
  FastDiv() = default;
  __host__ explicit FastDiv(uint32_t div) : d(div)
  {
    uint32_t l = 0;
    while ((1ull << l) < div)
      ++l;
    p = 31 + l;
    m = (uint32_t)(((1ull << p) + div - 1) / div);
  }
  __host__ __device__ uint32_t div(uint32_t n) const
  {
    return (uint32_t)(((uint64_t)n * m) >> p);
  }
};

__host__ __device__ constexpr int bitrev(int i, int R)
{
  int r = 0;
  for (int b = 1; b < R; b <<= 1)
  {
    r = (r << 1) | (i & 1);
    i >>= 1;
  }
  return r;
}


__host__ __device__ constexpr int ilog2(int v)
{
  int r = 0;
  while ((1 << r) < v)
    ++r;
  return r;
}

// In-register radix-2 DIT DFT of R points, natural order in and out.
// w[k] = exp(-2 pi i k / RM), k < RM / 2, RM >= R (conjugated for the
// inverse).  Every loop has a constant trip count and every index is a
// constant, so data and roots stay in registers.
template <int R, int RM, bool INV>
__device__ __forceinline__ void reg_fft(float2 (&a)[R],
                                        const float2 (&w)[RM / 2])
{
#pragma unroll
  for (int i = 0; i < R; ++i)
  {
    const int j = bitrev(i, R);
    if (j > i)
    {
      const float2 t = a[i];
      a[i] = a[j];
      a[j] = t;
    }
  }
  constexpr int LOG = ilog2(R);
#pragma unroll
  for (int st = 0; st < LOG; ++st)
  {
    const int half = 1 << st;
#pragma unroll
    for (int b = 0; b < R / 2; ++b)
    {
      const int k = b & (half - 1);
      const int i0 = ((b >> st) << (st + 1)) + k;
      const int i1 = i0 + half;
      const float2 u = a[i0];
      float2 v = a[i1];
      if (2 * k == half)
      {  // the quarter-turn root -i (+i inverse): exact, no multiply
        v = INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
        a[i0] = make_float2(u.x + v.x, u.y + v.y);
        a[i1] = make_float2(u.x - v.x, u.y - v.y);
      }
      else
      {
        if (k != 0)
        {
          float2 r = w[k * (RM >> (st + 1))];
          if (INV)
            r.y = -r.y;
          v = cmul(v, r);
        }
        a[i0] = add2(u, v);
        a[i1] = sub2(u, v);
      }
    }
  }
}

// Stage 1 of a line (thread lt < R2 holds a[j] = x[lt + R2 j]): R1-point
// DFT, twiddle, store to the line's exchange slots Y[(k1 * YP + lt) * YS]
// (YS: stride between consecutive slots of one line, so that lines can be
// interleaved for conflict-free access).
template <int L> struct Rm
{
  static constexpr int V = Shape<L>::T;  // roots kept for the larger DFT
};

template <int L, bool INV, int YS>
__device__ __forceinline__ void stage1(float2 (&a)[Shape<L>::R1], int lt,
                                       const float2 (&w)[Rm<L>::V / 2],
                                       const float2 *__restrict__ tw,
                                       float2 *__restrict__ Y)
{
  using S = Shape<L>;
  reg_fft<S::R1, Rm<L>::V, INV>(a, w);
#pragma unroll
  for (int k1 = 0; k1 < S::R1; ++k1)
  {
    float2 v = a[k1];
    if (k1 != 0)
    {
      float2 r = tw[(lt * k1) & (L - 1)];
      if (INV)
        r.y = -r.y;
      v = cmul(v, r);
    }
    Y[(k1 * S::YP + lt) * YS] = v;
  }
}

// Stage 2 (thread lt < R1): b[k2] = X[lt + R1 k2].
template <int L, bool INV, int YS>
__device__ __forceinline__ void stage2(float2 (&b)[Shape<L>::R2], int lt,
                                       const float2 (&w)[Rm<L>::V / 2],
                                       const float2 *__restrict__ Y)
{
  using S = Shape<L>;
#pragma unroll
  for (int t = 0; t < S::R2; ++t)
    b[t] = Y[(lt * S::YP + t) * YS];
  reg_fft<S::R2, Rm<L>::V, INV>(b, w);
}

template <int L>
__device__ __forceinline__ void load_reg_roots(float2 (&w)[Rm<L>::V / 2],
                                               const float2 *tw)
{
  constexpr int RM = Rm<L>::V;
#pragma unroll
  for (int k = 0; k < RM / 2; ++k)
    w[k] = tw[k * (L / RM)];
}

__device__ __forceinline__ void load_roots(float2 *tw, const float2 *roots,
                                           int L)
{
  for (int i = threadIdx.x; i < L; i += blockDim.x)
    tw[i] = __ldg(roots + i);
}

}  // namespace fftcore
}  // namespace gnufft
