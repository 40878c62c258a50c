// Bitwise check of the paired FP32 helpers (gpunufft_b200/csrc/f32x2.cuh)
// against the scalar round-to-nearest intrinsics on one GPU: random values
// of every magnitude plus signed zeros, infinities, NaN and subnormals.
// NaN results compare as NaN on both sides.  Prints "failures N".
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include <cuda_runtime.h>

#include "f32x2.cuh"

__global__ void k_check(const float *a, const float *b, const float *c, int n,
                        float *paired, float *scalar)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n / 2;
       i += gridDim.x * blockDim.x)
  {
    const float2 x = make_float2(a[2 * i], a[2 * i + 1]);
    const float2 y = make_float2(b[2 * i], b[2 * i + 1]);
    const float2 z = make_float2(c[2 * i], c[2 * i + 1]);
    const float2 r[4] = {gnufft::add2(x, y), gnufft::sub2(x, y),
                         gnufft::mul2(x, y), gnufft::fma2(x, y, z)};
    for (int o = 0; o < 4; ++o)
    {
      paired[(size_t)o * n + 2 * i] = r[o].x;
      paired[(size_t)o * n + 2 * i + 1] = r[o].y;
    }
    for (int h = 0; h < 2; ++h)
    {
      const int j = 2 * i + h;
      scalar[j] = __fadd_rn(a[j], b[j]);
      scalar[(size_t)n + j] = __fsub_rn(a[j], b[j]);
      scalar[(size_t)2 * n + j] = __fmul_rn(a[j], b[j]);
      scalar[(size_t)3 * n + j] = __fmaf_rn(a[j], b[j], c[j]);
    }
  }
}

int main()
{
  const int n = 1 << 20;
  std::mt19937 rng(7);
  std::uniform_int_distribution<uint32_t> bits;
  std::uniform_real_distribution<float> unit(-1.f, 1.f);
  const float specials[] = {0.f, -0.f, INFINITY, -INFINITY, NAN, 1e-45f,
                            -1e-45f, 1e-38f, 3.4e38f, -3.4e38f, 1.f, -1.f};
  std::vector<float> h[3];
  for (auto &v : h)
  {
    v.resize(n);
    for (int i = 0; i < n; ++i)
    {
      const int kind = i % 4;
      if (kind == 0)
        v[i] = specials[bits(rng) % (sizeof(specials) / sizeof(float))];
      else if (kind == 1)
      {
        const uint32_t u = bits(rng);
        std::memcpy(&v[i], &u, 4);  // any bit pattern
      }
      else
        v[i] = unit(rng) * std::ldexp(1.f, (int)(bits(rng) % 40) - 20);
    }
  }
  float *d[3], *dp, *ds;
  for (int k = 0; k < 3; ++k)
  {
    if (cudaMalloc(&d[k], n * sizeof(float)) != cudaSuccess)
      return 2;
    cudaMemcpy(d[k], h[k].data(), n * sizeof(float), cudaMemcpyHostToDevice);
  }
  if (cudaMalloc(&dp, 4 * (size_t)n * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&ds, 4 * (size_t)n * sizeof(float)) != cudaSuccess)
    return 2;
  k_check<<<256, 256>>>(d[0], d[1], d[2], n, dp, ds);
  std::vector<float> p(4 * (size_t)n), s(4 * (size_t)n);
  cudaMemcpy(p.data(), dp, p.size() * sizeof(float), cudaMemcpyDeviceToHost);
  cudaMemcpy(s.data(), ds, s.size() * sizeof(float), cudaMemcpyDeviceToHost);
  const cudaError_t e = cudaDeviceSynchronize();
  if (e != cudaSuccess)
  {
    std::printf("cuda error %s\n", cudaGetErrorString(e));
    return 2;
  }
  long long failures = 0;
  for (size_t i = 0; i < p.size(); ++i)
  {
    uint32_t up, us;
    std::memcpy(&up, &p[i], 4);
    std::memcpy(&us, &s[i], 4);
    const bool same = up == us || (std::isnan(p[i]) && std::isnan(s[i]));
    if (!same && failures++ < 10)
      std::printf("mismatch op %zu index %zu: %08x vs %08x\n", i / n, i % n,
                  up, us);
  }
  std::printf("checks %zu\nfailures %lld\n", p.size(), failures);
  for (int k = 0; k < 3; ++k)
    cudaFree(d[k]);
  cudaFree(dp);
  cudaFree(ds);
  return failures != 0;
}
