// Trajectory gradient of the forward operator (no upstream counterpart).
//
// The forward operator samples the oversampled spectrum H = FFT(pad(deapo *
// S_c * x)) with the separable Kaiser-Bessel kernel:
//   y[c][j] = s * sqrt(w_j) * sum_cells psi(d_x) psi(d_y) psi(d_z) H_c(cell),
//   d_a = (kcell_a - k_a[j]) * aniso_a,
// so its derivative with respect to a sample coordinate k_a[j] replaces
// psi(d_a) by dpsi/dk_a = psi'(d_a) * (-aniso_a) on that axis.  For a real
// loss L with dL/dy given as u (torch's convention: dL/dRe + i dL/dIm),
//   dL/dk_a[j] = sum_c Re( conj(u[c][j]) * dy[c][j]/dk_a[j] ).
// The same kernel serves the adjoint operator: for x = A^H y and dL/dx = v,
//   dL/dk_a[j] = sum_c Re( conj(y[c][j]) * d(A v)[c][j]/dk_a[j] ).
//
// psi is the kernel of the lookup table, KB(r) = I0(beta sqrt(1 - r^2)) /
// I0(beta), r = |d| / R.  Its derivative is tabulated as a function of d^2:
//   dpsi/dk = beta I1(beta s) / (s I0(beta) R^2) * d * aniso,
//   s = sqrt(1 - d^2 / R^2),
// (I1(beta s) / s -> beta / 2 as s -> 0), linearly interpolated.  Cell
// selection and the kernel values are exactly those of the forward
// interpolation (axis_footprint).
#include <cmath>
#include <vector>

#include "devutil.hpp"
#include "footprint.cuh"
#include "trajgrad.cuh"

namespace gnufft
{
namespace
{
constexpr int kGradThreads = 256;

__device__ __forceinline__ float deriv_lookup(const float *__restrict__ tab,
                                              int len, float mult, float d2)
{
  const float x = d2 * mult;
  int i = (int)x;
  if (i < 0)
    i = 0;
  if (i > len - 2)
    i = len - 2;
  const float f = fminf(fmaxf(x - (float)i, 0.f), 1.f);
  const float a = __ldg(tab + i), b = __ldg(tab + i + 1);
  return fmaf(f, b - a, a);
}

template <int DIM>
__global__ void __launch_bounds__(kGradThreads)
    k_traj_grad(const float *__restrict__ traj,
                const uint32_t *__restrict__ sec_sorted,
                const uint32_t *__restrict__ idx,
                const float *__restrict__ dens,
                const float2 *__restrict__ grid, Geo g,
                const float *__restrict__ lut,
                const float *__restrict__ dtab, int dlen, float dmult,
                uint32_t M, int C, float scale,
                const float2 *__restrict__ u, float *__restrict__ out)
{
  const int lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
       t < M; t += nwarps)
  {
    int sa[3];
    {
      const int s = (int)sec_sorted[t];
      sa[0] = s % g.S[0];
      const int r = s / g.S[0];
      sa[1] = r % g.S[1];
      sa[2] = r / g.S[1];
    }
    int cell[3][kSlots];
    float w[3][kSlots], dw[3][kSlots];
    int n[3] = {1, 1, 1};
    cell[2][0] = 0;
    w[2][0] = 1.f;
    dw[2][0] = 0.f;
#pragma unroll
    for (int a = 0; a < DIM; ++a)
    {
      const float c = traj[(size_t)a * M + t];
      int loc[kSlots];
      n[a] = axis_footprint(c, a, sa[a], g, lut, cell[a], w[a], loc);
      const int center = sa[a] * g.sw + (g.sw >> 1);
      for (int e = 0; e < n[a]; ++e)
      {
        const int gc = loc[e] + center - g.offset;
        const float k = __fsub_rn(grid_to_k(gc, a, g), 0.5f);
        const float d = __fmul_rn(__fsub_rn(k, c), g.aniso[a]);
        const float d2 = __fmul_rn(d, d);
        dw[a][e] = d2 < g.radius_sq
                       ? deriv_lookup(dtab, dlen, dmult, d2) * d * g.aniso[a]
                       : 0.f;
        // the FORWARD fftshift: the value of cell gw sits at gw + ceil(G/2)
        int q = cell[a][e] + g.shift_fwd[a];
        if (q >= g.G[a])
          q -= g.G[a];
        cell[a][e] = q;
      }
    }
    const uint32_t j = idx[t];
    float acc[3] = {0.f, 0.f, 0.f};
    for (int c = lane; c < C; c += 32)
    {
      const float2 *gc = grid + (long long)c * g.grid_count;
      float2 s[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f),
                     make_float2(0.f, 0.f)};
      for (int z = 0; z < n[2]; ++z)
      {
        const long long oz =
            DIM == 3 ? (long long)cell[2][z] * g.G[1] * g.G[0] : 0;
        const float wz = w[2][z], dwz = dw[2][z];
        for (int y = 0; y < n[1]; ++y)
        {
          const long long oy = oz + (long long)cell[1][y] * g.G[0];
          const float wy = w[1][y], dwy = dw[1][y];
          for (int x = 0; x < n[0]; ++x)
          {
            const float2 v = __ldg(gc + oy + cell[0][x]);
            const float fx = dw[0][x] * wy * wz;
            const float fy = w[0][x] * dwy * wz;
            s[0].x = fmaf(fx, v.x, s[0].x);
            s[0].y = fmaf(fx, v.y, s[0].y);
            s[1].x = fmaf(fy, v.x, s[1].x);
            s[1].y = fmaf(fy, v.y, s[1].y);
            if (DIM == 3)
            {
              const float fz = w[0][x] * wy * dwz;
              s[2].x = fmaf(fz, v.x, s[2].x);
              s[2].y = fmaf(fz, v.y, s[2].y);
            }
          }
        }
      }
      const float2 uu = u[(long long)c * M + j];
#pragma unroll
      for (int a = 0; a < DIM; ++a)
        acc[a] += uu.x * s[a].x + uu.y * s[a].y;
    }
#pragma unroll
    for (int a = 0; a < DIM; ++a)
      for (int o = 16; o > 0; o >>= 1)
        acc[a] += __shfl_xor_sync(0xffffffffu, acc[a], o);
    if (lane == 0)
    {
      const float f = dens ? scale * sqrtf(dens[t]) : scale;
#pragma unroll
      for (int a = 0; a < DIM; ++a)
        out[(size_t)a * M + j] = acc[a] * f;
    }
  }
}

double bessel_i(int order, double x) { return std::cyl_bessel_i((double)order, x); }
}  // namespace

void deriv_lut_fill(const Geo &g, float osf, int n, std::vector<float> &tab,
                    float &mult)
{
  const double kw = (double)g.kw;
  const double t = kw / (double)osf * ((double)osf - 0.5);
  const double beta = M_PI * std::sqrt(std::max(t * t - 0.8, 0.0));
  const double R2 = (double)g.radius_sq;
  const double i0b = bessel_i(0, beta);
  tab.assign(n, 0.f);
  for (int i = 0; i < n; ++i)
  {
    const double r2 = (double)i / (double)(n - 1);
    const double s = std::sqrt(std::max(1.0 - r2, 0.0));
    const double ratio = s > 1e-12 ? bessel_i(1, beta * s) / s : 0.5 * beta;
    tab[i] = (float)(beta * ratio / (i0b * R2));
  }
  mult = (float)((double)(n - 1) / R2);
}

void launch_traj_grad(const float *traj_sorted, const uint32_t *sec_sorted,
                      const uint32_t *idx, const float *dens_sorted,
                      const float2 *grid, const Geo &g, const float *lut,
                      const float *dtab, int dlen, float dmult, uint32_t M,
                      int C, float scale, const float2 *u, float *out,
                      cudaStream_t s)
{
  if (!M)
    return;
  const long long warps = (long long)M;
  const int per_block = kGradThreads / 32;
  const long long nb = std::min<long long>((warps + per_block - 1) / per_block,
                                           148LL * 64);
  if (g.dim == 3)
    k_traj_grad<3><<<(unsigned)nb, kGradThreads, 0, s>>>(
        traj_sorted, sec_sorted, idx, dens_sorted, grid, g, lut, dtab, dlen,
        dmult, M, C, scale, u, out);
  else
    k_traj_grad<2><<<(unsigned)nb, kGradThreads, 0, s>>>(
        traj_sorted, sec_sorted, idx, dens_sorted, grid, g, lut, dtab, dlen,
        dmult, M, C, scale, u, out);
  GN_LAUNCH_CHECK("trajectory gradient");
}

}  // namespace gnufft
