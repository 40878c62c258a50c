// Host-side geometry, kernel lookup table and deapodization.
// Upstream references are relative to the upstream CUDA/ directory.
#include "geometry.hpp"

#include <algorithm>
#include <cmath>
#include <complex>

#include "footprint.cuh"

namespace gnufft
{
namespace
{
// Modified Bessel function I0: Abramowitz & Stegun 9.8.1 (|x| < 3.75) and
// 9.8.2 polynomial approximations, evaluated in float like the upstream
// i0() (gpuNUFFT_utils.cpp:3-34).
float bessel_i0(float x)
{
  float ax = std::fabs(x);
  if (ax < 3.75f)
  {
    float y = x / 3.75f;
    y = y * y;
    return 1.0f +
           y * (3.5156229f +
                y * (3.0899424f +
                     y * (1.2067492f +
                          y * (0.2659732f + y * (0.360768e-1f + y * 0.45813e-2f)))));
  }
  float y = 3.75f / ax;
  return (std::exp(ax) / std::sqrt(ax)) *
         (0.39894228f +
          y * (0.1328592e-1f +
               y * (0.225319e-2f +
                    y * (-0.157565e-2f +
                         y * (0.916281e-2f +
                              y * (-0.2057706e-1f +
                                   y * (0.2635537e-1f +
                                        y * (-0.1647633e-1f + y * 0.392377e-2f))))))));
}

// Kaiser-Bessel shape parameter of Beatty et al. (MRM 2005), float like
// gpuNUFFT_utils.hpp:60-63 (the compiled upstream evaluates pow(t, 2) as t*t).
float kb_beta(uint32_t kw, float osf)
{
  const float t = (float)kw / osf * (osf - 0.5f);
  return (float)M_PI * std::sqrt(t * t - 0.8f);
}

// KB kernel at normalised radius r (gpuNUFFT_utils.hpp:72-75).
float kb_kernel(float r, uint32_t kw, float osf)
{
  return bessel_i0(kb_beta(kw, osf) * std::sqrt(1.0f - r * r)) /
         bessel_i0(kb_beta(kw, osf));
}
}  // namespace

long kernel_lut_size(float osf, uint32_t kw, bool lin_int)
{
  if (lin_int)
  {
    long kosf = (long)(std::floor(
        std::sqrt(0.37 / (double)((osf * osf) * 0.0001f))));
    return (long)(kosf * (float)kw * 0.5);
  }
  long kosf = (long)(std::floor(0.91f / (osf * 0.001f)));
  return (long)(kosf * (float)kw * 0.5);
}

void kernel_lut_fill(float *tab, long n, int kw, float osf)
{
  for (long i = 1; i < n - 1; i++)
  {
    if (kw == 1)
      tab[i] = 1.0f;
    else
    {
      double r = std::sqrt(i / (double)(n - 1));
      tab[i] = kb_kernel((float)r, (uint32_t)kw, osf);
    }
  }
  tab[0] = 1.0f;
  tab[n - 1] = 0.0f;
}

uint32_t host_sector_of(float c, int G, int sw)
{
  return sector_of_axis(c, (float)G, (float)sw);
}

bool make_geo(const uint32_t img[3], float osf, uint32_t kw, uint32_t sw,
              bool texture, Geo &g, std::string &err)
{
  g = Geo();
  if (img[0] == 0 || img[1] == 0)
  {
    err = "image width and height must be positive";
    return false;
  }
  if (kw < 1 || kw > (uint32_t)kMaxKernelWidth)
  {
    err = "kernel width must be in [1, 7]";
    return false;
  }
  if (sw < 1)
  {
    err = "sector width must be positive";
    return false;
  }
  if (!(osf >= 1.0f) || !std::isfinite(osf))
  {
    err = "oversampling factor must be >= 1";
    return false;
  }
  g.dim = img[2] == 0 ? 2 : 3;
  uint32_t grid[3];
  for (int a = 0; a < 3; ++a)
    grid[a] = (uint32_t)(img[a] * osf);  // gpuNUFFT_types.hpp:109-117
  for (int a = 0; a < g.dim; ++a)
  {
    if (grid[a] == 0)
    {
      err = "oversampled grid is empty";
      return false;
    }
  }
  long long gc = 1, ic = 1;
  for (int a = 0; a < 3; ++a)
  {
    bool used = a < g.dim;
    g.N[a] = used ? (int)img[a] : 1;
    g.G[a] = used ? (int)grid[a] : 1;
    // gpuNUFFT_operator_factory.cpp:22-26
    g.S[a] = used ? (int)std::ceil(static_cast<float>(grid[a]) / sw) : 1;
    g.Gf[a] = (float)g.G[a];
    g.halfG[a] = 0.5f * g.Gf[a];
    g.pow2G[a] = g.G[a] > 0 && (g.G[a] & (g.G[a] - 1)) == 0;
    g.invG[a] = g.pow2G[a] ? 1.0f / g.Gf[a] : 0.0f;
    gc *= g.G[a];
    ic *= g.N[a];
  }
  if (gc > (1LL << 31) || ic > (1LL << 31))
  {
    err = "grid too large (more than 2^31 cells)";
    return false;
  }
  g.grid_count = gc;
  g.img_count = ic;
  g.n_sectors = g.S[0] * g.S[1] * g.S[2];
  g.sw = (int)sw;
  g.kw = (int)kw;
  g.texture = texture ? 1 : 0;
  // gpuNUFFT_operator.cpp:101-141
  int gmax = std::max(std::max(grid[0], grid[1]), g.dim == 3 ? grid[2] : 0u);
  double kernel_radius = static_cast<double>(kw) / 2.0;
  double radius = kernel_radius / static_cast<double>(gmax);
  double radius_sq = radius * radius;
  double inv = 1.0 / radius_sq;
  long L = kernel_lut_size(osf, kw, texture);
  g.lut_len = (int)L;
  // texture operators size the multiplier by the 2-D table (unused there)
  long entries = texture ? L * L : L;
  g.dist_mult = (float)((unsigned)(entries - 1) * inv);
  g.kernel_radius = (float)kernel_radius;
  g.radius_sq = (float)radius_sq;
  g.radius_sq_inv = (float)inv;
  g.pad = (int)sw + 2 * (int)(std::floor((float)kw / 2.0f));
  g.offset = (int)std::floor((float)g.pad / 2.0f);
  for (int a = 0; a < 3; ++a)
  {
    bool used = a < g.dim;
    g.aniso[a] = used ? (float)grid[a] / (float)gmax : 0.0f;
    // std_gpuNUFFT_kernels.cu:546-556 (offset in float, truncated)
    g.crop[a] = used ? (int)(uint32_t)(img[a] * (osf - 1.0f) / 2.0f) : 0;
    // std_gpuNUFFT_kernels.cu:635-648
    g.shift_inv[a] = used ? (int)std::floor((float)grid[a] / 2.0f) : 0;
    g.shift_fwd[a] = used ? (int)std::ceil((float)grid[a] / 2.0f) : 0;
  }
  // std_gpuNUFFT_kernels.cu:135
  g.fft_scale = 1.0f / std::sqrt((float)(uint32_t)gc);
  return true;
}

int host_axis_footprint(float c, int ax, int sector_ax, const Geo &g,
                        const float *lut, int *cells, float *w)
{
  return axis_footprint(c, ax, sector_ax, g, lut, cells, w);
}

void compute_deapo(const Geo &g, const float *lut, std::vector<float> &out)
{
  // the upstream computes the deapodization with sector width 8
  Geo g8 = g;
  g8.sw = 8;
  g8.pad = 8 + 2 * (int)(std::floor((float)g.kw / 2.0f));
  g8.offset = (int)std::floor((float)g8.pad / 2.0f);
  std::vector<double> mag[3];
  for (int a = 0; a < g.dim; ++a)
  {
    int s = (int)host_sector_of(0.0f, g.G[a], 8);
    int cells[kSlots];
    float w[kSlots];
    int n = host_axis_footprint(0.0f, a, s, g8, lut, cells, w);
    mag[a].assign(g.N[a], 0.0);
    for (int i = 0; i < g.N[a]; ++i)
    {
      long long k = ((long long)i + g.crop[a] + g.shift_inv[a]) % g.G[a];
      std::complex<double> h(0.0, 0.0);
      for (int j = 0; j < n; ++j)
      {
        double ph = 2.0 * M_PI * (double)((cells[j] * k) % g.G[a]) / g.G[a];
        h += (double)w[j] * std::complex<double>(std::cos(ph), std::sin(ph));
      }
      mag[a][i] = std::abs(h);
    }
  }
  out.resize((size_t)g.img_count);
  size_t p = 0;
  int nz = g.dim == 3 ? g.N[2] : 1;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < g.N[1]; ++y)
      for (int x = 0; x < g.N[0]; ++x)
      {
        double m = mag[0][x] * mag[1][y] * (g.dim == 3 ? mag[2][z] : 1.0);
        out[p++] = (float)(1.0 / m);
      }
}

}  // namespace gnufft
