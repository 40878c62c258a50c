// Per-sample sector id and per-axis kernel footprint, shared verbatim by the
// host (plan set-up, deapodization) and the device kernels.
//
// Each floating-point step is written with an explicit rounding intrinsic on
// the device so that nvcc cannot contract or reorder it; the results are
// then bit-identical to the upstream expressions they restate.  Host code
// is compiled with -ffp-contract=off for the same reason.
// Upstream references are relative to the upstream CUDA/ directory.
#pragma once

#include <cmath>
#include <cstdint>

#include "geometry.hpp"

#if defined(__CUDA_ARCH__)
#define GN_FMUL(a, b) __fmul_rn((a), (b))
#define GN_FADD(a, b) __fadd_rn((a), (b))
#define GN_FSUB(a, b) __fsub_rn((a), (b))
#define GN_FDIV(a, b) __fdiv_rn((a), (b))
#define GN_FMA(a, b, c) __fmaf_rn((a), (b), (c))
#define GN_DDIV(a, b) __ddiv_rn((a), (b))
#define GN_DADD(a, b) __dadd_rn((a), (b))
#define GN_LDG(p) __ldg(p)
#else
#define GN_FMUL(a, b) ((a) * (b))
#define GN_FADD(a, b) ((a) + (b))
#define GN_FSUB(a, b) ((a) - (b))
#define GN_FDIV(a, b) ((a) / (b))
#define GN_FMA(a, b, c) std::fma((a), (b), (c))
#define GN_DDIV(a, b) ((a) / (b))
#define GN_DADD(a, b) ((a) + (b))
#define GN_LDG(p) (*(p))
#endif

#if defined(__CUDACC__)
#define GN_HD __host__ __device__ __forceinline__
#else
#define GN_HD inline
#endif

namespace gnufft
{

// Sector of one coordinate along one axis (precomp_utils.hpp:34-48):
// floor(round(c*G + 0.5*G) / sw), clamped to [0, ceil(G/sw) - 1].  c*G is a
// float product; the sum, round and division are double.
GN_HD uint32_t sector_of_axis(float c, float G, float sw)
{
  double p = GN_DADD((double)GN_FMUL(c, G), 0.5 * (double)G);
  int s = (int)floor(GN_DDIV(round(p), (double)sw));
  int top = (int)ceilf(GN_FDIV(G, sw));
  if (s >= top)
    s = top - 1;
  if (s < 0)
    s = 0;
  return (uint32_t)s;
}

// gc / G in float (mapGridToKSpace, gpuNUFFT_utils.hpp:202-209); for a
// power-of-two G the product with the exact reciprocal is the same number.
GN_HD float grid_to_k(int gc, int ax, const Geo &g)
{
  return g.pow2G[ax] ? GN_FMUL((float)gc, g.invG[ax])
                     : GN_FDIV((float)gc, g.Gf[ax]);
}

// Linear interpolation of a table over normalised coordinate u, the way the
// texture unit filters a normalised, clamp-addressed texture: texel
// coordinate u*W - 0.5, weight quantised to 8 fractional bits
// (cuda_utils.cuh:27-37 with load2DKernel; the 2-D table of the upstream is
// the outer product of the 1-D table, so its bilinear lookup factorises).
// The texture unit derives its 8-bit weight from a coordinate it holds with
// fewer bits than float, so weights next to a rounding boundary may differ
// by 1/256 from this model: host code (the deapodization) uses the model,
// device code uses the texture unit itself (texture_weight).
GN_HD float lerp_table(const float *tab, int W, float u)
{
  float x = GN_FSUB(GN_FMUL(u, (float)W), 0.5f);
  float fl = floorf(x);
  float a = GN_FSUB(x, fl);
  a = GN_FMUL(rintf(GN_FMUL(a, 256.0f)), 0.00390625f);
  int i0 = (int)fl;
  int i1 = i0 + 1;
  i0 = i0 < 0 ? 0 : (i0 > W - 1 ? W - 1 : i0);
  i1 = i1 < 0 ? 0 : (i1 > W - 1 ? W - 1 : i1);
  float t0 = GN_LDG(tab + i0), t1 = GN_LDG(tab + i1);
  return GN_FADD(GN_FMUL(GN_FSUB(1.0f, a), t0), GN_FMUL(a, t1));
}

// Weight of the TEXTURE operators at normalised coordinate u = d^2 / R^2:
// on the device the hardware-filtered fetch from the plan's texture object,
// exactly the lookup the upstream texture kernels make
// (cuda_utils.cuh:27-37, std_gpuNUFFT_kernels.cu:49-60: linear filtering,
// normalised coordinates, clamp); the software model on the host.
GN_HD float texture_weight(const Geo &g, const float *lut, float u)
{
#if defined(__CUDA_ARCH__)
  if (g.lut_tex)
    return tex1D<float>((cudaTextureObject_t)g.lut_tex, u);
#endif
  return lerp_table(lut, g.lut_len, u);
}

// One axis of the upstream footprint of a sample with coordinate c that
// belongs to sector index `sector_ax` along this axis, computed in that
// sector's tile frame exactly as the upstream kernels do
// (atomic_gpuNUFFT_kernels.cu:302-451 and 966-1131):
//   pos   = mapKSpaceToGrid  (gpuNUFFT_utils.hpp:194-199; c*G + 0.5*G is
//           one fused multiply-add in the compiled upstream kernels)
//   range = set_minmax       (gpuNUFFT_utils.hpp:89-104) within the tile
//   kx    = mapGridToKSpace  (gpuNUFFT_utils.hpp:202-209)
//   keep  d^2 < R^2 (per axis); weight = LUT[round(d^2 * dist_mult)]
// TEXTURE operators keep every cell of the range and weight it with the
// linearly interpolated table at d^2 / R^2 (texture_gpuNUFFT_kernels.cu
// :63-97).  Outputs the wrap-around grid cells (calculateOppositeIndex,
// gpuNUFFT_utils.hpp:268-278), the weights and, if `local` is given, the
// tile-frame indices; returns their count.
GN_HD int axis_footprint(float c, int ax, int sector_ax, const Geo &g,
                         const float *lut, int *cells, float *w,
                         int *local = nullptr)
{
  const int center = sector_ax * g.sw + (g.sw >> 1);
  float pos = GN_FMA(c, g.Gf[ax], g.halfG[ax]);
  pos = GN_FADD(GN_FSUB(pos, (float)center), (float)g.offset);
  const int pmax = g.pad - 1;
  int imin = (int)ceilf(GN_FSUB(pos, g.kernel_radius));
  int imax = (int)floorf(GN_FADD(pos, g.kernel_radius));
  if (imin < 0)
    imin = 0;
  if (imax < 0)
    imax = 0;
  if (imax >= pmax)
    imax = pmax;
  if (imin >= pmax)
    imin = (int)(pmax - 2 * g.kernel_radius);
  if (imax - imin + 1 > kSlots)
    imax = imin + kSlots - 1;  // unreachable for kw <= kMaxKernelWidth
  const int G = g.G[ax];
  int n = 0;
  for (int i = imin; i <= imax; ++i)
  {
    int gc = i + center - g.offset;
    float k = GN_FSUB(grid_to_k(gc, ax, g), 0.5f);
    float d = GN_FMUL(GN_FSUB(k, c), g.aniso[ax]);
    float d2 = GN_FMUL(d, d);
    float wt;
    if (g.texture)
    {
      wt = texture_weight(g, lut, GN_FMUL(d2, g.radius_sq_inv));
    }
    else
    {
      if (!(d2 < g.radius_sq))
        continue;
      int li = (int)roundf(GN_FMUL(d2, g.dist_mult));
      li = li < 0 ? 0 : (li > g.lut_len - 1 ? g.lut_len - 1 : li);
      wt = GN_LDG(lut + li);
    }
    int gw = gc;
    if (gw >= G)
      gw -= G;
    else if (gw < 0)
      gw += G;
    if (gw < 0 || gw >= G)  // grids smaller than a tile: wrap fully
      gw = ((gc % G) + G) % G;
    cells[n] = gw;
    w[n] = wt;
    if (local)
      local[n] = i;
    ++n;
  }
  return n;
}

}  // namespace gnufft
