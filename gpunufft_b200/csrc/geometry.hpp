// Problem geometry shared by host and device code.
//
// Every quantity is computed with the upstream's arithmetic (float vs double
// exactly where the upstream uses them) so that integer results -- sector
// ids, footprint bounds, lookup-table indices -- are bit-identical to the
// upstream's.  Upstream references are relative to its CUDA/ directory.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace gnufft
{

// Footprint slots per axis: ceil(p-kw/2)..floor(p+kw/2) spans <= kw+1 cells.
constexpr int kMaxKernelWidth = 7;
constexpr int kSlots = kMaxKernelWidth + 1;

// Samples per work item of the upstream balanced operators
// (MAXIMUM_PAYLOAD, gpuNUFFT_types.hpp:23); used for the exported
// processing order only.
constexpr uint32_t kUpstreamPayload = 256;

// POD handed to every kernel by value.
struct Geo
{
  int dim;          // 2 or 3
  int N[3];         // image dims (x, y, z); z == 1 in 2-D
  int G[3];         // oversampled grid dims; z == 1 in 2-D
  int S[3];         // sectors per axis; z == 1 in 2-D
  int sw, kw, pad, offset;
  float Gf[3];      // (float)G
  float halfG[3];   // 0.5f * (float)G
  float invG[3];    // 1 / G, used instead of a division when G is a power
                    // of two (then x * (1/G) == x / G exactly)
  int pow2G[3];     // G is a power of two
  float kernel_radius;   // kw / 2
  float radius_sq;       // (kw/2 / max G)^2, stored float (double math)
  float radius_sq_inv;
  float dist_mult;       // (L - 1) / radius_sq
  float aniso[3];        // G_axis / max G
  int lut_len;
  int texture;           // linear-interpolated LUT, no radius cut
  // TEXTURE operators on the device: the lookup table as a normalised,
  // clamp-addressed, linearly filtered texture object (0 on the host side
  // and for the other operator types)
  unsigned long long lut_tex;
  int crop[3];           // (uint)(N * (osf - 1) / 2) per axis
  int shift_inv[3];      // floor(G/2): INVERSE fftshift offset
  int shift_fwd[3];      // ceil(G/2): FORWARD fftshift offset
  int n_sectors;
  long long grid_count;  // Gx*Gy*Gz
  long long img_count;   // Nx*Ny*Nz
  float fft_scale;       // 1 / sqrt(grid_count) (float, as upstream)
};

// Host-side geometry builder (gpuNUFFT_operator.cpp:53-146 and the factory
// helpers).  `img` is (width, height, depth) with depth 0 for 2-D.
bool make_geo(const uint32_t img[3], float osf, uint32_t kw, uint32_t sw,
              bool texture, Geo &g, std::string &err);

// Upstream LUT sizes (gpuNUFFT_utils.cpp:47-60) and values (:74-107).
long kernel_lut_size(float osf, uint32_t kw, bool lin_int);
void kernel_lut_fill(float *tab, long n, int kw, float osf);

// Per-axis sector id of one coordinate (precomp_utils.hpp:34-48).
uint32_t host_sector_of(float c, int G, int sw);

// One axis of the footprint of a sample (host twin of the device routine):
// wrapped grid cells and weights.  Returns the count (<= kSlots).
int host_axis_footprint(float c, int ax, int sector_ax, const Geo &g,
                        const float *lut, int *cells, float *w);

// Deapodization (gpuNUFFT_operator_factory.cpp:359-448) evaluated directly:
// the upstream grids one unit sample at k = 0 with sector width 8, inverse
// FFTs, crops and scales, then takes 1/|h * sqrt(Ng)|.  The grid is the
// outer product of per-axis weight vectors, so |h| is the product of the
// per-axis DFT magnitudes, evaluated here in double.  Output [image].
void compute_deapo(const Geo &g, const float *lut, std::vector<float> &out);

}  // namespace gnufft
