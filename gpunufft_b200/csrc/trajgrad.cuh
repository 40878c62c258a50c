// Trajectory gradient of the forward operator: kernel launcher and the
// tabulated Kaiser-Bessel derivative.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "geometry.hpp"

namespace gnufft
{

// Entries of the derivative table.
constexpr int kDerivLutLen = 4096;

// tab[i] = beta I1(beta s) / (s I0(beta) R^2) at d^2 = i / mult,
// s = sqrt(1 - d^2 / R^2); dpsi/dk = tab(d^2) * d * aniso.
void deriv_lut_fill(const Geo &g, float osf, int n, std::vector<float> &tab,
                    float &mult);

// out[a][idx[t]] = scale * sqrt(dens[t]) * sum_c Re(conj(u[c][idx[t]]) *
//   sum_cells dpsi/dk_a * grid_c(cell)) for every sorted sample t; grid is
// the FORWARD-FFT output [C][G] before the FORWARD shift (folded in here).
void launch_traj_grad(const float *traj_sorted, const uint32_t *sec_sorted,
                      const uint32_t *idx, const float *dens_sorted,
                      const float2 *grid, const Geo &g, const float *lut,
                      const float *dtab, int dlen, float dmult, uint32_t M,
                      int C, float scale, const float2 *u, float *out,
                      cudaStream_t s);

}  // namespace gnufft
