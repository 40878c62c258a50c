// Separable, pruned Cartesian transforms of the operator path, fused with
// its image-space stages.
//
// The forward operator transforms a zero-padded image: of the grid lines
// along x only the N_y (x N_z) rows that hold image pixels are non-zero,
// and along y only N_z planes.  The adjoint keeps only the cropped N of G
// outputs per axis.  Transforming axis by axis and skipping the lines that
// are zero (forward) or not needed (adjoint) moves (1/4 + 1/2 + 1) instead
// of 3 grids through HBM per direction in 3-D at osf 2, and the first
// (forward) or last (adjoint) pass carries the sensitivity multiply,
// deapodization, pad/crop, fftshift and coil combine.
//
// Each line of length L = R1 * R2 is transformed in two register stages:
// R2 threads each do an R1-point DFT (radix-2, in registers), multiply by
// exp(-+2 pi i t k1 / L) and exchange through shared memory; R1 threads
// then do the R2-point DFTs.  Roots come from a table computed on the host
// in double precision.  Results equal cuFFT's (unnormalised) transforms to
// rounding.
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "geometry.hpp"
#include "tma.cuh"

namespace gnufft
{

// Every grid axis a power of two in [16, 1024].
bool pruned_fft_supported(const Geo &g);

// tab[j] = exp(-2 pi i j / L), j < L.
void fft_roots(int L, std::vector<float2> &tab);

// Scratch (complex elements) of the pruned passes for C coils.
size_t pruned_scratch_a(const Geo &g, int C);
size_t pruned_scratch_b(const Geo &g, int C);

// Forward: image ([N] with maps, else [C][N]) -> sens multiply ->
// deapodization -> zero pad -> INVERSE fftshift -> unnormalised forward DFT
// -> FORWARD fftshift -> grid [C][G] (so cell q of the shifted spectrum, the
// one the interpolation reads, is stored at q).
// roots[a]: the root table of axis a (length G[a]).
// zrange (3-D, optional): per (y, x) column the z rows to write; the
// others are left as they are (the interpolation never reads them).
// err (optional): the mapped error flag of the tensor-copy passes (set when
// a tile copy does not complete within its bounded wait); without it the
// passes load their tiles with plain loads.  paired (3-D, needs err and
// every grid axis <= 256): the grid is written with coil pairs interleaved,
// cell q of coil c at ((c / 2) * G + q) * 2 + c % 2 (C rounded up to even
// coils of storage).  ztiles (paired only): the n_ztiles column tiles of
// ztile_cols columns (ascending) that hold a z range; the z pass transforms
// only these (the others have no cell the interpolation reads).
void launch_pruned_forward(const float2 *image, const float2 *sens,
                           const float *deapo, const Geo &g, int C,
                           const float2 *const roots[3], float2 *tmp_a,
                           float2 *tmp_b, float2 *grid, cudaStream_t s,
                           const uint2 *zrange = nullptr,
                           tma::CopyWait cw = tma::CopyWait(),
                           bool paired = false,
                           const uint32_t *ztiles = nullptr, int n_ztiles = 0,
                           int ztile_cols = 0);

// Adjoint: grid [C][G] (INVERSE fftshift folded in by the adjoint spread)
// -> unnormalised inverse DFT -> crop of the second INVERSE fftshift ->
// 1/sqrt(Ng) -> (stage 2) deapodization -> conj(sens) coil sum.  stage 1
// writes the cropped, scaled image per coil (the upstream FFT output
// stage); `accumulate` adds the coil sum to `out`.
void launch_pruned_adjoint(const float2 *grid, const float *deapo,
                           const float2 *sens, const Geo &g, int C, int stage,
                           int accumulate, const float2 *const roots[3],
                           float2 *tmp_a, float2 *tmp_b, float2 *out,
                           cudaStream_t s);

// The adjoint with the x transform done first (fused into the spread,
// launch_adjoint_spmm_xfft): xrows [C][G_z][G_y][N_x] -> (3-D) y pass into
// tmp_b [C][G_z][N_y][N_x] -> last pass (z in 3-D, y in 2-D) fused with
// crop, 1/sqrt(Ng), deapodization and the conj(S) coil sum (per coil group,
// the groups' sums added in group order through `part`, C x N complex).
void launch_pruned_adjoint_xfirst(const float2 *xrows, const float *deapo,
                                  const float2 *sens, const Geo &g, int C,
                                  int stage, int accumulate,
                                  const float2 *const roots[3],
                                  float2 *tmp_b, float2 *part, float2 *out,
                                  cudaStream_t s,
                                  tma::CopyWait cw = tma::CopyWait());
size_t pruned_scratch_xfirst(const Geo &g, int C);

}  // namespace gnufft
