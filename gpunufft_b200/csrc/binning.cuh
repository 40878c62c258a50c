// Plan-time integer work on the device: sector assignment, stable sort,
// scans, the interpolation matrix and the forward column ranges.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "devutil.hpp"
#include "geometry.hpp"

namespace gnufft
{

// Exclusive prefix sum of n u32 values (in may equal out).  `scratch`
// (device, scan_scratch_elems(n) u32, or NULL) holds the block sums; with
// NULL the call allocates them and synchronises the stream before freeing.
void scan_exclusive(const uint32_t *in, uint32_t *out, size_t n,
                    cudaStream_t s, uint32_t *scratch = nullptr);
size_t scan_scratch_elems(size_t n);

// Stable LSD radix sort of (key, value) pairs on the low `key_bits` bits of
// the keys.  Sorted output ends in keys_out / vals_out.
void sort_pairs(const uint32_t *keys_in, const uint32_t *vals_in,
                uint32_t *keys_out, uint32_t *vals_out, size_t n, int key_bits,
                cudaStream_t s);

// Counts of `n` keys in [0, bins) -> offsets[bins + 1] (exclusive scan).
void histogram_offsets(const uint32_t *keys, size_t n, uint32_t bins,
                       uint32_t *offsets, cudaStream_t s);

// Sector of every sample, original order (assignSectors,
// gpuNUFFT_operator_factory.cpp:128-181; precomp_kernels.cu:8-45).
void assign_sectors(const float *traj, uint32_t M, const Geo &g,
                    uint32_t *sector, cudaStream_t s);

// traj_sorted[a][t] = traj[a][idx[t]]; dens_sorted[t] = dens[idx[t]]
// (sortArraysKernel, precomp_kernels.cu:85-113).
void gather_sorted(const float *traj, const float *dens, const uint32_t *idx,
                   uint32_t M, int dim, float *traj_sorted, float *dens_sorted,
                   cudaStream_t s);

// Interpolation matrix of the trajectory in CSR form keyed by grid cell:
// for every (unshifted, x-fastest) grid cell the list of (sorted sample t,
// kernel weight) pairs whose footprint covers it, ascending in t.  The
// weights are the upstream's (K[z] * K[y]) * K[x] (or the texture
// interpolation), footprints as the upstream kernels compute them.
// Output: row_off [G + 1] (u32) and nz [nnz] (uint2: t, weight bits).
// Returns nnz.
size_t build_interp_matrix(const float *traj_sorted,
                           const uint32_t *sector_sorted, uint32_t M,
                           const Geo &g, const float *lut,
                           DeviceBuffer &row_off, DeviceBuffer &nz,
                           cudaStream_t s);

// Per (y, x) column of the grid, the range [lo, hi] of z cells that carry
// interpolation weights (widened by one; lo > hi when none): the forward
// transform writes only these cells, the only ones the interpolation reads.
// `tiles` lists (ascending, n_tiles of them) the tiles of kColTile adjacent
// columns (tile t: columns t * kColTile ...) that hold at least one range;
// the forward z pass transforms only those.
constexpr int kColTile = 8;
void build_column_ranges(const uint32_t *row_off, const Geo &g,
                         DeviceBuffer &range, DeviceBuffer &tiles,
                         int &n_tiles, cudaStream_t s);

}  // namespace gnufft
