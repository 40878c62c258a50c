// Per-call device kernels of the operator path.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "geometry.hpp"
#include "tma.cuh"

namespace gnufft
{

// Forward work item: samples [begin, end) of one sector, at most
// kFwdItemSamples of them.
constexpr int kFwdItemSamples = 256;
struct FwdItem
{
  int sector;
  int begin;
  int end;
  int pad_;
};

// Whether the sector tiles of this geometry fit the kernels (why if not).
bool gridding_supported(const Geo &g, std::string &why);
// Coil-group width of the forward interpolation for C coils.
int forward_coil_group(int C, int dim, int pad);
// Dynamic shared memory of the forward interpolation (general grids).
size_t forward_smem_bytes(const Geo &g, int cg);

// ks[t*CP + c] = kspace[c*M + idx[t]] * sqrt(dens[t]) (dens may be NULL);
// zero for C <= c < CP.  (selectOrderedGPU, precomp_kernels.cu:179-205,
// and performDensityCompensation, std_gpuNUFFT_kernels.cu:220-242.)
void launch_gather_kspace(const float2 *kspace, const uint32_t *idx,
                          const float *dens_sorted, uint32_t M, int C, int CP,
                          float2 *ks, cudaStream_t s);
// The same result, reading the k-space in its original order (coalesced)
// and writing each sample's coil row to its sorted position inv[j]
// (inv = the inverse of the data-index permutation).
void launch_gather_kspace_inv(const float2 *kspace, const uint32_t *inv,
                              const float *dens_sorted, uint32_t M, int C,
                              int CP, float2 *ks, cudaStream_t s);
// inv[idx[t]] = t.
void launch_invert_permutation(const uint32_t *idx, uint32_t M,
                               uint32_t *inv, cudaStream_t s);

// Coil-group width of the sparse adjoint (lanes per cell).
int spmm_coil_group(int C);

// Adjoint spread as a product with the interpolation matrix (CSR by grid
// cell): grid [C][G] = W * ks, every cell written once.  With `shift`, cell
// g is stored at (g - floor(G/2)) mod G per axis (the upstream's INVERSE
// fftshift ahead of the inverse FFT).  ks: [M][CP] sorted k-space.
void launch_adjoint_spmm(const uint32_t *row_off, const uint2 *nz,
                         const float2 *ks, int CP, const Geo &g, int C,
                         bool shift, float2 *grid, cudaStream_t s);

// Adjoint spread of whole grid rows with the inverse DFT along x fused:
// out [C][G_z][G_y][N_x] (the cropped x outputs of every INVERSE-shifted
// grid row; the grid itself is not written).  Returns false (nothing
// launched) when the row length or coil grouping does not suit it.
bool launch_adjoint_spmm_xfft(const uint32_t *row_off, const uint2 *nz,
                              const float2 *ks, int CP, const Geo &g, int C,
                              const float2 *roots_x, float2 *out,
                              cudaStream_t s);

// Adjoint finish: crop of the (shifted) inverse-FFT output, 1/sqrt(Ng),
// deapodization, conj(sens) multiply and coil sum.  stage: 1 = FFT (crop +
// scale per coil), 2 = DEAPODIZATION.  With `accumulate` (maps only) the
// coil sum is added to `out` (the upstream's running sum over coil passes).
void launch_adjoint_finish(const float2 *grid, const float *deapo,
                           const float2 *sens, const Geo &g, int C, int stage,
                           bool accumulate, float2 *out, cudaStream_t s);

// Forward prepare: sens multiply, deapodization, zero pad and INVERSE
// fftshift into grid [C][G].  With `image_grid` the image is written
// unpadded and unshifted (DENSITY_ESTIMATION, image-sized grid).  With
// `signs` (every G even) cell (x, y, z) is multiplied by (-1)^(x+y+z), so
// that the forward transform yields the FORWARD-shifted spectrum.
void launch_forward_prepare(const float2 *image, const float2 *sens,
                            const float *deapo, const Geo &g, int C,
                            bool image_grid, float2 *grid, cudaStream_t s,
                            bool signs = false);

// Forward interpolation from grid [C][G] (the raw FFT output; with `shift`
// the upstream's FORWARD fftshift is folded into the tile gather), scaled by
// `scale` and sqrt(dens), scattered to out [C][M] in original order.
void launch_forward_interp(const FwdItem *items, int n_items,
                           const float *traj_sorted, const uint32_t *idx,
                           const float *dens_sorted, const float2 *grid,
                           const Geo &g, const float *lut, uint32_t M, int C,
                           bool shift, float scale, float2 *out,
                           cudaStream_t s, int tile_coils = 0);

// Forward interpolation with each sector tile fetched by one bulk tensor
// copy (tiles that wrap around the grid edge by plain loads).  The grid
// must hold the FORWARD-shifted spectrum (cell q at q).  cw.err (device
// pointer) is set to 1 if a copy did not complete within its bounded wait
// (cw.polls polls).
// Returns false when the geometry does not suit tensor copies (nothing is
// launched then).
bool launch_forward_interp_tma(const FwdItem *items, int n_items,
                               const float *traj_sorted, const uint32_t *idx,
                               const float *dens_sorted, const float2 *grid,
                               const Geo &g, const float *lut, uint32_t M,
                               int C, float scale, float2 *out,
                               tma::CopyWait cw, cudaStream_t s,
                               int tile_coils = 0, bool paired = false,
                               const uint32_t *lane_order = nullptr);

// The order in which the coil-pair forward (3-D) takes each work item's
// samples: `order` [M] lists, per item, sorted sample indices such that
// each eight adjacent lanes read their tile cells from different
// shared-memory bank groups.  Performance only: results do not depend on it.
void build_forward_lane_order(const FwdItem *items, int n_items,
                              const float *traj_sorted, uint32_t M,
                              const Geo &g, const float *lut, uint32_t *order,
                              cudaStream_t s);

// Whether the 3-D forward of this geometry runs on a grid written with coil
// pairs interleaved (cell q of coil c at ((c / 2) * G + q) * 2 + c % 2;
// launch_pruned_forward(paired) writes it, launch_forward_interp_tma(paired)
// reads it).
bool forward_pairs(const Geo &g, int tile_coils);

// --------------------------------------------------------------------------
// Batches of independent operators: every stage of all instances in one
// launch.  Each stage is a list of work units (instance, unit) with the
// instances' units consecutive; persistent blocks take unit indices from a
// counter (atomicAdd, no waiting) and run the unit with the template
// configuration of its instance.  The transforms between the stages are
// one cuFFT call per instance.
// --------------------------------------------------------------------------
constexpr int kBatchMax = 512;
enum BatchStage
{
  kBatchPrepare = 0,  // S x, deapodization, pad, shift (forward)
  kBatchInterp,       // interpolation to the samples (forward, 2-D)
  kBatchInterp3,      // the same for 3-D instances (its own launch)
  kBatchGather,       // k-space to sorted, coil-interleaved order (adjoint)
  kBatchSpread,       // interpolation matrix x k-space into the grid
  kBatchFinish,       // crop, scale, deapodization, conj(S) coil sum
  kBatchStages
};

struct BatchInst
{
  Geo g;
  uint32_t M;
  int C;        // coils of the instance
  int CP;       // coil lanes of the sorted k-space (multiple of spmm_cg)
  int spmm_cg;  // coils per spread group
  int fwd_cg;   // coils per forward tile
  int slots;    // footprint slots per axis of the interpolation stage
  int signs;    // grid cells multiplied by (-1)^(x+y+z) before the forward
                // transform (grids even along every axis)
  int tpr;      // prepare: threads per grid row
  int n_items;
  const FwdItem *items;
  const float *traj, *dens, *lut, *deapo;
  const uint32_t *di, *di_inv, *w_rows;
  const uint2 *w_nz;
  const float2 *sens;  // coil maps [C][N] (coil combine), or NULL
  float2 *grid;        // scratch [C][G]
  float2 *ks;          // scratch [M][CP]
  uint32_t first[kBatchStages];  // the instance's first unit of each stage
};

// Per-call data pointers of the instances (stage inputs / outputs).
struct BatchIo
{
  const float2 *in[kBatchMax];
  float2 *out[kBatchMax];
};

// Fills the configuration fields of `b` (CP, spmm_cg, fwd_cg, slots, tpr)
// from its geometry and coil count; tile_coils > 0 asks for that forward
// tile (reduced to fit).
void batch_configure(BatchInst &b, int tile_coils);
// Units of each stage for one configured instance.
void batch_units(const BatchInst &b, uint32_t units[kBatchStages]);
// Dynamic shared memory of the instance's interpolation units.
size_t batch_interp_smem(const BatchInst &b);
// One launch of `stage` over the n instances (device array `inst`, units
// `total`); `counter` (device, zero before the launch) hands out the units.
// `io` carries the inputs / outputs of the stages that read or write the
// caller's data.  Returns the number of blocks launched.
unsigned launch_batch_stage(int stage, const BatchInst *inst, int n,
                            uint32_t total, const BatchIo *io,
                            unsigned *counter, size_t interp_smem,
                            cudaStream_t s);

}  // namespace gnufft
