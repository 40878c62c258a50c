/*
 * gpunufft_b200 -- C ABI of the B200 (sm_100a) gpuNUFFT operator path.
 *
 * One opaque plan per trajectory replaces one upstream GpuNUFFTOperator:
 *
 *   upstream (andyschwarzl/gpuNUFFT, paths relative to CUDA/)      here
 *   -------------------------------------------------------------- ---------------------------
 *   GpuNUFFTOperatorFactory::createGpuNUFFTOperator                gnufft_plan_create
 *     (inc/gpuNUFFT_operator_factory.hpp:81-123,
 *      src/gpuNUFFT_operator_factory.cpp:450-553)
 *   GpuNUFFTOperatorFactory::loadPrecomputedGpuNUFFTOperator       gnufft_plan_load
 *     (inc/gpuNUFFT_operator_factory.hpp:142-172,
 *      src/gpuNUFFT_operator_factory.cpp:576-626)
 *   delete GpuNUFFTOperator (inc/gpuNUFFT_operator.hpp:73-87)      gnufft_plan_destroy
 *   GpuNUFFTOperator::performGpuNUFFTAdj(Array, Array&, Output)    gnufft_adjoint_host
 *     (inc/gpuNUFFT_operator.hpp:243-300, src/gpuNUFFT_operator.cpp:615-861)
 *   GpuNUFFTOperator::performGpuNUFFTAdj(GpuArray, GpuArray&, ..)  gnufft_adjoint_device
 *     (src/gpuNUFFT_operator.cpp:370-580)
 *   GpuNUFFTOperator::performForwardGpuNUFFT(Array, Array&, ..)    gnufft_forward_host
 *     (inc/gpuNUFFT_operator.hpp:301-345, src/gpuNUFFT_operator.cpp:1092-1268)
 *   GpuNUFFTOperator::performForwardGpuNUFFT(GpuArray, ..)         gnufft_forward_device
 *     (src/gpuNUFFT_operator.cpp:895-1059)
 *   getters getDataIndices/getSectorDataCount/getSectorCenters/    gnufft_export_tables
 *     getKSpaceTraj/getDens, BalancedOperator::getSectorProcessing  gnufft_plan_get_info
 *     Order (inc/gpuNUFFT_operator.hpp:92-216, balanced_operator.hpp:13-20)
 *   setSens / applySensData (inc/gpuNUFFT_operator.hpp:110-113,    gnufft_set_sens
 *     :348-357)
 *   HANDLE_ERROR -> exit(EXIT_FAILURE) (inc/cuda_utils.hpp:22-30), status codes +
 *     std::invalid_argument / runtime_error from the factory       gnufft_last_error
 *
 * Layouts are the upstream ones: trajectory float32 structure-of-arrays
 * [x_0..x_{M-1}, y_0.., (z_0..)] in [-0.5, 0.5); k-space complex64 (float2)
 * [coil][sample] in ORIGINAL sample order; images complex64
 * [coil][z][y][x] (x fastest); sensitivity maps like images; density
 * compensation float32 [sample].  Coordinates are interpreted exactly as the
 * upstream does (sector binning, footprint, wrap-around).
 *
 * Errors never terminate the process: every call returns a gnufft_status and
 * gnufft_last_error() describes the last failure of the calling thread.
 * A plan is not reentrant (its scratch buffers are shared by its calls);
 * distinct plans are independent and may be used from different threads.
 */
#ifndef GPUNUFFT_B200_H
#define GPUNUFFT_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define GNUFFT_API __attribute__((visibility("default")))
#else
#define GNUFFT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gnufft_plan gnufft_plan;

typedef enum gnufft_status {
  GNUFFT_SUCCESS = 0,
  /* upstream: std::invalid_argument (gpuNUFFT_operator_factory.cpp:460-466) */
  GNUFFT_ERROR_INVALID_ARGUMENT = 1,
  /* upstream: std::runtime_error from checkMemoryConsumption (:628-663) */
  GNUFFT_ERROR_OUT_OF_MEMORY = 2,
  /* upstream: HANDLE_ERROR -> exit (cuda_utils.hpp:22-30) */
  GNUFFT_ERROR_CUDA = 3,
  /* upstream: printed and ignored (gpuNUFFT_operator.cpp:489-495) */
  GNUFFT_ERROR_CUFFT = 4,
  GNUFFT_ERROR_NOT_SUPPORTED = 5,
  GNUFFT_ERROR_INTERNAL = 6
} gnufft_status;

/* upstream OperatorType (gpuNUFFT_types.hpp:193-205) */
typedef enum gnufft_operator_type {
  GNUFFT_DEFAULT = 0,
  GNUFFT_TEXTURE = 1,
  GNUFFT_BALANCED = 2,
  GNUFFT_BALANCED_TEXTURE = 3
} gnufft_operator_type;

/* upstream GpuNUFFTOutput (gpuNUFFT_types.hpp:167-181) */
typedef enum gnufft_output {
  GNUFFT_CONVOLUTION = 0,
  GNUFFT_FFT = 1,
  GNUFFT_DEAPODIZATION = 2,
  GNUFFT_DENSITY_ESTIMATION = 3
} gnufft_output;

/* Plan flags. */
/* Order samples inside each sector exactly as the upstream factory's
 * std::sort does (host sort); default is a stable GPU counting sort.  Both
 * give identical sector offsets, centers and per-sector index sets. */
#define GNUFFT_FLAG_REFERENCE_ORDER 0x1u
/* Execute every call the way the upstream operator does: one coil per pass,
 * sensitivity maps copied per coil per call, a device synchronisation per
 * coil.  For comparisons only; the default executes all coils of a call in
 * one pass with resident maps. */
#define GNUFFT_FLAG_PLAIN 0x2u
/* Run the Cartesian transforms through cuFFT (the full 3 passes over the
 * oversampled grid) instead of the separable pruned transforms fused with the
 * image-space stages, which are the default when every grid axis is a power
 * of two in [16, 1024].  For comparisons. */
#define GNUFFT_FLAG_CUFFT 0x4u
/* Forward-interpolation tile shape (the autotuner's knob): coils staged per
 * sector tile, n = 1, 2, 4, 8, 16 or 32, stored in bits 8-11 as
 * log2(n) + 1; 0 selects automatically.  n is reduced until the tile fits
 * in shared memory. */
#define GNUFFT_FLAG_FWD_TILE_COILS(n)                                        \
  ((uint32_t)((n) <= 1 ? 1 : (n) <= 2 ? 2 : (n) <= 4 ? 3 : (n) <= 8 ? 4 :   \
              (n) <= 16 ? 5 : 6) << 8)
#define GNUFFT_FLAG_FWD_TILE_MASK 0xF00u

typedef struct gnufft_desc {
  uint32_t img_dims[3];  /* width, height, depth; depth == 0 selects 2-D */
  uint32_t n_samples;    /* M */
  uint32_t n_coils;      /* channels of the sensitivity maps, 0 if none */
  uint32_t kernel_width; /* upstream kernelWidth (1..7) */
  uint32_t sector_width; /* upstream sectorWidth (>= 1) */
  float osf;             /* upstream osf (grid = (uint)(img * osf)) */
  int32_t operator_type; /* gnufft_operator_type */
  uint32_t flags;        /* GNUFFT_FLAG_* */
  int32_t device;        /* CUDA device ordinal */
} gnufft_desc;

typedef struct gnufft_plan_info {
  uint32_t dim;               /* 2 or 3 */
  uint32_t img_dims[3];       /* width, height, depth (depth 0 for 2-D) */
  uint32_t grid_dims[3];      /* oversampled grid (depth 0 for 2-D) */
  uint32_t sector_dims[3];    /* sectors per axis (depth 0 for 2-D) */
  uint32_t n_sectors;         /* product of the non-zero sector_dims */
  uint32_t n_samples;
  uint32_t n_coils;           /* channels of the sensitivity maps, 0 if none */
  uint32_t kernel_lut_len;    /* entries of the kernel lookup table */
  uint32_t n_processing_order;/* entries of the balanced processing order */
  uint32_t has_dens;
  uint64_t device_bytes;      /* device memory held by the plan */
} gnufft_plan_info;

/* Create a plan (upstream createGpuNUFFTOperator).  traj: host float32
 * SoA [dim * n_samples]; dens: host float32 [n_samples] or NULL; sens: host
 * complex64 [n_coils][image] or NULL.  Sector binning, sorting and the
 * deapodization function are computed here; all tables stay resident. */
GNUFFT_API gnufft_status gnufft_plan_create(const gnufft_desc *desc, const float *traj,
                                 const float *dens, const void *sens,
                                 gnufft_plan **plan);

/* Create a plan from precomputed tables (upstream
 * loadPrecomputedGpuNUFFTOperator, the MATLAB 7-array contract):
 * traj_sorted [dim * M], data_indices [M], sector_data_count [S + 1],
 * processing_order [2 * n_order] (may be NULL), sector_centers [dim * S],
 * dens_sorted [M] or NULL, sens [n_coils][image] or NULL, deapo [image].
 * Host pointers.  Tables are validated (sizes, ranges, monotone offsets). */
GNUFFT_API gnufft_status gnufft_plan_load(const gnufft_desc *desc,
                               const float *traj_sorted,
                               const uint32_t *data_indices,
                               const uint32_t *sector_data_count,
                               const uint32_t *processing_order,
                               uint32_t n_order,
                               const uint32_t *sector_centers,
                               const float *dens_sorted, const void *sens,
                               const float *deapo, gnufft_plan **plan);

GNUFFT_API gnufft_status gnufft_plan_destroy(gnufft_plan *plan);

GNUFFT_API gnufft_status gnufft_plan_get_info(const gnufft_plan *plan,
                                   gnufft_plan_info *info);

/* Copy the plan's tables to host buffers (any pointer may be NULL):
 * traj_sorted [dim*M], data_indices [M], sector_data_count [S+1],
 * processing_order [2*n_processing_order], sector_centers [dim*S],
 * dens_sorted [M] (only if the plan has density compensation),
 * deapo [image], kernel_lut [kernel_lut_len]. */
GNUFFT_API gnufft_status gnufft_export_tables(const gnufft_plan *plan, float *traj_sorted,
                                   uint32_t *data_indices,
                                   uint32_t *sector_data_count,
                                   uint32_t *processing_order,
                                   uint32_t *sector_centers,
                                   float *dens_sorted, float *deapo,
                                   float *kernel_lut);

/* Replace (or with sens == NULL remove) the sensitivity maps; host pointer,
 * complex64 [n_coils][image]. */
GNUFFT_API gnufft_status gnufft_set_sens(gnufft_plan *plan, const void *sens,
                              uint32_t n_coils);

/* Replace the sensitivity maps from DEVICE memory: complex64
 * [n_coils][image] copied device-to-device into the plan, ordered on
 * `stream` (no host copy, no synchronisation; for serving loops that keep
 * maps on the GPU).  Not for plans created with GNUFFT_FLAG_PLAIN, which
 * stream host maps per coil like the upstream. */
GNUFFT_API gnufft_status gnufft_set_sens_device(gnufft_plan *plan,
                                       const void *sens, uint32_t n_coils,
                                       void *stream);

/* Adjoint NUFFT.  kspace: complex64 [n_coils][M]; image (output):
 *   CONVOLUTION / DENSITY_ESTIMATION: raw grid [n_coils][grid]
 *   FFT: [n_coils][image] after inverse FFT, crop and 1/sqrt(grid count)
 *   DEAPODIZATION: [image] coil-combined when the plan has sensitivity
 *                  maps, else [n_coils][image].
 * _host: host buffers, synchronous.  _device: device buffers, ordered on
 * `stream` (a cudaStream_t; NULL = the legacy default stream).
 * Host arrays of 16 MB or more (and host sensitivity maps given to
 * gnufft_set_sens / gnufft_plan_create) are copied through a process-wide
 * ring of two 8 MB pinned buffers per device, allocated on first use and
 * kept until the process ends, filled and drained by up to four short-lived
 * host threads per chunk; smaller ones with one pageable copy. */
GNUFFT_API gnufft_status gnufft_adjoint_host(gnufft_plan *plan, const void *kspace,
                                  void *image, uint32_t n_coils,
                                  int32_t output);
GNUFFT_API gnufft_status gnufft_adjoint_device(gnufft_plan *plan, const void *kspace,
                                    void *image, uint32_t n_coils,
                                    int32_t output, void *stream);

/* Forward NUFFT.  image: [image] when the plan has sensitivity maps (the
 * image is multiplied by every map), else [n_coils][image]; kspace
 * (output): complex64 [n_coils][M] in original sample order.
 * DENSITY_ESTIMATION interpolates straight from the (deapodized) image array
 * treated as the grid, like the upstream (meaningful at osf = 1). */
GNUFFT_API gnufft_status gnufft_forward_host(gnufft_plan *plan, const void *image,
                                  void *kspace, uint32_t n_coils,
                                  int32_t output);
GNUFFT_API gnufft_status gnufft_forward_device(gnufft_plan *plan, const void *image,
                                    void *kspace, uint32_t n_coils,
                                    int32_t output, void *stream);

/* Adjoint up to the CONVOLUTION stage -- the raw oversampled grid
 * [n_coils][grid], as gnufft_adjoint_device with GNUFFT_CONVOLUTION -- that
 * performs no device allocation of any kind.  No counterpart in the
 * upstream library.  It is for callers that may not allocate while they
 * run: real-time reconstruction loops and serving workers that reserve all
 * memory up front, code living inside another framework's fixed memory
 * budget, and callers that cannot afford the device synchronisation that
 * cudaMalloc / cudaFree imply.  The regular entry points grow the plan's
 * scratch on first use; this one stages the sorted k-space in a fixed
 * device array of GNUFFT_NOALLOC_SCRATCH_BYTES inside the library (held on
 * every GPU that loads the library until the process exits), so
 * n_samples x coil lanes x 8 bytes must fit in it (coil lanes: n_coils
 * rounded up to 1, 2, 4, 8, 16 or a multiple of 32); larger requests are
 * rejected with GNUFFT_ERROR_INVALID_ARGUMENT.  kspace and grid are device
 * buffers; the call is ordered on `stream`.  Every call looks up the
 * array's device address on the plan's device (the first call on a device
 * also loads the library's device code there); make that first call before
 * any stream capture.  All calls on a device share the array: calls that
 * overlap on the GPU race and must be serialised by the caller. */
#define GNUFFT_NOALLOC_SCRATCH_BYTES ((size_t)16 << 20)
GNUFFT_API gnufft_status gnufft_adjoint_convolution_noalloc(
    gnufft_plan *plan, const void *kspace, void *grid, uint32_t n_coils,
    void *stream);

/* Gradient of a real loss with respect to the trajectory (no upstream
 * counterpart; used by the differentiable operator).  With y = forward(image)
 * (the plan's maps and density weights included) and kspace_weights u
 * [n_coils][M] (original order, device), writes
 *   grad_traj[a][j] = sum_c Re( conj(u[c][j]) * d y[c][j] / d k_a[j] )
 * (float32 [dim][M], device), the derivative taken through the Kaiser-Bessel
 * interpolation of the oversampled spectrum.  For the adjoint x = A^H y and
 * dL/dx = v, pass image = v and kspace_weights = y.  image as for
 * gnufft_forward_device.  Ordered on `stream`. */
GNUFFT_API gnufft_status gnufft_traj_grad_device(gnufft_plan *plan, const void *image,
                                      const void *kspace_weights,
                                      uint32_t n_coils, float *grad_traj,
                                      void *stream);

/* Device time (ms) of the stages of the last call on this plan, measured
 * with CUDA events when timing is enabled (gnufft_set_timing). */
typedef struct gnufft_stage_times {
  float prepare_ms;   /* k-space gather / image pad */
  float gridding_ms;  /* adjoint spread or forward interpolation */
  float fft_ms;       /* cuFFT */
  float finish_ms;    /* crop / deapodization / coil combine / scatter */
  uint32_t launches;  /* kernels of this library launched by the call */
} gnufft_stage_times;
GNUFFT_API gnufft_status gnufft_set_timing(gnufft_plan *plan, int enable);

/* Device memory of a call.  The plan's scratch buffers (sorted k-space,
 * grid, transform buffers) grow on first use to what a call with n_coils
 * coils needs (gnufft_call_scratch_bytes reports that figure) and are kept.
 * A call whose scratch for all its coils would not fit the plan's memory
 * limit -- by default the device memory free at the call plus the scratch
 * the plan holds already, less 256 MiB -- runs in passes of as many coils
 * as fit (at least one), like the upstream's concurrent coil count
 * (gpuNUFFT_operator.cpp:327-368, there for 2-D only); results are the
 * same up to the order of the coil sum.  gnufft_set_memory_limit sets the
 * limit in bytes (0: the free memory). */
GNUFFT_API gnufft_status gnufft_set_memory_limit(gnufft_plan *plan,
                                                 uint64_t bytes);
GNUFFT_API gnufft_status gnufft_call_scratch_bytes(const gnufft_plan *plan,
                                                   uint32_t n_coils,
                                                   uint64_t *bytes);

/* Tile copies of this library's kernels complete on a bounded wait: a copy
 * that has not completed after the wait's polls sets a flag, the block
 * stops (after a bounded wait for its copies in flight) and the call
 * reports GNUFFT_ERROR_CUDA ("a tile copy did not complete within its
 * wait") -- the host calls at their end, a device call at the plan's next
 * call or at gnufft_plan_check after the caller synchronised its stream.
 * No counterpart in the upstream (which waits without bound).
 * gnufft_set_copy_wait sets the polls of each block's first wait for a copy
 * (negative: the default, about 4 million); a small value exercises the
 * failure path (0 gives up at once).  gnufft_plan_check returns and clears
 * a pending copy failure of the plan. */
GNUFFT_API gnufft_status gnufft_set_copy_wait(gnufft_plan *plan,
                                              int64_t polls);
GNUFFT_API gnufft_status gnufft_plan_check(gnufft_plan *plan);
GNUFFT_API gnufft_status gnufft_get_stage_times(const gnufft_plan *plan,
                                     gnufft_stage_times *times);

/* Batches of independent operators (no counterpart in the upstream, whose
 * operators each run their own per-coil loop).  A batch runs the full
 * operator (DEAPODIZATION output: coil combine when the plan has maps) of
 * many instances -- different trajectories, image sizes, oversampling,
 * kernel widths, sector widths and coil counts -- with every gridding
 * stage of all instances in one persistent launch: forward = prepare
 * (maps, deapodization, pad, shift), one cuFFT call per instance,
 * interpolation (one launch per dimensionality present); adjoint = k-space
 * gather, spread, one cuFFT call per instance, finish (crop,
 * deapodization, conj(maps) coil sum).  Each stage's blocks take
 * (instance, work item) units from a device counter.  The cuFFT calls run
 * on up to 8 side streams of the batch, forked from and joined back into
 * the caller's stream (instances sharing a plan share a side stream).
 *
 * gnufft_batch_create: plans[i] and n_coils[i] describe instance i (n_coils
 * must equal the plan's map channels when it has maps); one plan may appear
 * several times (frames sharing a trajectory).  All plans on one device;
 * they must outlive the batch, and their maps must not be removed or
 * replaced with a different channel count while it exists (the batch reads
 * the plans' tables and maps in place; maps replaced with the same channel
 * count are read in their new values).  The batch owns the instances'
 * scratch (grid and sorted k-space).  At most 512 instances.
 *
 * gnufft_batch_forward: images[i] (device): [n_coils][image] complex64, or
 * [image] when the plan has maps; kspace[i] (device, output):
 * [n_coils][M] in original sample order.  gnufft_batch_adjoint: the
 * reverse.  Calls are ordered on `stream` and may be captured into a CUDA
 * graph; a batch is not reentrant. */
typedef struct gnufft_batch gnufft_batch;
typedef struct
{
  uint32_t n_instances;
  uint32_t units[5];       /* work units per stage: prepare, interpolation,
                              gather, spread, finish */
  uint32_t kernels_forward; /* this library's launches per forward */
  uint32_t kernels_adjoint; /* ... per adjoint (cuFFT calls not counted) */
  uint32_t fft_calls;       /* cuFFT calls per forward or adjoint */
  uint64_t device_bytes;    /* scratch and descriptors owned by the batch */
} gnufft_batch_info;

GNUFFT_API gnufft_status gnufft_batch_create(gnufft_plan *const *plans,
                                             const uint32_t *n_coils,
                                             uint32_t n_instances,
                                             gnufft_batch **out);
GNUFFT_API gnufft_status gnufft_batch_forward(gnufft_batch *batch,
                                              const void *const *images,
                                              void *const *kspace,
                                              void *stream);
GNUFFT_API gnufft_status gnufft_batch_adjoint(gnufft_batch *batch,
                                              const void *const *kspace,
                                              void *const *images,
                                              void *stream);
GNUFFT_API gnufft_status gnufft_batch_get_info(const gnufft_batch *batch,
                                               gnufft_batch_info *info);
GNUFFT_API gnufft_status gnufft_batch_destroy(gnufft_batch *batch);

GNUFFT_API const char *gnufft_last_error(void);
GNUFFT_API const char *gnufft_status_string(gnufft_status status);
GNUFFT_API const char *gnufft_version(void);

#ifdef __cplusplus
}
#endif

#endif /* GPUNUFFT_B200_H */
