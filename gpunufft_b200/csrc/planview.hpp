// Read-only view of a plan's resident device tables, for entry points that
// live in their own translation unit.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>
#include <cufft.h>

#include "geometry.hpp"
#include "gridding.cuh"

struct gnufft_plan;

namespace gnufft
{

struct PlanView
{
  Geo g;
  uint32_t M;
  int device;
  uint32_t sens_coils;
  const uint32_t *data_indices;  // sorted position -> original sample
  const float *dens_sorted;      // NULL without density compensation
  const uint32_t *w_rows;        // interpolation matrix: CSR rows [G + 1]
  const uint2 *w_nz;             // (sorted sample, weight bits)
};

// Fill `v` from `p`; false if `p` is NULL.
bool plan_view(const gnufft_plan *p, PlanView *v);

// What a batch of operators reads from one plan: its resident tables, its
// maps (when it has maps for n_coils channels) and its cuFFT plan for
// n_coils transforms of the grid (created on first use; the plan's device
// must be current).
struct PlanTables
{
  Geo g;
  uint32_t M;
  int device;
  uint32_t sens_coils;
  int tile_coils;  // forward tile coils asked for at creation (0: automatic)
  const FwdItem *items;
  int n_items;
  const float *traj_sorted, *dens_sorted, *lut, *deapo;
  const uint32_t *data_indices, *inverse_indices, *w_rows;
  const uint2 *w_nz;
  const float2 *sens;  // NULL without maps
  cufftHandle fft;
};
bool plan_tables(gnufft_plan *p, uint32_t n_coils, PlanTables *t);

// Set the message returned by gnufft_last_error() for this thread.
void set_last_error(const std::string &msg);

}  // namespace gnufft
