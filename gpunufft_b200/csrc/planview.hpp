// Read-only view of a plan's resident device tables, for entry points that
// live in their own translation unit.
#pragma once

#include <cstdint>
#include <string>

#include <cuda_runtime.h>

#include "geometry.hpp"

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

// Set the message returned by gnufft_last_error() for this thread.
void set_last_error(const std::string &msg);

}  // namespace gnufft
