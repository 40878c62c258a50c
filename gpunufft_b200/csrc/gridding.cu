// Per-call kernels of the operator path (sm_100a).
//
// Adjoint ("owner" spread): one CTA per owner sector.  The CTA accumulates
// the sector's sw^d interior cells for a group of CG coils in shared memory
// from every sample whose footprint reaches them (its own samples and the
// boundary samples of neighbouring sectors, listed at plan time), then
// writes each owned grid cell exactly once with coalesced stores.  No grid
// memset, no global atomics (except for the few targets whose candidate list
// is split over several CTAs), no halo write-back.  Warp lanes map to coils,
// so the footprint arithmetic of a sample is done once per warp and the
// shared-memory updates of a sample are 32 consecutive float2.
//
// Forward: one CTA per (sector, sample slice) gathers the sector tile plus
// halo for CG coils into shared memory (wrap-around and the upstream's
// FORWARD fftshift folded into the gather), then each warp interpolates
// samples with lanes over coils and scatters scaled results straight to the
// original sample order.
//
// Upstream references are relative to the upstream CUDA/ directory.
#include "gridding.cuh"

#include <algorithm>

#include "devutil.hpp"
#include "footprint.cuh"

namespace gnufft
{
namespace
{
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

__device__ __forceinline__ void split_sector(int s, const Geo &g, int *sa)
{
  sa[0] = s % g.S[0];
  int r = s / g.S[0];
  sa[1] = r % g.S[1];
  sa[2] = r / g.S[1];
}

__device__ __forceinline__ int wrap_mod(int v, int G)
{
  return v >= G ? v - G : (v < 0 ? v + G : v);
}

// --------------------------------------------------------------------------
// k-space gather into sorted order, coil-interleaved
// --------------------------------------------------------------------------
constexpr int kGatherSamples = 64;
constexpr int kGatherCoils = 32;

__global__ void __launch_bounds__(kThreads)
    k_gather_kspace(const float2 *__restrict__ kspace,
                    const uint32_t *__restrict__ idx,
                    const float *__restrict__ dens, uint32_t M, int C, int CP,
                    float2 *__restrict__ ks)
{
  __shared__ float2 tile[kGatherSamples][kGatherCoils + 1];
  __shared__ float sd[kGatherSamples];
  const size_t t0 = (size_t)blockIdx.x * kGatherSamples;
  const int c0 = blockIdx.y * kGatherCoils;
  const int nc = min(kGatherCoils, CP - c0);
  for (int i = threadIdx.x; i < kGatherSamples; i += kThreads)
  {
    const size_t t = t0 + i;
    sd[i] = (dens && t < M) ? sqrtf(dens[t]) : 1.0f;
  }
  for (int i = threadIdx.x; i < kGatherSamples * nc; i += kThreads)
  {
    const int tl = i % kGatherSamples, cl = i / kGatherSamples;
    const size_t t = t0 + tl;
    const int c = c0 + cl;
    float2 v = make_float2(0.f, 0.f);
    if (t < M && c < C)
      v = kspace[(size_t)c * M + idx[t]];
    tile[tl][cl] = v;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kGatherSamples * nc; i += kThreads)
  {
    const int cl = i % nc, tl = i / nc;
    const size_t t = t0 + tl;
    if (t < M)
    {
      float2 v = tile[tl][cl];
      if (dens)
      {  // density compensation: x * sqrt(w) per component
        v.x = __fmul_rn(v.x, sd[tl]);
        v.y = __fmul_rn(v.y, sd[tl]);
      }
      ks[t * CP + c0 + cl] = v;
    }
  }
}

// --------------------------------------------------------------------------
// adjoint owner spread
// --------------------------------------------------------------------------
template <int DIM>
__device__ __forceinline__ int owned_axis(float c, int ax, int sec_ax,
                                          int tgt_ax, const Geo &g,
                                          const float *lut, int *loc,
                                          float *w)
{
  int cells[kSlots];
  float wt[kSlots];
  const int n = axis_footprint(c, ax, sec_ax, g, lut, cells, wt);
  const int o = tgt_ax * g.sw;
  int k = 0;
  for (int i = 0; i < n; ++i)
  {
    const int l = cells[i] - o;
    if (l >= 0 && l < g.sw)
    {
      loc[k] = l;
      w[k] = wt[i];
      ++k;
    }
  }
  return k;
}

template <int DIM, int CG>
__global__ void __launch_bounds__(kThreads)
    k_adjoint_spread(const AdjItem *__restrict__ items,
                     const uint32_t *__restrict__ cand,
                     const uint32_t *__restrict__ sector_sorted,
                     const float *__restrict__ traj, const float2 *__restrict__ ks,
                     int CP, Geo g, const float *__restrict__ lut, uint32_t M,
                     int C, int shift, float2 *__restrict__ grid)
{
  extern __shared__ float2 tile[];  // [sw^DIM][CG + 1]
  constexpr int SLOTS = 32 / CG;
  constexpr int PITCH = CG + 1;
  const AdjItem it = items[blockIdx.x];
  const int group = blockIdx.y;
  const int sw = g.sw;
  const int cells = DIM == 3 ? sw * sw * sw : sw * sw;
  for (int i = threadIdx.x; i < cells * PITCH; i += kThreads)
    tile[i] = make_float2(0.f, 0.f);

  int ta[3];
  split_sector(it.target, g, ta);
  __syncthreads();

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = lane / CG, coil = lane % CG;
  const int gcoil = group * CG + coil;

  for (int j = it.begin + warp * SLOTS + slot; j < it.end;
       j += kWarps * SLOTS)
  {
    const uint32_t t = cand[j];
    int sa[3];
    split_sector((int)sector_sorted[t], g, sa);
    int lx[kSlots], ly[kSlots], lz[kSlots];
    float wx[kSlots], wy[kSlots], wz[kSlots];
    const int nx = owned_axis<DIM>(traj[t], 0, sa[0], ta[0], g, lut, lx, wx);
    const int ny =
        owned_axis<DIM>(traj[(size_t)M + t], 1, sa[1], ta[1], g, lut, ly, wy);
    int nz = 1;
    lz[0] = 0;
    wz[0] = 1.0f;
    if (DIM == 3)
      nz = owned_axis<DIM>(traj[2 * (size_t)M + t], 2, sa[2], ta[2], g, lut,
                           lz, wz);
    const float2 v = ks[(size_t)t * CP + gcoil];
    for (int z = 0; z < nz; ++z)
    {
      for (int y = 0; y < ny; ++y)
      {
        // upstream weight order: (K[z] * K[y]) * K[x]
        const float wzy = DIM == 3 ? __fmul_rn(wz[z], wy[y]) : wy[y];
        const int rowb = ((DIM == 3 ? lz[z] * sw : 0) + ly[y]) * sw;
        for (int x = 0; x < nx; ++x)
        {
          const float w = __fmul_rn(wzy, wx[x]);
          float2 *cell = tile + (size_t)(rowb + lx[x]) * PITCH + coil;
          atomicAdd(&cell->x, __fmul_rn(w, v.x));
          atomicAdd(&cell->y, __fmul_rn(w, v.y));
        }
      }
    }
  }
  __syncthreads();

  // store the owned cells (x fastest) of each coil of the group
  const long long G = g.grid_count;
  const int ox = ta[0] * sw, oy = ta[1] * sw, oz = DIM == 3 ? ta[2] * sw : 0;
  for (int i = threadIdx.x; i < cells * CG; i += kThreads)
  {
    const int cl = i / cells;
    const int cell = i - cl * cells;
    const int c = group * CG + cl;
    if (c >= C)
      continue;
    const int x = cell % sw;
    const int y = (cell / sw) % sw;
    const int z = DIM == 3 ? cell / (sw * sw) : 0;
    int gx = ox + x, gy = oy + y, gz = oz + z;
    if (gx >= g.G[0] || gy >= g.G[1] || gz >= g.G[2])
      continue;
    if (shift)
    {
      gx = wrap_mod(gx - g.shift_inv[0], g.G[0]);
      gy = wrap_mod(gy - g.shift_inv[1], g.G[1]);
      gz = DIM == 3 ? wrap_mod(gz - g.shift_inv[2], g.G[2]) : 0;
    }
    const long long q =
        ((long long)gz * g.G[1] + gy) * g.G[0] + gx + (long long)c * G;
    const float2 v = tile[(size_t)cell * PITCH + cl];
    if (it.split)
    {
      atomicAdd(&grid[q].x, v.x);
      atomicAdd(&grid[q].y, v.y);
    }
    else
    {
      grid[q] = v;
    }
  }
}

template <int DIM>
__global__ void k_zero_split(const int *__restrict__ targets, Geo g, int C,
                             int shift, float2 *__restrict__ grid)
{
  int ta[3];
  split_sector(targets[blockIdx.x], g, ta);
  const int sw = g.sw;
  const int cells = DIM == 3 ? sw * sw * sw : sw * sw;
  for (int i = threadIdx.x; i < cells * C; i += blockDim.x)
  {
    const int c = i / cells, cell = i - c * cells;
    int gx = ta[0] * sw + cell % sw, gy = ta[1] * sw + (cell / sw) % sw;
    int gz = DIM == 3 ? ta[2] * sw + cell / (sw * sw) : 0;
    if (gx >= g.G[0] || gy >= g.G[1] || gz >= g.G[2])
      continue;
    if (shift)
    {
      gx = wrap_mod(gx - g.shift_inv[0], g.G[0]);
      gy = wrap_mod(gy - g.shift_inv[1], g.G[1]);
      gz = DIM == 3 ? wrap_mod(gz - g.shift_inv[2], g.G[2]) : 0;
    }
    grid[((long long)gz * g.G[1] + gy) * g.G[0] + gx +
         (long long)c * g.grid_count] = make_float2(0.f, 0.f);
  }
}

// --------------------------------------------------------------------------
// forward interpolation
// --------------------------------------------------------------------------
template <int DIM, int CG>
__global__ void __launch_bounds__(kThreads)
    k_forward_interp(const FwdItem *__restrict__ items,
                     const float *__restrict__ traj,
                     const uint32_t *__restrict__ idx,
                     const float *__restrict__ dens,
                     const float2 *__restrict__ grid, Geo g,
                     const float *__restrict__ lut, uint32_t M, int C,
                     int shift, float scale, float2 *__restrict__ out)
{
  extern __shared__ float2 tile[];  // [pad^DIM][CG + 1]
  constexpr int SLOTS = 32 / CG;
  constexpr int PITCH = CG + 1;
  const FwdItem it = items[blockIdx.x];
  const int group = blockIdx.y;
  const int pad = g.pad;
  const int tcells = DIM == 3 ? pad * pad * pad : pad * pad;
  int sa[3];
  split_sector(it.sector, g, sa);
  int base[3];
  for (int a = 0; a < 3; ++a)
    base[a] = sa[a] * g.sw + (g.sw >> 1) - g.offset;
  const long long G = g.grid_count;

  // gather the tile (x fastest) for every coil of the group
  for (int i = threadIdx.x; i < tcells * CG; i += kThreads)
  {
    const int cl = i / tcells;
    const int cell = i - cl * tcells;
    const int c = group * CG + cl;
    float2 v = make_float2(0.f, 0.f);
    if (c < C)
    {
      const int ix = cell % pad, iy = (cell / pad) % pad;
      const int iz = DIM == 3 ? cell / (pad * pad) : 0;
      int q[3];
      const int li[3] = {ix, iy, iz};
      for (int a = 0; a < DIM; ++a)
      {
        int gc = base[a] + li[a];
        int gw = wrap_mod(gc, g.G[a]);
        if (gw < 0 || gw >= g.G[a])
          gw = ((gc % g.G[a]) + g.G[a]) % g.G[a];
        if (shift)  // FORWARD fftshift: value of cell gw is at gw + ceil(G/2)
          gw = wrap_mod(gw + g.shift_fwd[a], g.G[a]);
        q[a] = gw;
      }
      if (DIM == 2)
        q[2] = 0;
      v = grid[((long long)q[2] * g.G[1] + q[1]) * g.G[0] + q[0] +
               (long long)c * G];
    }
    tile[(size_t)cell * PITCH + cl] = v;
  }
  __syncthreads();

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = lane / CG, coil = lane % CG;
  const int c = group * CG + coil;
  for (int t = it.begin + warp * SLOTS + slot; t < it.end;
       t += kWarps * SLOTS)
  {
    int cx[kSlots], cy[kSlots], cz[kSlots];
    int ix[kSlots], iy[kSlots], iz[kSlots];
    float wx[kSlots], wy[kSlots], wz[kSlots];
    const int nx = axis_footprint(traj[t], 0, sa[0], g, lut, cx, wx, ix);
    const int ny =
        axis_footprint(traj[(size_t)M + t], 1, sa[1], g, lut, cy, wy, iy);
    int nz = 1;
    iz[0] = 0;
    wz[0] = 1.0f;
    if (DIM == 3)
      nz = axis_footprint(traj[2 * (size_t)M + t], 2, sa[2], g, lut, cz, wz,
                          iz);
    float ax = 0.f, ay = 0.f;
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
      {
        const float wzy = DIM == 3 ? __fmul_rn(wz[z], wy[y]) : wy[y];
        const int rowb = ((DIM == 3 ? iz[z] * pad : 0) + iy[y]) * pad;
        for (int x = 0; x < nx; ++x)
        {
          const float w = __fmul_rn(wzy, wx[x]);
          const float2 gv = tile[(size_t)(rowb + ix[x]) * PITCH + coil];
          ax = __fmaf_rn(gv.x, w, ax);
          ay = __fmaf_rn(gv.y, w, ay);
        }
      }
    if (c < C)
    {
      // performFFTScaling then performDensityCompensation
      // (std_gpuNUFFT_kernels.cu:114-140, 220-242)
      ax = __fmul_rn(ax, scale);
      ay = __fmul_rn(ay, scale);
      if (dens)
      {
        const float sd = sqrtf(dens[t]);
        ax = __fmul_rn(ax, sd);
        ay = __fmul_rn(ay, sd);
      }
      out[(size_t)c * M + idx[t]] = make_float2(ax, ay);
    }
  }
}

// --------------------------------------------------------------------------
// image-space stages
// --------------------------------------------------------------------------
template <bool SENS>
__global__ void k_adjoint_finish(const float2 *__restrict__ grid,
                                 const float *__restrict__ deapo,
                                 const float2 *__restrict__ sens, Geo g, int C,
                                 int stage, int accumulate,
                                 float2 *__restrict__ out)
{
  const long long N = g.img_count, G = g.grid_count;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x)
  {
    const int x = (int)(p % g.N[0]);
    const int y = (int)((p / g.N[0]) % g.N[1]);
    const int z = (int)(p / ((long long)g.N[0] * g.N[1]));
    // crop of the second INVERSE fftshift: index (n + crop + floor(G/2)) % G
    const int sx = (x + g.crop[0] + g.shift_inv[0]) % g.G[0];
    const int sy = (y + g.crop[1] + g.shift_inv[1]) % g.G[1];
    const int sz = (z + g.crop[2] + g.shift_inv[2]) % g.G[2];
    const long long src = ((long long)sz * g.G[1] + sy) * g.G[0] + sx;
    const float d = deapo[p];
    float accx = 0.f, accy = 0.f;
    for (int c = 0; c < C; ++c)
    {
      float2 v = grid[src + (long long)c * G];
      // crop -> FFT scaling -> deapodization (gpuNUFFT_operator.cpp:800-819)
      v.x = __fmul_rn(v.x, g.fft_scale);
      v.y = __fmul_rn(v.y, g.fft_scale);
      if (stage == 1)
      {
        out[p + (long long)c * N] = v;
        continue;
      }
      v.x = __fmul_rn(v.x, d);
      v.y = __fmul_rn(v.y, d);
      if (SENS)
      {
        // conj(S) * v, then the running coil sum
        // (std_gpuNUFFT_kernels.cu:158-218)
        const float2 s = sens[p + (long long)c * N];
        accx += v.x * s.x + v.y * s.y;
        accy += v.y * s.x - v.x * s.y;
      }
      else
      {
        out[p + (long long)c * N] = v;
      }
    }
    if (SENS && stage != 1)
    {
      if (accumulate)
      {
        const float2 o = out[p];
        accx = o.x + accx;
        accy = o.y + accy;
      }
      out[p] = make_float2(accx, accy);
    }
  }
}

template <bool SENS>
__global__ void k_forward_prepare(const float2 *__restrict__ image,
                                  const float2 *__restrict__ sens,
                                  const float *__restrict__ deapo, Geo g,
                                  int image_grid, float2 *__restrict__ grid)
{
  const int c = blockIdx.y;
  const long long N = g.img_count, G = g.grid_count;
  const long long total = image_grid ? N : G;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
       q < total; q += (long long)gridDim.x * blockDim.x)
  {
    long long p = q;
    bool inside = true;
    if (!image_grid)
    {
      const int qx = (int)(q % g.G[0]);
      const int qy = (int)((q / g.G[0]) % g.G[1]);
      const int qz = (int)(q / ((long long)g.G[0] * g.G[1]));
      // INVERSE fftshift of the padded grid: shifted[q] = padded[q+floor(G/2)]
      const int px = (qx + g.shift_inv[0]) % g.G[0] - g.crop[0];
      const int py = (qy + g.shift_inv[1]) % g.G[1] - g.crop[1];
      const int pz = (qz + g.shift_inv[2]) % g.G[2] - g.crop[2];
      inside = px >= 0 && px < g.N[0] && py >= 0 && py < g.N[1] && pz >= 0 &&
               pz < g.N[2];
      p = ((long long)pz * g.N[1] + py) * g.N[0] + px;
    }
    float2 v = make_float2(0.f, 0.f);
    if (inside)
    {
      if (SENS)
      {  // sensMulKernel (std_gpuNUFFT_kernels.cu:142-156)
        const float2 a = image[p];
        const float2 s = sens[p + (long long)c * N];
        v.x = a.x * s.x - a.y * s.y;
        v.y = a.x * s.y + a.y * s.x;
      }
      else
      {
        v = image[p + (long long)c * N];
      }
      const float d = deapo[p];
      v.x = __fmul_rn(v.x, d);
      v.y = __fmul_rn(v.y, d);
    }
    grid[q + (long long)c * (image_grid ? N : G)] = v;
  }
}

template <typename K>
void set_smem(K kernel, size_t bytes)
{
  if (bytes > 48 * 1024)
    GN_CUDA(cudaFuncSetAttribute(kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)bytes));
}

template <int DIM, int CG>
void adj_dispatch(const AdjItem *items, int n_items, const uint32_t *cand,
                  const uint32_t *sector_sorted, const float *traj,
                  const float2 *ks, int CP, const Geo &g, const float *lut,
                  uint32_t M, int C, bool shift, float2 *grid, cudaStream_t s)
{
  const size_t smem = adjoint_smem_bytes(g, CG);
  auto k = k_adjoint_spread<DIM, CG>;
  set_smem(k, smem);
  dim3 grd(n_items, (C + CG - 1) / CG);
  k<<<grd, kThreads, smem, s>>>(items, cand, sector_sorted, traj, ks, CP, g,
                                lut, M, C, shift ? 1 : 0, grid);
  GN_LAUNCH_CHECK("adjoint spread");
}

template <int DIM, int CG>
void fwd_dispatch(const FwdItem *items, int n_items, const float *traj,
                  const uint32_t *idx, const float *dens, const float2 *grid,
                  const Geo &g, const float *lut, uint32_t M, int C,
                  bool shift, float scale, float2 *out, cudaStream_t s)
{
  const size_t smem = forward_smem_bytes(g, CG);
  auto k = k_forward_interp<DIM, CG>;
  set_smem(k, smem);
  dim3 grd(n_items, (C + CG - 1) / CG);
  k<<<grd, kThreads, smem, s>>>(items, traj, idx, dens, grid, g, lut, M, C,
                                shift ? 1 : 0, scale, out);
  GN_LAUNCH_CHECK("forward interpolation");
}

int pow2_at_least(int c)
{
  int p = 1;
  while (p < c)
    p <<= 1;
  return p;
}
}  // namespace

int adjoint_coil_group(int C) { return C > 16 ? 32 : pow2_at_least(C); }

int forward_coil_group(int C, int dim, int pad)
{
  int cg = C > 16 ? 32 : pow2_at_least(C);
  // keep the tile + halo within shared memory
  const size_t cells = dim == 3 ? (size_t)pad * pad * pad : (size_t)pad * pad;
  while (cg > 1 && cells * (cg + 1) * sizeof(float2) > 200 * 1024)
    cg >>= 1;
  return cg;
}

size_t adjoint_smem_bytes(const Geo &g, int cg)
{
  const size_t cells = g.dim == 3 ? (size_t)g.sw * g.sw * g.sw
                                  : (size_t)g.sw * g.sw;
  return cells * (cg + 1) * sizeof(float2);
}

size_t forward_smem_bytes(const Geo &g, int cg)
{
  const size_t cells = g.dim == 3 ? (size_t)g.pad * g.pad * g.pad
                                  : (size_t)g.pad * g.pad;
  return cells * (cg + 1) * sizeof(float2);
}

void launch_gather_kspace(const float2 *kspace, const uint32_t *idx,
                          const float *dens_sorted, uint32_t M, int C, int CP,
                          float2 *ks, cudaStream_t s)
{
  if (!M)
    return;
  dim3 grd((M + kGatherSamples - 1) / kGatherSamples,
           (CP + kGatherCoils - 1) / kGatherCoils);
  k_gather_kspace<<<grd, kThreads, 0, s>>>(kspace, idx, dens_sorted, M, C, CP,
                                           ks);
  GN_LAUNCH_CHECK("gather k-space");
}

void launch_zero_split(const int *targets, int n_targets, const Geo &g, int C,
                       bool shift, float2 *grid, cudaStream_t s)
{
  if (n_targets <= 0)
    return;
  if (g.dim == 3)
    k_zero_split<3><<<n_targets, kThreads, 0, s>>>(targets, g, C, shift,
                                                   grid);
  else
    k_zero_split<2><<<n_targets, kThreads, 0, s>>>(targets, g, C, shift,
                                                   grid);
  GN_LAUNCH_CHECK("zero split targets");
}

void launch_adjoint_spread(const AdjItem *items, int n_items,
                           const uint32_t *cand, const uint32_t *sector_sorted,
                           const float *traj_sorted, const float2 *ks, int CP,
                           const Geo &g, const float *lut, uint32_t M, int C,
                           bool shift, float2 *grid, cudaStream_t s)
{
  if (n_items <= 0)
    return;
  const int cg = adjoint_coil_group(C);
#define GN_ADJ(D, CGV)                                                         \
  adj_dispatch<D, CGV>(items, n_items, cand, sector_sorted, traj_sorted, ks,  \
                       CP, g, lut, M, C, shift, grid, s)
#define GN_ADJ_CG(D)                                                           \
  switch (cg)                                                                  \
  {                                                                            \
  case 1: GN_ADJ(D, 1); break;                                                 \
  case 2: GN_ADJ(D, 2); break;                                                 \
  case 4: GN_ADJ(D, 4); break;                                                 \
  case 8: GN_ADJ(D, 8); break;                                                 \
  case 16: GN_ADJ(D, 16); break;                                               \
  default: GN_ADJ(D, 32); break;                                               \
  }
  if (g.dim == 3)
  {
    GN_ADJ_CG(3)
  }
  else
  {
    GN_ADJ_CG(2)
  }
#undef GN_ADJ_CG
#undef GN_ADJ
}

void launch_adjoint_finish(const float2 *grid, const float *deapo,
                           const float2 *sens, const Geo &g, int C, int stage,
                           bool accumulate, float2 *out, cudaStream_t s)
{
  const unsigned nb = grid_for((size_t)g.img_count, kThreads, 148 * 16);
  if (sens)
    k_adjoint_finish<true><<<nb, kThreads, 0, s>>>(grid, deapo, sens, g, C,
                                                   stage, accumulate ? 1 : 0,
                                                   out);
  else
    k_adjoint_finish<false><<<nb, kThreads, 0, s>>>(grid, deapo, nullptr, g,
                                                    C, stage, 0, out);
  GN_LAUNCH_CHECK("adjoint finish");
}

void launch_forward_prepare(const float2 *image, const float2 *sens,
                            const float *deapo, const Geo &g, int C,
                            bool image_grid, float2 *grid, cudaStream_t s)
{
  const size_t total = image_grid ? (size_t)g.img_count : (size_t)g.grid_count;
  dim3 grd(grid_for(total, kThreads, 148 * 8), C);
  if (sens)
    k_forward_prepare<true><<<grd, kThreads, 0, s>>>(image, sens, deapo, g,
                                                     image_grid, grid);
  else
    k_forward_prepare<false><<<grd, kThreads, 0, s>>>(image, nullptr, deapo,
                                                      g, image_grid, grid);
  GN_LAUNCH_CHECK("forward prepare");
}

void launch_forward_interp(const FwdItem *items, int n_items,
                           const float *traj_sorted, const uint32_t *idx,
                           const float *dens_sorted, const float2 *grid,
                           const Geo &g, const float *lut, uint32_t M, int C,
                           bool shift, float scale, float2 *out,
                           cudaStream_t s)
{
  if (n_items <= 0)
    return;
  const int cg = forward_coil_group(C, g.dim, g.pad);
#define GN_FWD(D, CGV)                                                         \
  fwd_dispatch<D, CGV>(items, n_items, traj_sorted, idx, dens_sorted, grid, g, \
                       lut, M, C, shift, scale, out, s)
#define GN_FWD_CG(D)                                                           \
  switch (cg)                                                                  \
  {                                                                            \
  case 1: GN_FWD(D, 1); break;                                                 \
  case 2: GN_FWD(D, 2); break;                                                 \
  case 4: GN_FWD(D, 4); break;                                                 \
  case 8: GN_FWD(D, 8); break;                                                 \
  case 16: GN_FWD(D, 16); break;                                               \
  default: GN_FWD(D, 32); break;                                               \
  }
  if (g.dim == 3)
  {
    GN_FWD_CG(3)
  }
  else
  {
    GN_FWD_CG(2)
  }
#undef GN_FWD_CG
#undef GN_FWD
}

}  // namespace gnufft
