// Per-call kernels of the operator path (sm_100a).
//
// Adjoint: the sorted k-space is gathered coil-interleaved (one row of coil
// values per sample), then spread as a sparse product with the plan's
// interpolation matrix: one block per grid row chunk and coil group streams
// the chunk's nonzeros in equal shares per unit of lanes, keeps running
// cell sums in registers and finishes cells cut by share boundaries in
// unit order (deterministic, no atomics).  On power-of-two grids the spread
// takes whole rows and runs the inverse x transform in place before writing
// only the cropped outputs (k_adjoint_spmm_xfft).
//
// Forward: one block per work item (<= 256 samples of one sector) stages the
// sector tile plus halo of a coil group in shared memory -- by tensor copies
// when the grid holds the FORWARD-shifted spectrum and the tile is a box of
// it, else by cp.async gathers with wrap-around and shift folded in -- and
// interpolates the item's samples, scattering scaled results straight to
// the original sample order.
//
// Batches: every stage above, and the elementwise prepare / finish, as one
// persistent launch over the (instance, unit) lists of many operators.
//
// Upstream references are relative to the upstream CUDA/ directory.
#include "gridding.cuh"

#include <algorithm>
#include <type_traits>

#include <cuda.h>

#include "devutil.hpp"
#include "fftcore.cuh"
#include "footprint.cuh"
#include "tma.cuh"

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

// Asynchronous global -> shared copies (no register round trip, many in
// flight per thread); completed by cp_async_wait_all() + __syncthreads().
__device__ __forceinline__ void cp_async8(void *smem_dst, const void *gsrc)
{
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s),
               "l"(gsrc)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all()
{
  asm volatile("cp.async.wait_all;\n" ::: "memory");
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

// The same gather driven by the original order: a block reads 64
// consecutive original samples of 32 coils (coalesced per coil), and writes
// each sample's coil row (contiguous) to its sorted position inv[j].  One
// unit: sample block jb, coil block cb.
__device__ __forceinline__ void gather_inv_unit(
    int jb, int cb, const float2 *__restrict__ kspace,
    const uint32_t *__restrict__ inv, const float *__restrict__ dens,
    uint32_t M, int C, int CP, float2 *__restrict__ ks)
{
  __shared__ float2 tile[kGatherSamples][kGatherCoils + 1];
  __shared__ uint32_t s_t[kGatherSamples];
  __shared__ float sd[kGatherSamples];
  const size_t j0 = (size_t)jb * kGatherSamples;
  const int c0 = cb * kGatherCoils;
  const int nc = min(kGatherCoils, CP - c0);
  for (int i = threadIdx.x; i < kGatherSamples; i += kThreads)
  {
    const size_t j = j0 + i;
    const uint32_t t = j < M ? __ldg(inv + j) : 0u;
    s_t[i] = t;
    sd[i] = (dens && j < M) ? sqrtf(__ldg(dens + t)) : 1.0f;
  }
  for (int i = threadIdx.x; i < kGatherSamples * nc; i += kThreads)
  {
    const int jl = i % kGatherSamples, cl = i / kGatherSamples;
    const size_t j = j0 + jl;
    const int c = c0 + cl;
    float2 v = make_float2(0.f, 0.f);
    if (j < M && c < C)
      v = __ldg(kspace + (size_t)c * M + j);
    tile[jl][cl] = v;
  }
  __syncthreads();
  // one sample's coil row per nc consecutive threads (a whole block of
  // coils: nc is a constant, so the row and lane are a shift and a mask)
  auto put = [&](int i, int n) {
    const int cl = i % n, jl = i / n;
    if (j0 + jl < M)
    {
      float2 v = tile[jl][cl];
      if (dens)
      {  // density compensation: x * sqrt(w) per component
        v.x = __fmul_rn(v.x, sd[jl]);
        v.y = __fmul_rn(v.y, sd[jl]);
      }
      ks[(size_t)s_t[jl] * CP + c0 + cl] = v;
    }
  };
  if (nc == kGatherCoils)
  {
#pragma unroll
    for (int i = threadIdx.x; i < kGatherSamples * kGatherCoils; i += kThreads)
      put(i, kGatherCoils);
  }
  else
    for (int i = threadIdx.x; i < kGatherSamples * nc; i += kThreads)
      put(i, nc);
}

__global__ void __launch_bounds__(kThreads)
    k_gather_kspace_inv(const float2 *__restrict__ kspace,
                        const uint32_t *__restrict__ inv,
                        const float *__restrict__ dens, uint32_t M, int C,
                        int CP, float2 *__restrict__ ks)
{
  gather_inv_unit(blockIdx.x, blockIdx.y, kspace, inv, dens, M, C, CP, ks);
}

__global__ void k_invert(const uint32_t *__restrict__ idx, uint32_t M,
                         uint32_t *__restrict__ inv)
{
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < M;
       t += (size_t)gridDim.x * blockDim.x)
    inv[idx[t]] = (uint32_t)t;
}

// --------------------------------------------------------------------------
// compact per-axis footprints (phase A: one sample per thread)
// --------------------------------------------------------------------------
// An axis is described by up to KS (index, weight) entries with static
// register indices: the consecutive cells imin.. of the footprint in the
// frame of the sample's own sector tile.
template <int KS>
__device__ __forceinline__ int compact_axis(float c, int ax, int sec_ax,
                                            const Geo &g, const float *lut,
                                            int *li, float *w)
{
  const int center = sec_ax * g.sw + (g.sw >> 1);
  float pos = __fmaf_rn(c, g.Gf[ax], g.halfG[ax]);
  pos = __fadd_rn(__fsub_rn(pos, (float)center), (float)g.offset);
  const int pmax = g.pad - 1;
  int imin = (int)ceilf(__fsub_rn(pos, g.kernel_radius));
  int imax = (int)floorf(__fadd_rn(pos, g.kernel_radius));
  if (imin < 0)
    imin = 0;
  if (imax < 0)
    imax = 0;
  if (imax >= pmax)
    imax = pmax;
  if (imin >= pmax)
    imin = (int)(pmax - 2 * g.kernel_radius);
  int n = 0;
#pragma unroll
  for (int k = 0; k < KS; ++k)
  {
    li[k] = 0;
    w[k] = 0.0f;
  }
#pragma unroll
  for (int k = 0; k < KS; ++k)
  {
    const int i = imin + k;
    const int gc = i + center - g.offset;
    const float kx = __fsub_rn(grid_to_k(gc, ax, g), 0.5f);
    const float d = __fmul_rn(__fsub_rn(kx, c), g.aniso[ax]);
    const float d2 = __fmul_rn(d, d);
    bool valid = i <= imax && i >= 0;
    float wt;
    if (g.texture)
      wt = texture_weight(g, lut, __fmul_rn(d2, g.radius_sq_inv));
    else
    {
      valid = valid && d2 < g.radius_sq;
      int lx = (int)roundf(__fmul_rn(d2, g.dist_mult));
      lx = lx < 0 ? 0 : (lx > g.lut_len - 1 ? g.lut_len - 1 : lx);
      wt = valid ? __ldg(lut + lx) : 0.0f;
    }
    // append (static indices only: entry j receives candidate k if j == n)
#pragma unroll
    for (int j = 0; j < KS; ++j)
      if (valid && j == n)
      {
        li[j] = i;
        w[j] = wt;
      }
    n += valid ? 1 : 0;
  }
  return n;
}

// Sector widths above this are rejected (plan-time tables and tiles are
// sized for it).
constexpr int kMaxSectorWidth = 32;

// --------------------------------------------------------------------------
// adjoint as a product with the interpolation matrix (CSR by grid cell)
// --------------------------------------------------------------------------
// One block per (grid row, 64-cell x chunk, coil group).  The chunk's
// nonzeros (a contiguous CSR range) are split into equal shares, one per
// warp slot ("unit"); a unit streams its share with the CG coils of a
// sample in its lanes (8*CG contiguous bytes of the sorted k-space per
// entry) and keeps a running sum per cell in registers.  A cell inside one
// unit's share is stored once.  A cell cut by share boundaries is summed by
// the unit where it starts: after a barrier it adds the partial sums of the
// following units that continue the cell, in unit order.  So the summation
// order is fixed (results are bitwise reproducible) and there are no
// atomics.  The chunk is then written once per coil with coalesced stores
// (INVERSE fftshift folded into the store position).
constexpr int kSpmmCells = 64;

// Position of (cell, coil c) in a spread accumulator of CG coils per cell:
// rows padded to CG + 1 (SR2 == 0), or rows of CG with the coil index
// XOR-swizzled by the cell (SR2 = R2 of the row transform that runs in place
// on the accumulator).  The swizzle flips coil bits 1-3 only (those below
// CG), so coil pairs stay adjacent (16-byte stores), and it varies with both cell % SR2 and
// cell / SR2, so that the transform's stage-1 accesses (cells r0 + lt) and
// stage-2 accesses (cells k1 * SR2 + t) each spread over all banks.
template <int CG, int SR2>
__device__ __forceinline__ int acc_pos(int cell, int c)
{
  if constexpr (SR2 == 0)
    return cell * (CG + 1) + c;
  else
  {
    const int sw = ((cell % SR2) ^ (cell / SR2)) & 7;
    return cell * CG + (c ^ ((sw << 1) & (CG - 1)));
  }
}

// The streaming accumulation of a block's cell range [0, nxc) (offsets
// s_off, nonzeros from s_off[0] to s_off[nxc]) for the CG coils of `group`:
// equal shares of the nonzeros per warp slot, running cell sums in
// registers, cells cut by share boundaries finished in slot order.  acc
// (laid out by acc_pos<CG, SR2>) must be zero and head/tail_cell -1 on
// entry (after a barrier); acc holds every cell after the caller's next
// barrier.  A unit whose last cell continues in the next shares leaves its
// partial sum in acc; the following units' partials (part_head) are added
// to it in unit order.  With ZG the caller zeroes only the empty cells
// before the row's first and after its last nonzero: every unit stores
// each cell it passes (zero sums included), and the empty cells between
// two units' cells are zeroed by the later unit.
template <int CG, int V, int SR2 = 0, bool ZG = false>
__device__ __forceinline__ void spmm_accumulate(
    const uint32_t *s_off, int nxc, const uint2 *__restrict__ nz,
    const float2 *__restrict__ ks, int CP, int group, float2 *acc,
    float2 *part_head, int *head_cell, int *tail_cell)
{
  constexpr int LS = CG / V;          // lanes per slot
  constexpr int SLOTS = 32 / LS;
  constexpr int NU = kWarps * SLOTS;  // streaming units per block
  constexpr int B = 8 / V;            // entries per batch
  const uint32_t A = s_off[0], E = s_off[nxc];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = lane / LS, cl = lane % LS;
  const int unit = warp * SLOTS + slot;
  const float2 *ksg = ks + group * CG + cl * V;
  // an equal share of the block's contiguous nonzero range per unit
  const uint32_t len = (E - A + NU - 1) / NU;
  const uint32_t u0 = min(E, A + unit * len), u1 = min(E, u0 + len);
  // first cell whose range contains u0: the number of bounds
  // s_off[1..nxc] <= u0 (nondecreasing).  Slots of 16 or 32 lanes count
  // them with ballots (nxc / LS steps); narrower slots, for which that
  // loop is long, by a branchless binary search with the same trip count
  // in every lane
  int cell = 0;
  if constexpr (LS >= 16)
  {
    const unsigned slot_bits =
        (LS == 32 ? 0xffffffffu : ((1u << LS) - 1u)) << (slot * LS);
    for (int base = 0; base < nxc; base += LS)
    {
      const int i = base + cl + 1;
      const bool le = i <= nxc && s_off[i] <= u0;
      cell += __popc(__ballot_sync(0xffffffffu, le) & slot_bits);
    }
  }
  else
  {
    for (int step = nxc > 0 ? 1 << (31 - __clz(nxc)) : 0; step > 0;
         step >>= 1)
      if (cell + step <= nxc && s_off[cell + step] <= u0)
        cell += step;
  }
  if (ZG && A < u0 && u0 < u1)
  {  // empty cells just before this unit's first cell start at u0
    for (int c = cell - 1; c >= 0 && s_off[c] == u0; --c)
#pragma unroll
      for (int v = 0; v < V; ++v)
        acc[acc_pos<CG, SR2>(c, cl * V + v)] = make_float2(0.f, 0.f);
  }
  if (u0 < u1)
  {
    uint32_t bound = s_off[cell + 1];
    float ax[V], ay[V];
#pragma unroll
    for (int v = 0; v < V; ++v)
      ax[v] = ay[v] = 0.f;
    // a cell boundary: the finished cell lies inside this share (store) or
    // started in an earlier share (head partial)
#define GN_SPMM_FLUSH(KK)                                                      \
  while ((KK) >= bound)                                                        \
  {                                                                            \
    if (s_off[cell] < u0)                                                      \
    {                                                                          \
      _Pragma("unroll") for (int v = 0; v < V; ++v)                            \
          part_head[unit * CG + cl * V + v] = make_float2(ax[v], ay[v]);             \
      if (cl == 0)                                                             \
        head_cell[unit] = cell;                                                \
    }                                                                          \
    else                                                                       \
    {                                                                          \
      _Pragma("unroll") for (int v = 0; v < V; ++v)                            \
          acc[acc_pos<CG, SR2>(cell, cl * V + v)] = make_float2(ax[v], ay[v]);  \
    }                                                                          \
    _Pragma("unroll") for (int v = 0; v < V; ++v) ax[v] = ay[v] = 0.f;        \
    ++cell;                                                                    \
    bound = s_off[cell + 1];                                                   \
  }
  // k-space values of a lane's V coils for sample row q
#define GN_SPMM_LOAD(DST, Q)                                                   \
  if (V == 2)                                                                  \
  {                                                                            \
    const float4 f4 = __ldg(reinterpret_cast<const float4 *>(                  \
        ksg + (Q) * (uint32_t)CP));                                            \
    DST[0] = make_float2(f4.x, f4.y);                                          \
    DST[V - 1] = make_float2(f4.z, f4.w);                                      \
  }                                                                            \
  else                                                                         \
    DST[0] = __ldg(ksg + (Q) * (uint32_t)CP);
    // whole batches of B entries: the next batch's (sample, weight) pairs
    // load while this batch's k-space rows are read
    const uint32_t kfull = u0 + (u1 - u0) / B * B;
    uint32_t k0 = u0;
    if (k0 < kfull)
    {
      uint2 q[B];
#pragma unroll
      for (int u = 0; u < B; ++u)
        q[u] = __ldg(nz + k0 + u);
      for (; k0 < kfull; k0 += B)
      {
        float2 vv[B][V];
#pragma unroll
        for (int u = 0; u < B; ++u)
        {
          GN_SPMM_LOAD(vv[u], q[u].x)
        }
        uint2 qn[B];
#pragma unroll
        for (int u = 0; u < B; ++u)
        {  // clamped: always a valid entry of this share
          const uint32_t kn = k0 + B + u;
          qn[u] = __ldg(nz + (kn < u1 ? kn : u1 - 1));
        }
#pragma unroll
        for (int u = 0; u < B; ++u)
        {
          GN_SPMM_FLUSH(k0 + u)
          const float w = __uint_as_float(q[u].y);
#pragma unroll
          for (int v = 0; v < V; ++v)
          {
            ax[v] = __fmaf_rn(w, vv[u][v].x, ax[v]);
            ay[v] = __fmaf_rn(w, vv[u][v].y, ay[v]);
          }
        }
#pragma unroll
        for (int u = 0; u < B; ++u)
          q[u] = qn[u];
      }
    }
    for (; k0 < u1; ++k0)
    {  // the remainder, one entry at a time
      const uint2 q = __ldg(nz + k0);
      float2 vv[V];
      GN_SPMM_LOAD(vv, q.x)
      GN_SPMM_FLUSH(k0)
      const float w = __uint_as_float(q.y);
#pragma unroll
      for (int v = 0; v < V; ++v)
      {
        ax[v] = __fmaf_rn(w, vv[v].x, ax[v]);
        ay[v] = __fmaf_rn(w, vv[v].y, ay[v]);
      }
    }
#undef GN_SPMM_LOAD
#undef GN_SPMM_FLUSH
    if (s_off[cell] < u0)
    {
#pragma unroll
      for (int v = 0; v < V; ++v)
        part_head[unit * CG + cl * V + v] = make_float2(ax[v], ay[v]);
      if (cl == 0)
        head_cell[unit] = cell;
    }
    else
    {  // the cell started in this share; if it continues in the next
       // shares, this is its first partial sum
#pragma unroll
      for (int v = 0; v < V; ++v)
        acc[acc_pos<CG, SR2>(cell, cl * V + v)] = make_float2(ax[v], ay[v]);
      if (bound > u1 && cl == 0)
        tail_cell[unit] = cell;
    }
  }
  __syncthreads();
  {  // the unit where a cut cell starts adds the continuations in order
    const int tc = tail_cell[unit];
    if (tc >= 0)
    {
#pragma unroll
      for (int v = 0; v < V; ++v)
      {
        const int c = cl * V + v;
        const int pos = acc_pos<CG, SR2>(tc, c);
        float2 sum = acc[pos];
        for (int u = unit + 1; u < NU && head_cell[u] == tc; ++u)
        {
          sum.x = __fadd_rn(sum.x, part_head[u * CG + c].x);
          sum.y = __fadd_rn(sum.y, part_head[u * CG + c].y);
        }
        acc[pos] = sum;
      }
    }
  }
}

// V coils per lane (V = 2 reads a lane's two coils as one 16-byte load and
// halves the per-entry instructions per coil).  One unit: grid row
// (y + G1 * z), chunk of kSpmmCells cells along x, coil group.  Shared
// memory (SpmmSmem): acc [kSpmmCells][CG + 1], offsets [kSpmmCells + 1],
// the cut cells' partial sums [NU][CG] and cell indices [NU] x 2.
template <int CG, int V> struct SpmmSmem
{
  static constexpr int NU = kWarps * (32 / (CG / V));  // streaming units
  static constexpr size_t acc = 0;
  static constexpr size_t part = acc + (size_t)kSpmmCells * (CG + 1) * 8;
  static constexpr size_t off = part + (size_t)NU * CG * 8;
  static constexpr size_t cells = off + ((kSpmmCells + 1) * 4 + 7) / 8 * 8;
  static constexpr size_t bytes = cells + (size_t)2 * NU * 4;
};

template <int CG, int V>
__device__ __forceinline__ void adjoint_spmm_unit(
    int row, int chunk, int group, const uint32_t *__restrict__ row_off,
    const uint2 *__restrict__ nz, const float2 *__restrict__ ks, int CP,
    const Geo &g, int C, int shift, float2 *__restrict__ grid,
    unsigned char *sm)
{
  using L = SpmmSmem<CG, V>;
  constexpr int NU = L::NU;
  float2 *acc_s = reinterpret_cast<float2 *>(sm + L::acc);
  uint32_t *s_off = reinterpret_cast<uint32_t *>(sm + L::off);
  // cells cut by share boundaries: head = the partial sum of the unit's
  // first cell when it started in an earlier share, tail = its last cell
  // when it started in this share and continues in the next
  float2 *part_head = reinterpret_cast<float2 *>(sm + L::part);
  int *head_cell = reinterpret_cast<int *>(sm + L::cells);
  int *tail_cell = head_cell + NU;
  const int x0 = chunk * kSpmmCells;
  const int nxc = min(kSpmmCells, g.G[0] - x0);
  const long long rowbase = (long long)row * g.G[0] + x0;
  for (int i = threadIdx.x; i <= nxc; i += kThreads)
    s_off[i] = __ldg(row_off + rowbase + i);
  __syncthreads();
  const uint32_t A = s_off[0], E = s_off[nxc];
  // output row after the optional INVERSE fftshift
  int y = row % g.G[1], z = row / g.G[1];
  if (shift)
  {
    y = wrap_mod(y - g.shift_inv[1], g.G[1]);
    z = wrap_mod(z - g.shift_inv[2], g.G[2]);
  }
  const long long orow = ((long long)z * g.G[1] + y) * g.G[0];
  if (A == E)
  {  // no sample reaches these cells: plain zero stores
    for (int idx = threadIdx.x; idx < CG * kSpmmCells; idx += kThreads)
    {
      const int cl = idx / kSpmmCells, xi = idx - cl * kSpmmCells;
      const int c = group * CG + cl;
      if (xi >= nxc || c >= C)
        continue;
      int x = x0 + xi;
      if (shift)
        x = wrap_mod(x - g.shift_inv[0], g.G[0]);
      grid[(long long)c * g.grid_count + orow + x] = make_float2(0.f, 0.f);
    }
    return;
  }
  for (int i = threadIdx.x; i < kSpmmCells * (CG + 1); i += kThreads)
    acc_s[i] = make_float2(0.f, 0.f);
  for (int i = threadIdx.x; i < NU; i += kThreads)
    head_cell[i] = tail_cell[i] = -1;
  __syncthreads();

  spmm_accumulate<CG, V>(s_off, nxc, nz, ks, CP, group, acc_s, part_head,
                         head_cell, tail_cell);
  __syncthreads();
  for (int idx = threadIdx.x; idx < CG * kSpmmCells; idx += kThreads)
  {
    const int cl = idx / kSpmmCells, xi = idx - cl * kSpmmCells;
    const int c = group * CG + cl;
    if (xi >= nxc || c >= C)
      continue;
    int x = x0 + xi;
    if (shift)
      x = wrap_mod(x - g.shift_inv[0], g.G[0]);
    grid[(long long)c * g.grid_count + orow + x] = acc_s[xi * (CG + 1) + cl];
  }
}

template <int CG, int V>
__global__ void __launch_bounds__(kThreads, 3)
    k_adjoint_spmm(const uint32_t *__restrict__ row_off,
                   const uint2 *__restrict__ nz, const float2 *__restrict__ ks,
                   int CP, Geo g, int C, int shift, float2 *__restrict__ grid)
{
  __shared__ __align__(16) unsigned char sm[SpmmSmem<CG, V>::bytes];
  adjoint_spmm_unit<CG, V>(blockIdx.x, blockIdx.y, blockIdx.z, row_off, nz,
                           ks, CP, g, C, shift, grid, sm);
}

// --------------------------------------------------------------------------
// adjoint spread of whole grid rows with the inverse x transform fused
// --------------------------------------------------------------------------
// One block per (grid row (z, y), coil group): the row's G_x cells are
// accumulated like k_adjoint_spmm (deterministic, no atomics) into shared
// memory, then each coil's row is transformed along x (inverse DFT, INVERSE
// fftshift of the grid folded into the input index) and only the N_x cropped
// outputs are written: out [C][G_z][G_y][N_x] (rows in the INVERSE-shifted
// frame the next passes expect).  The grid itself is never written.
// With 4 to 32 coils per group (L <= 256) the row transforms run in place on
// the accumulator (coil-swizzled rows, acc_pos), which keeps the block near
// 72 KB at L = 256 and 32 coils (three blocks per SM), near 40 KB with 16
// coils (four blocks per SM) and 22 KB with 8 coils (five blocks per SM, the
// register limit).  At L = 512 (padded rows, up to 16 coils, about 108 KB)
// two blocks share an SM.  Shared memory: acc | roots [L] |
// spread scratch (partial sums, offsets), followed, for the other coil
// groups (acc rows padded to CG + 1), by an exchange area for the
// transform that overlaps the scratch.
// accumulation rows of L x coils complex values stay near 64 KB
constexpr int xfft_max_coils(int L)
{
  return L <= 256 ? 32 : (L == 512 ? 16 : 8);
}

// blocks per SM the spread with the x transform is compiled for (register
// limit 65536 / (256 x blocks)): as many as its shared memory admits where
// that spills few or no registers
constexpr int xfft_min_blocks(int CG, int L)
{
  if (L > 256)
    return L == 512 ? 2 : 1;
  if (CG == 8)
    return L == 256 ? 5 : 4;
  return CG == 16 || CG == 4 ? 4 : 3;
}

template <int CG, int L> struct XfftLayout
{
  using S = fftcore::Shape<L>;
  static constexpr bool IP = CG >= 4 && L <= 256;
  static constexpr int SR2 = IP ? S::R2 : 0;
  static constexpr int ACC = IP ? L * CG : L * (CG + 1);
  static size_t scratch(int NU)
  {
    return (size_t)NU * CG * sizeof(float2) + (size_t)(L + 1) * 4 +
           (size_t)(2 * NU + 2) * 4;
  }
  static size_t smem(int NU)
  {
    const size_t head = (size_t)(ACC + L) * sizeof(float2);
    const size_t exch =
        IP ? 0 : (size_t)S::NL * S::R1 * S::YP * sizeof(float2);
    const size_t sc = scratch(NU);
    return head + (sc > exch ? sc : exch);
  }
};

template <int CG, int V, int L>
__global__ void __launch_bounds__(kThreads, xfft_min_blocks(CG, L))
    k_adjoint_spmm_xfft(const uint32_t *__restrict__ row_off,
                        const uint2 *__restrict__ nz,
                        const float2 *__restrict__ ks, int CP, Geo g, int C,
                        const float2 *__restrict__ roots,
                        float2 *__restrict__ out)
{
  using S = fftcore::Shape<L>;
  using Lay = XfftLayout<CG, L>;
  constexpr bool IP = Lay::IP;
  constexpr int SR2 = Lay::SR2;
  static_assert(S::T * S::NL == kThreads, "one line per T threads");
  static_assert(S::T <= 32, "a line's threads share a warp");
  constexpr int NU = kWarps * (32 / (CG / V));
  extern __shared__ __align__(128) unsigned char smraw[];
  float2 *acc = reinterpret_cast<float2 *>(smraw);
  float2 *tw = acc + Lay::ACC;
  float2 *ex = tw + L;  // scratch, then (padded layout) exchange area
  float2 *part_head = ex;
  uint32_t *s_off = reinterpret_cast<uint32_t *>(part_head + NU * CG);
  int *head_cell = reinterpret_cast<int *>(s_off + L + 1);
  int *tail_cell = head_cell + NU;
  const int row = blockIdx.x;  // y + G1 * z
  const int group = blockIdx.y;
  const int y = wrap_mod(row % g.G[1] - g.shift_inv[1], g.G[1]);
  const int z = wrap_mod(row / g.G[1] - g.shift_inv[2], g.G[2]);
  const long long rowbase = (long long)row * L;
  for (int i = threadIdx.x; i <= L; i += kThreads)
    s_off[i] = __ldg(row_off + rowbase + i);
  fftcore::load_roots(tw, roots, L);
  __syncthreads();
  const bool empty = s_off[0] == s_off[L];
  const int Nx = g.N[0];
  const long long plane = (long long)g.G[2] * g.G[1] * Nx;
  const long long orow = ((long long)z * g.G[1] + y) * Nx;
  if (empty)
  {  // no sample reaches this row: its transform is zero
    for (int i = threadIdx.x; i < CG * Nx; i += kThreads)
    {
      const int cl = i / Nx, x = i - cl * Nx;
      const int c = group * CG + cl;
      if (c < C)
        out[(long long)c * plane + orow + x] = make_float2(0.f, 0.f);
    }
    return;
  }
  // only the empty cells before the row's first and after its last nonzero
  // need zeros (the spread stores every other cell): find both ends, then
  // zero those whole cells (contiguous in either layout)
  int *s_ends = tail_cell + NU;
  for (int i = threadIdx.x; i < L; i += kThreads)
  {
    const uint32_t a = s_off[i], b = s_off[i + 1];
    if (a == s_off[0] && b > a)
      s_ends[0] = i;
    if (a < b && b == s_off[L])
      s_ends[1] = i;
  }
  for (int i = threadIdx.x; i < NU; i += kThreads)
    head_cell[i] = tail_cell[i] = -1;
  __syncthreads();
  {
    constexpr int PITCH = IP ? CG : CG + 1;  // float2 per cell
    float2 *lo_end = acc + (size_t)s_ends[0] * PITCH;
    for (float2 *q = acc + threadIdx.x; q < lo_end; q += kThreads)
      *q = make_float2(0.f, 0.f);
    for (float2 *q = acc + (size_t)(s_ends[1] + 1) * PITCH + threadIdx.x;
         q < acc + (size_t)L * PITCH; q += kThreads)
      *q = make_float2(0.f, 0.f);
  }
  spmm_accumulate<CG, V, SR2, true>(s_off, L, nz, ks, CP, group, acc,
                                    part_head, head_cell, tail_cell);
  __syncthreads();

  // inverse DFT along x of each coil's row, NL coils per pass
  float2 w[fftcore::Rm<L>::V / 2];
  fftcore::load_reg_roots<L>(w, tw);
  const int line = threadIdx.x / S::T, lt = threadIdx.x % S::T;
  // FFT input n holds the cell stored at n: logical x = (n + floor(G/2)),
  // G = L a power of two (the launcher checks shift_inv[0] == L / 2)
  constexpr int sx = L / 2;
  // FFT output k holds image x = (k - crop - floor(G/2)) mod G when < N
  int out_add = (-(g.crop[0] + g.shift_inv[0])) % L;
  if (out_add < 0)
    out_add += L;
  // writes the N_x cropped outputs of a transformed line
  auto store = [&](const float2(&b)[S::R2], int c) {
    float2 *o = out + (long long)c * plane + orow;
#pragma unroll
    for (int k2 = 0; k2 < S::R2; ++k2)
    {
      const int x = (lt + S::R1 * k2 + out_add) & (L - 1);
      if (x < Nx)
        o[x] = b[k2];
    }
  };
  for (int cb = 0; cb < CG; cb += S::NL)
  {
    const int cl = cb + line;
    const int c = group * CG + cl;
    if constexpr (IP)
    {  // in place: a line's R2 stage-1 threads read all their cells, then
       // write the twiddled values to cells k1 * R2 + lt of the same coil
       // column; the line's threads share a warp
      float2 a[S::R1];
      if (lt < S::R2 && cl < CG)
      {
#pragma unroll
        for (int j = 0; j < S::R1; ++j)
          a[j] = acc[acc_pos<CG, SR2>((lt + S::R2 * j + sx) & (L - 1), cl)];
      }
      __syncwarp();
      if (lt < S::R2 && cl < CG)
      {
        fftcore::reg_fft<S::R1, fftcore::Rm<L>::V, true>(a, w);
#pragma unroll
        for (int k1 = 0; k1 < S::R1; ++k1)
        {
          float2 v = a[k1];
          if (k1 != 0)
          {
            float2 r = tw[(lt * k1) & (L - 1)];
            r.y = -r.y;
            v = cmul(v, r);
          }
          acc[acc_pos<CG, SR2>(k1 * S::R2 + lt, cl)] = v;
        }
      }
      __syncwarp();
      if (lt < S::R1 && cl < CG && c < C)
      {
        float2 b[S::R2];
#pragma unroll
        for (int t = 0; t < S::R2; ++t)
          b[t] = acc[acc_pos<CG, SR2>(lt * S::R2 + t, cl)];
        fftcore::reg_fft<S::R2, fftcore::Rm<L>::V, true>(b, w);
        store(b, c);
      }
    }
    else
    {
      float2 *Y = ex + line * S::R1 * S::YP;
      if (lt < S::R2 && cl < CG)
      {
        float2 a[S::R1];
#pragma unroll
        for (int j = 0; j < S::R1; ++j)
          a[j] = acc[((lt + S::R2 * j + sx) & (L - 1)) * (CG + 1) + cl];
        fftcore::stage1<L, true, 1>(a, lt, w, tw, Y);
      }
      __syncthreads();
      if (lt < S::R1 && cl < CG && c < C)
      {
        float2 b[S::R2];
        fftcore::stage2<L, true, 1>(b, lt, w, Y);
        store(b, c);
      }
      __syncthreads();
    }
  }
}

// --------------------------------------------------------------------------
// forward interpolation
// --------------------------------------------------------------------------
// Shared memory: [tile: pad^DIM cells x (CG+1) float2][per-sample geometry
// (DIM ints) and weights (DIM x KS floats)].
// One unit: work item `it`, coil group `group` of CG coils (a power of two
// <= 32: lanes per sample; a constant where the caller has one); smem as
// above.
template <int DIM, int KS>
__device__ __forceinline__ void forward_interp_unit(
    const FwdItem it, int group, const float *__restrict__ traj,
    const uint32_t *__restrict__ idx, const float *__restrict__ dens,
    const float2 *__restrict__ grid, const Geo &g,
    const float *__restrict__ lut, uint32_t M, int C, int shift, float scale,
    float2 *__restrict__ out, float2 *smem, const int CG)
{
  const int SLOTS = 32 / CG;
  const int PITCH = CG + 1;
  constexpr int CH = kThreads;
  const int pad = g.pad;
  const int tcells = DIM == 3 ? pad * pad * pad : pad * pad;
  float2 *tile = smem;
  int *s_b = reinterpret_cast<int *>(smem + (size_t)tcells * PITCH);
  float *s_w = reinterpret_cast<float *>(s_b + DIM * CH);
  int sa[3];
  split_sector(it.sector, g, sa);
  int base[3];
  for (int a = 0; a < 3; ++a)
    base[a] = sa[a] * g.sw + (g.sw >> 1) - g.offset;
  const long long G = g.grid_count;

  // per-axis source offsets of the tile cells (wrap-around and the
  // FORWARD fftshift folded in: the value of cell gw sits at gw + ceil(G/2))
  long long *s_qz = reinterpret_cast<long long *>(
      reinterpret_cast<uintptr_t>(s_w + DIM * KS * CH + 1) & ~uintptr_t(7));
  int *s_qy = reinterpret_cast<int *>(s_qz + pad);
  int *s_qx = s_qy + pad;
  for (int i = threadIdx.x; i < pad; i += kThreads)
  {
    int q[3] = {0, 0, 0};
#pragma unroll
    for (int a = 0; a < DIM; ++a)
    {
      const int gc = base[a] + i;
      int gw = wrap_mod(gc, g.G[a]);
      if (gw < 0 || gw >= g.G[a])
        gw = ((gc % g.G[a]) + g.G[a]) % g.G[a];
      if (shift)
        gw = wrap_mod(gw + g.shift_fwd[a], g.G[a]);
      q[a] = gw;
    }
    s_qx[i] = q[0];
    s_qy[i] = q[1] * g.G[0];
    s_qz[i] = DIM == 3 ? (long long)q[2] * g.G[1] * g.G[0] : 0;
  }
  __syncthreads();
  {
    const int nrows = DIM == 3 ? pad * pad : pad;
    const int lanes_per_row = pad < 32 ? pad : 32;
    const int x0 = threadIdx.x % lanes_per_row;
    const int rstep = kThreads / lanes_per_row;
    const int r0 = threadIdx.x / lanes_per_row;
    if (r0 < rstep)
    {
      for (int cl = 0; cl < CG; ++cl)
      {
        const int c = group * CG + cl;
        const float2 *gcp = grid + (long long)c * G;
        int iy = r0, iz = 0;
        if (DIM == 3)
        {
          iy = r0 % pad;
          iz = r0 / pad;
        }
        const int sy = DIM == 3 ? rstep % pad : 0, sz = DIM == 3 ? rstep / pad : 0;
        for (int r = r0; r < nrows; r += rstep)
        {
          const long long ro = s_qz[iz] + s_qy[iy];
          for (int x = x0; x < pad; x += lanes_per_row)
          {
            float2 *dst = tile + (size_t)(r * pad + x) * PITCH + cl;
            if (c < C)
              cp_async8(dst, gcp + ro + s_qx[x]);
            else
              *dst = make_float2(0.f, 0.f);
          }
          if (DIM == 3)
          {  // advance (iy, iz) by rstep rows without a division
            iy += sy;
            iz += sz;
            if (iy >= pad)
            {
              iy -= pad;
              ++iz;
            }
          }
          else
            iy += rstep;
        }
      }
    }
  }
  cp_async_wait_all();

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int slot = lane / CG, coil = lane % CG;
  const int c = group * CG + coil;
  for (int b0 = it.begin; b0 < it.end; b0 += CH)
  {
    __syncthreads();
    {
      const int t = b0 + threadIdx.x;
#pragma unroll
      for (int a = 0; a < DIM; ++a)
      {
        int l[KS];
        float w[KS];
        int nn = 0;
        if (t < it.end)
          nn = compact_axis<KS>(traj[(size_t)a * M + t], a, sa[a], g, lut, l,
                                w);
        // tile frame: entries are consecutive cells starting at l[0]
        s_b[a * CH + threadIdx.x] = (nn ? l[0] : 0) | (nn << 16);
#pragma unroll
        for (int k = 0; k < KS; ++k)
          s_w[(a * KS + k) * CH + threadIdx.x] = nn ? w[k] : 0.f;
      }
    }
    __syncthreads();
    const int nc = min(CH, it.end - b0);
    for (int i = warp * SLOTS + slot; i < nc; i += kWarps * SLOTS)
    {
      const int bx = s_b[i], by = s_b[CH + i];
      const int x0 = bx & 0xffff, nx = bx >> 16;
      const int y0 = by & 0xffff, ny = by >> 16;
      int z0 = 0, nz = 1;
      if (DIM == 3)
      {
        const int bz = s_b[2 * CH + i];
        z0 = bz & 0xffff;
        nz = bz >> 16;
      }
      float wx[KS];
#pragma unroll
      for (int k = 0; k < KS; ++k)
        wx[k] = s_w[k * CH + i];
      float ax = 0.f, ay = 0.f;
      for (int z = 0; z < nz; ++z)
      {
        const float wz = DIM == 3 ? s_w[(2 * KS + z) * CH + i] : 1.0f;
        for (int y = 0; y < ny; ++y)
        {
          const float wy = s_w[(KS + y) * CH + i];
          const float wzy = DIM == 3 ? __fmul_rn(wz, wy) : wy;
          const int rowb = ((DIM == 3 ? (z0 + z) * pad : 0) + y0 + y) * pad;
          float2 gv[KS];
#pragma unroll
          for (int x = 0; x < KS; ++x)
          {
            if (x >= nx)
              break;
            gv[x] = tile[(size_t)(rowb + x0 + x) * PITCH + coil];
          }
#pragma unroll
          for (int x = 0; x < KS; ++x)
          {
            if (x >= nx)
              break;
            const float w = __fmul_rn(wzy, wx[x]);
            ax = __fmaf_rn(gv[x].x, w, ax);
            ay = __fmaf_rn(gv[x].y, w, ay);
          }
        }
      }
      const int t = b0 + i;
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
}

template <int DIM, int CG, int KS>
__global__ void __launch_bounds__(kThreads)
    k_forward_interp(const FwdItem *__restrict__ items,
                     const float *__restrict__ traj,
                     const uint32_t *__restrict__ idx,
                     const float *__restrict__ dens,
                     const float2 *__restrict__ grid, Geo g,
                     const float *__restrict__ lut, uint32_t M, int C,
                     int shift, float scale, float2 *__restrict__ out)
{
  extern __shared__ float2 smem[];
  forward_interp_unit<DIM, KS>(items[blockIdx.x], blockIdx.y, traj, idx, dens,
                               grid, g, lut, M, C, shift, scale, out, smem,
                               CG);
}

// --------------------------------------------------------------------------
// forward interpolation, tile by TMA (the grid holds the FORWARD-shifted
// spectrum, so a sector tile is one box of the grid unless it wraps)
// --------------------------------------------------------------------------
// Shared memory: tile [CG][PZ][PY][PX] (x fastest; PX = pad + 1 rounded up
// to even, so that the box starts on an even x, i.e. a 16-byte boundary)
// and one mbarrier.  Thread 0 issues one bulk tensor copy of the box at
// (x0, y0, z0, first coil); tiles that wrap around the grid edge are
// gathered with plain loads instead.  Then every thread takes one sample:
// its per-axis footprint (tile frame, upstream arithmetic) in registers,
// and for each footprint cell the CG coil values of the tile.
using tma::kMbarSpin;
using tma::mbar_wait_bounded;
using tma::smem_addr;

template <int DIM, int CG, int KS>
__global__ void __launch_bounds__(kThreads)
    k_forward_tma(const __grid_constant__ CUtensorMap tmap,
                  const FwdItem *__restrict__ items,
                  const float *__restrict__ traj,
                  const uint32_t *__restrict__ idx,
                  const float *__restrict__ dens,
                  const float2 *__restrict__ grid, Geo g,
                  const float *__restrict__ lut, uint32_t M, int C, int PX,
                  float scale, float2 *__restrict__ out, tma::CopyWait cw)
{
  extern __shared__ __align__(128) unsigned char smraw[];
  const int pad = g.pad;
  const int PY = pad, PZ = DIM == 3 ? pad : 1;
  const int cstride = PZ * PY * PX;  // elements per coil
  float2 *tile = reinterpret_cast<float2 *>(smraw);
  uint64_t *mbar = reinterpret_cast<uint64_t *>(
      smraw + (size_t)CG * cstride * sizeof(float2));
  int &s_fail = *reinterpret_cast<int *>(mbar + 1);
  const FwdItem it = items[blockIdx.x];
  const int c0 = blockIdx.y * CG;
  int sa[3];
  split_sector(it.sector, g, sa);
  int base[3] = {0, 0, 0};
  for (int a = 0; a < DIM; ++a)
    base[a] = sa[a] * g.sw + (g.sw >> 1) - g.offset;
  const int x0 = base[0] & ~1;  // even start (floor, negative included)
  const int dx = base[0] - x0;
  bool inside = true;
  for (int a = 0; a < DIM; ++a)
    inside = inside && base[a] >= 0 && base[a] + pad <= g.G[a];
  if (inside)
  {
    const uint32_t bar = smem_addr(mbar);
    if (threadIdx.x == 0)
    {
      s_fail = 0;
      const uint32_t bytes = (uint32_t)(CG * cstride * sizeof(float2));
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar)
                   : "memory");
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
      asm volatile(
          "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
          "r"(bytes)
          : "memory");
      const uint32_t dst = smem_addr(tile);
      const uint64_t tm = reinterpret_cast<uint64_t>(&tmap);
      if (DIM == 3)
        asm volatile(
            "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::"
            "complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
            "l"(tm), "r"(x0), "r"(base[1]), "r"(base[2]), "r"(c0), "r"(bar)
            : "memory");
      else
        asm volatile(
            "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::"
            "complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
            "l"(tm), "r"(x0), "r"(base[1]), "r"(c0), "r"(bar)
            : "memory");
    }
    if (threadIdx.x == 0)
    {  // one thread waits (bounded); the others wait at the barrier below,
       // which orders the copied tile before their reads
      if (!mbar_wait_bounded(bar, 0u, cw.polls))
        s_fail = 1;
    }
    __syncthreads();
    if (s_fail)
    {  // the copy did not complete: report, do not use the tile, and give
       // the copy still in flight a bounded wait before the block's shared
       // memory is released
      if (threadIdx.x == 0)
      {
        atomicExch(cw.err, 1);
        mbar_wait_bounded(bar, 0u);
      }
      return;
    }
  }
  else
  {  // a tile that wraps around the grid edge: plain loads
    const long long G = g.grid_count;
    for (int e = threadIdx.x; e < CG * cstride; e += kThreads)
    {
      const int c = e / cstride;
      int r = e - c * cstride;
      const int z = r / (PY * PX);
      r -= z * PY * PX;
      const int y = r / PX, x = r - y * PX;
      float2 v = make_float2(0.f, 0.f);
      if (c0 + c < C)
      {
        int q[3] = {x0 + x, base[1] + y, DIM == 3 ? base[2] + z : 0};
        for (int a = 0; a < DIM; ++a)
          q[a] = ((q[a] % g.G[a]) + g.G[a]) % g.G[a];
        v = __ldg(grid + (long long)(c0 + c) * G +
                  ((long long)q[2] * g.G[1] + q[1]) * g.G[0] + q[0]);
      }
      tile[e] = v;
    }
    __syncthreads();
  }

  for (int t = it.begin + threadIdx.x; t < it.end; t += kThreads)
  {
    int l[3][KS];
    float w[3][KS];
    int n[3] = {1, 1, 1};
    l[2][0] = 0;
    w[2][0] = 1.f;
#pragma unroll
    for (int a = 0; a < DIM; ++a)
      n[a] = compact_axis<KS>(__ldg(traj + (size_t)a * M + t), a, sa[a], g,
                              lut, l[a], w[a]);
    float2 acc[CG];
#pragma unroll
    for (int c = 0; c < CG; ++c)
      acc[c] = make_float2(0.f, 0.f);
    // tile-frame entries are consecutive cells starting at l[a][0]
    const int xb = l[0][0] + dx;
    for (int z = 0; z < n[2]; ++z)
    {
      float wzv = 1.f;
#pragma unroll
      for (int k = 0; k < KS; ++k)
        if (k == z)
          wzv = w[2][k];
      for (int y = 0; y < n[1]; ++y)
      {
        float wyv = 0.f;
#pragma unroll
        for (int k = 0; k < KS; ++k)
          if (k == y)
            wyv = w[1][k];
        const float wzy = DIM == 3 ? __fmul_rn(wzv, wyv) : wyv;
        const int row = ((DIM == 3 ? (l[2][0] + z) * PY : 0) + l[1][0] + y) *
                            PX + xb;
#pragma unroll
        for (int x = 0; x < KS; ++x)
        {
          if (x < n[0])
          {
            const float wt = __fmul_rn(wzy, w[0][x]);
#pragma unroll
            for (int c = 0; c < CG; ++c)
            {
              const float2 v = tile[c * cstride + row + x];
              acc[c].x = __fmaf_rn(v.x, wt, acc[c].x);
              acc[c].y = __fmaf_rn(v.y, wt, acc[c].y);
            }
          }
        }
      }
    }
    const uint32_t j = __ldg(idx + t);
    const float sd = dens ? sqrtf(__ldg(dens + t)) : 1.0f;
#pragma unroll
    for (int c = 0; c < CG; ++c)
    {
      if (c0 + c < C)
      {
        // performFFTScaling then performDensityCompensation
        // (std_gpuNUFFT_kernels.cu:114-140, 220-242)
        float ax = __fmul_rn(acc[c].x, scale), ay = __fmul_rn(acc[c].y, scale);
        if (dens)
        {
          ax = __fmul_rn(ax, sd);
          ay = __fmul_rn(ay, sd);
        }
        out[(size_t)(c0 + c) * M + j] = make_float2(ax, ay);
      }
    }
  }
}

// The same interpolation with every coil group of an item in one block (3-D
// grids written with coil pairs interleaved, cell q of coil c at
// ((c / 2) * G + q) * 2 + c % 2).  Each thread computes the footprint of
// its samples (kFwdSpt per thread: one for items of up to 256 samples)
// once, in registers; the samples of an item are
// taken in the plan's lane order (build_forward_lane_order), which puts
// samples whose footprints start in different shared-memory bank groups on
// each eight adjacent lanes, so that the 16-byte tile reads of a quarter
// warp, which all lanes make at the same footprint offset, do not collide.
// The block walks the coil groups through a ring of `nbuf` tile buffers; the copy of group g + nbuf is issued as soon
// as group g's buffer is released, so nbuf - 1 copies overlap each group's
// accumulation.  A tile is one 4-D box {2 pad, pad, pad, CG / 2 pairs}
// whose innermost axis runs over x with the two coils of a pair interleaved
// (2 G_x values of 8 bytes): a box row is a tile row of both coils (160
// bytes at pad 10) rather than a single cell, the sector's x start (2 x 8
// bytes per cell) needs no rounding, and one 16-byte shared load reads two
// coils of a cell.  Per sample and coil the arithmetic (cell order z, y, x;
// weight (wz * wy) * wx; one fused multiply-add per cell) is that of
// k_forward_tma.
// Shared memory: nbuf tiles [CG / 2][pad][pad][pad][2] | nbuf mbarriers |
// flag.
constexpr int kFwdSpt = (kFwdItemSamples + kThreads - 1) / kThreads;

// Tile buffers of the coil-pair kernel start on 128-byte boundaries.
__host__ __device__ constexpr int pair_tile_stride(int pad)
{
  return (2 * pad * pad * pad * 16 + 127) / 128 * 8;  // in float4
}

template <int CG, int KS, int MINB>
__global__ void __launch_bounds__(kThreads, MINB)
    k_forward_tma_groups(const __grid_constant__ CUtensorMap tmap,
                         const FwdItem *__restrict__ items,
                         const uint32_t *__restrict__ order,
                         const float *__restrict__ traj,
                         const uint32_t *__restrict__ idx,
                         const float *__restrict__ dens,
                         const float2 *__restrict__ grid, Geo g,
                         const float *__restrict__ lut, uint32_t M, int C,
                         int nbuf, float scale, float2 *__restrict__ out,
                         tma::CopyWait cw)
{
  static_assert(CG % 2 == 0, "coil pairs");
  constexpr int NP = CG / 2;  // coil pairs per group
  extern __shared__ __align__(128) unsigned char smraw[];
  const int pad = g.pad;
  const int pstride = pad * pad * pad;  // cells per pair
  const int tile_cells = NP * pstride;
  static_assert(NP == 2, "buffer stride sized for two pairs");
  const int tstride = pair_tile_stride(pad);  // >= tile_cells
  float4 *tiles = reinterpret_cast<float4 *>(smraw);
  uint64_t *mbar = reinterpret_cast<uint64_t *>(
      smraw + (size_t)nbuf * tstride * sizeof(float4));
  int &s_fail = *reinterpret_cast<int *>(mbar + nbuf);
  const FwdItem it = items[blockIdx.x];
  const int ng = (C + CG - 1) / CG;
  int sa[3];
  split_sector(it.sector, g, sa);
  int base[3];
  for (int a = 0; a < 3; ++a)
    base[a] = sa[a] * g.sw + (g.sw >> 1) - g.offset;
  constexpr int dx = 0;  // the box starts at the sector's own x
  bool inside = true;
  for (int a = 0; a < 3; ++a)
    inside = inside && base[a] >= 0 && base[a] + pad <= g.G[a];
  const uint32_t bar_base = smem_addr(mbar);
  const uint32_t tbytes = (uint32_t)(tile_cells * sizeof(float4));
  const uint64_t tm = reinterpret_cast<uint64_t>(&tmap);
  auto issue = [&](int gi) {  // thread 0: copy coil group gi's tile
    const int b = gi % nbuf;
    const uint32_t bar = bar_base + 8u * (uint32_t)b;
    const uint32_t dst = smem_addr(tiles + (size_t)b * tstride);
    asm volatile(
        "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
        "r"(tbytes)
        : "memory");
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::"
        "complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
        "l"(tm), "r"(2 * base[0]), "r"(base[1]), "r"(base[2]), "r"(gi * NP),
        "r"(bar)
        : "memory");
  };
  if (inside && threadIdx.x == 0)
  {
    s_fail = 0;
    for (int b = 0; b < nbuf; ++b)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(
                       bar_base + 8u * (uint32_t)b)
                   : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    for (int gi = 0; gi < nbuf && gi < ng; ++gi)
      issue(gi);
  }

  // Items of at most kThreads / 2 samples (most of them) run two coil
  // groups at once: the block's halves take groups g and g + 1 (both tile
  // buffers), each thread of a half one sample; larger items walk the
  // groups one at a time.  The copy schedule is the same either way (group
  // g in buffer g % nbuf, its copy issued once group g - nbuf is done).
  const int nsamp = it.end - it.begin;
  const bool two = inside && nbuf == 2 && nsamp <= kThreads / 2;
  const int half = two ? (int)(threadIdx.x / (kThreads / 2)) : 0;
  const int first = two ? (int)(threadIdx.x % (kThreads / 2)) : threadIdx.x;
  // footprint, original position and sqrt(density) of this thread's
  // samples (the item's samples in lane order), kept for all coil groups
  int l0[kFwdSpt][3], n[kFwdSpt][3];
  float w[kFwdSpt][3][KS];
  uint32_t jdst[kFwdSpt];
  float sdv[kFwdSpt];
#pragma unroll
  for (int s = 0; s < kFwdSpt; ++s)
  {
    const int k = it.begin + first + s * kThreads;
    const bool live = k < it.end;
    const uint32_t t = live ? (order ? __ldg(order + k) : (uint32_t)k) : 0u;
    jdst[s] = 0;
    sdv[s] = 1.0f;
    if (live)
    {
      jdst[s] = __ldg(idx + t);
      if (dens)
        sdv[s] = sqrtf(__ldg(dens + t));
    }
#pragma unroll
    for (int a = 0; a < 3; ++a)
    {
      int l[KS];
      n[s][a] = 0;
      if (live)
        n[s][a] = compact_axis<KS>(__ldg(traj + (size_t)a * M + t), a, sa[a],
                                   g, lut, l, w[s][a]);
      else
      {
#pragma unroll
        for (int k2 = 0; k2 < KS; ++k2)
          w[s][a][k2] = 0.f;
        l[0] = 0;
      }
      l0[s][a] = l[0];
    }
  }

  const int step = two ? 2 : 1;
  for (int gi = 0; gi < ng; gi += step)
  {
    const int gn = min(step, ng - gi);  // groups of this phase
    const int gh = gi + half;           // this half's group
    const float4 *tile =
        tiles + (size_t)(inside ? gh % nbuf : 0) * tstride;
    if (inside)
    {
      // the k-th use of a buffer completes phase k of its barrier
      if (threadIdx.x == 0)
        for (int q = gi; q < gi + gn; ++q)
          if (!mbar_wait_bounded(bar_base + 8u * (uint32_t)(q % nbuf),
                                 (uint32_t)(q / nbuf) & 1u, cw.polls))
            s_fail = 1;
      __syncthreads();
      if (s_fail)
      {  // a copy did not complete: report, and give the copies still in
         // flight (groups gi .. gi + nbuf - 1) a bounded wait before the
         // block's shared memory is released
        if (threadIdx.x == 0)
        {
          atomicExch(cw.err, 1);
          for (int q = gi; q < ng && q < gi + nbuf; ++q)
            mbar_wait_bounded(bar_base + 8u * (uint32_t)(q % nbuf),
                              (uint32_t)(q / nbuf) & 1u);
        }
        return;
      }
    }
    else
    {  // a tile that wraps around the grid edge: plain loads (a pair of
       // coils per 16 bytes; the second coil of an odd last pair is zero)
      float4 *dst = tiles;
      const long long G = g.grid_count;
      for (int e = threadIdx.x; e < tile_cells; e += kThreads)
      {
        const int pr = e / pstride;
        int r = e - pr * pstride;
        const int z = r / (pad * pad);
        r -= z * pad * pad;
        const int y = r / pad, x = r - y * pad;
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        const int c = gi * CG + 2 * pr;
        if (c < C)
        {
          int q[3] = {base[0] + x, base[1] + y, base[2] + z};
          for (int a = 0; a < 3; ++a)
            q[a] = ((q[a] % g.G[a]) + g.G[a]) % g.G[a];
          const long long cell =
              ((long long)q[2] * g.G[1] + q[1]) * g.G[0] + q[0];
          v = __ldg(reinterpret_cast<const float4 *>(grid) +
                    (long long)(c >> 1) * G + cell);
          if (c + 1 >= C)
            v.z = v.w = 0.f;
        }
        dst[e] = v;
      }
      __syncthreads();
    }

    // performFFTScaling then performDensityCompensation
    // (std_gpuNUFFT_kernels.cu:114-140, 220-242)
    auto emit = [&](int c, float2 a, int s) {
      const int cc = gh * CG + c;
      if (cc < C)
      {
        float ax = __fmul_rn(a.x, scale), ay = __fmul_rn(a.y, scale);
        if (dens)
        {
          ax = __fmul_rn(ax, sdv[s]);
          ay = __fmul_rn(ay, sdv[s]);
        }
        out[(size_t)cc * M + jdst[s]] = make_float2(ax, ay);
      }
    };
#pragma unroll
    for (int s = 0; s < kFwdSpt; ++s)
    {
      if (gh >= ng || it.begin + first + s * kThreads >= it.end)
        continue;
      float2 acc[CG];
#pragma unroll
      for (int c = 0; c < CG; ++c)
        acc[c] = make_float2(0.f, 0.f);
      // y and x unrolled over the footprint slots with early exits, so that
      // their weights are register reads (no select over the slots)
      const int row0 = (l0[s][2] * pad + l0[s][1]) * pad + l0[s][0] + dx;
      for (int z = 0; z < n[s][2]; ++z)
      {
        float wzv = 0.f;
#pragma unroll
        for (int k = 0; k < KS; ++k)
          if (k == z)
            wzv = w[s][2][k];
#pragma unroll
        for (int y = 0; y < KS; ++y)
        {
          if (y >= n[s][1])
            break;
          const float wzy = __fmul_rn(wzv, w[s][1][y]);
          const int row = row0 + (z * pad + y) * pad;
#pragma unroll
          for (int x = 0; x < KS; ++x)
          {
            if (x >= n[s][0])
              break;
            const float wt = __fmul_rn(wzy, w[s][0][x]);
#pragma unroll
            for (int pr = 0; pr < NP; ++pr)
            {
              const float4 v = tile[pr * pstride + row + x];
              acc[2 * pr].x = __fmaf_rn(v.x, wt, acc[2 * pr].x);
              acc[2 * pr].y = __fmaf_rn(v.y, wt, acc[2 * pr].y);
              acc[2 * pr + 1].x = __fmaf_rn(v.z, wt, acc[2 * pr + 1].x);
              acc[2 * pr + 1].y = __fmaf_rn(v.w, wt, acc[2 * pr + 1].y);
            }
          }
        }
      }
#pragma unroll
      for (int c = 0; c < CG; ++c)
        emit(c, acc[c], s);
    }
    __syncthreads();  // this phase's buffers are free
    if (inside && threadIdx.x == 0)
      for (int q = gi; q < gi + gn; ++q)
        if (q + nbuf < ng)
          issue(q + nbuf);
  }
}

// --------------------------------------------------------------------------
// image-space stages
// --------------------------------------------------------------------------
// Image pixel p of the adjoint from the transformed grid.
template <bool SENS>
__device__ __forceinline__ void finish_pixel(long long p,
                                             const float2 *__restrict__ grid,
                                             const float *__restrict__ deapo,
                                             const float2 *__restrict__ sens,
                                             const Geo &g, int C, int stage,
                                             int accumulate,
                                             float2 *__restrict__ out)
{
  const long long N = g.img_count, G = g.grid_count;
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
        const float2 t = cmul_conj(v, s);
        accx = __fadd_rn(accx, t.x);
        accy = __fadd_rn(accy, t.y);
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
__global__ void k_adjoint_finish(const float2 *__restrict__ grid,
                                 const float *__restrict__ deapo,
                                 const float2 *__restrict__ sens, Geo g, int C,
                                 int stage, int accumulate,
                                 float2 *__restrict__ out)
{
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
       p < g.img_count; p += (long long)gridDim.x * blockDim.x)
    finish_pixel<SENS>(p, grid, deapo, sens, g, C, stage, accumulate, out);
}

// Each block handles grid rows (coil, z, y) with threads along x, two
// cells per thread (16-byte stores).  Rows whose (shifted) position falls
// outside the zero-padded image are pure zero stores.
template <bool SENS>
__device__ __forceinline__ float2 prepare_value(const float2 *__restrict__ image,
                                                const float2 *__restrict__ sens,
                                                const float *__restrict__ deapo,
                                                long long p, long long cN)
{
  float2 v;
  if (SENS)
  {  // sensMulKernel (std_gpuNUFFT_kernels.cu:142-156)
    const float2 a = __ldg(image + p);
    const float2 s = __ldg(sens + p + cN);
    v = cmul(a, s);
  }
  else
  {
    v = __ldg(image + p + cN);
  }
  const float d = __ldg(deapo + p);
  v.x = __fmul_rn(v.x, d);
  v.y = __fmul_rn(v.y, d);
  return v;
}

// Block (y chunk, z, coil - c0): rows of tpr threads each, no index
// division.  With signs (grids even along every axis) each cell (x, y, z)
// is multiplied by (-1)^(x+y+z): the transform then yields the spectrum
// FORWARD-shifted by G/2 = ceil(G/2) on every axis, whose sector tiles are
// boxes of the grid.
// One unit: rows yb * rpb .. of plane z of coil c.
template <bool SENS>
__device__ __forceinline__ void prepare_unit(
    int yb, int z, int c, const float2 *__restrict__ image,
    const float2 *__restrict__ sens, const float *__restrict__ deapo,
    const Geo &g, int image_grid, int signs, int tpr,
    float2 *__restrict__ grid)
{
  const int X = image_grid ? g.N[0] : g.G[0];
  const int Y = image_grid ? g.N[1] : g.G[1];
  const int Z = image_grid ? g.N[2] : g.G[2];
  const long long N = g.img_count;
  const long long plane = (long long)X * Y * Z;
  const int X2 = X >> 1;  // cell pairs per row
  const bool vec = (X & 1) == 0;
  const int rpb = kThreads / tpr;  // rows per block
  const int lr = threadIdx.x / tpr, lt = threadIdx.x - lr * tpr;
  const int y = yb * rpb + lr;
  if (lr >= rpb || y >= Y)
    return;
  float2 *dst = grid + (long long)c * plane + ((long long)z * Y + y) * X;
  int py = y, pz = z;
  if (!image_grid)
  {
    // INVERSE fftshift of the padded grid: shifted[q] = padded[q+floor(G/2)]
    py = wrap_mod(y + g.shift_inv[1], g.G[1]) - g.crop[1];
    pz = wrap_mod(z + g.shift_inv[2], g.G[2]) - g.crop[2];
  }
  const bool row_in = py >= 0 && py < g.N[1] && pz >= 0 && pz < g.N[2];
  const long long prow = ((long long)pz * g.N[1] + py) * g.N[0];
  const long long cN = (long long)c * N;
  const bool odd_row = ((y + z) & 1) != 0;
  if (vec)
  {
    // even rows start on even cells: 16-byte aligned pairs
    float4 *d4 = reinterpret_cast<float4 *>(dst);
    for (int j = lt; j < X2; j += tpr)
    {
      float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
      if (row_in)
      {
        const int xa = 2 * j;
        const int pa = image_grid ? xa
                                  : wrap_mod(xa + g.shift_inv[0], g.G[0]) -
                                        g.crop[0];
        const int pb = image_grid ? xa + 1
                                  : wrap_mod(xa + 1 + g.shift_inv[0],
                                             g.G[0]) -
                                        g.crop[0];
        if (pa >= 0 && pa < g.N[0])
        {
          const float2 v = prepare_value<SENS>(image, sens, deapo, prow + pa,
                                               cN);
          o.x = v.x;
          o.y = v.y;
        }
        if (pb >= 0 && pb < g.N[0])
        {
          const float2 v = prepare_value<SENS>(image, sens, deapo, prow + pb,
                                               cN);
          o.z = v.x;
          o.w = v.y;
        }
        if (signs)
        {  // cells 2j and 2j + 1 of this row: opposite signs
          if (odd_row)
          {
            o.x = -o.x;
            o.y = -o.y;
          }
          else
          {
            o.z = -o.z;
            o.w = -o.w;
          }
        }
      }
      d4[j] = o;
    }
  }
  else
  {
    for (int x = lt; x < X; x += tpr)
    {
      float2 v = make_float2(0.f, 0.f);
      if (row_in)
      {
        const int px = image_grid ? x
                                  : wrap_mod(x + g.shift_inv[0], g.G[0]) -
                                        g.crop[0];
        if (px >= 0 && px < g.N[0])
          v = prepare_value<SENS>(image, sens, deapo, prow + px, cN);
        if (signs && (((x & 1) != 0) != odd_row))
          v = make_float2(-v.x, -v.y);
      }
      dst[x] = v;
    }
  }
}

template <bool SENS>
__global__ void __launch_bounds__(kThreads)
    k_forward_prepare(const float2 *__restrict__ image,
                      const float2 *__restrict__ sens,
                      const float *__restrict__ deapo, Geo g, int c0,
                      int image_grid, int signs, int tpr,
                      float2 *__restrict__ grid)
{
  prepare_unit<SENS>(blockIdx.x, blockIdx.y, c0 + blockIdx.z, image, sens,
                     deapo, g, image_grid, signs, tpr, grid);
}

template <typename K>
void set_smem(K kernel, size_t bytes)
{
  if (bytes > 48 * 1024)
    GN_CUDA(cudaFuncSetAttribute(kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)bytes));
}

template <int DIM, int CG, int KS>
void fwd_dispatch(const FwdItem *items, int n_items, const float *traj,
                  const uint32_t *idx, const float *dens, const float2 *grid,
                  const Geo &g, const float *lut, uint32_t M, int C,
                  bool shift, float scale, float2 *out, cudaStream_t s)
{
  const size_t smem = forward_smem_bytes(g, CG);
  auto k = k_forward_interp<DIM, CG, KS>;
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

// footprint slots per axis: kw + 1 cells
int slots_for(const Geo &g) { return g.kw + 1 <= 4 ? 4 : 8; }

// --------------------------------------------------------------------------
// batches: one persistent launch per stage over all instances
// --------------------------------------------------------------------------
constexpr int kBatchSlots = 8;
// Copies instance i's descriptor into shared memory (all threads; a
// barrier follows) unless it is already there.
__device__ __forceinline__ void batch_load(const BatchInst *__restrict__ inst,
                                           int i, BatchInst *s_b, int *s_cur)
{
  if (*s_cur == i)
    return;
  constexpr int W = (int)(sizeof(BatchInst) / 4);
  const uint32_t *src = reinterpret_cast<const uint32_t *>(inst + i);
  uint32_t *dst = reinterpret_cast<uint32_t *>(s_b);
  __syncthreads();
  for (int k = threadIdx.x; k < W; k += kThreads)
    dst[k] = __ldg(src + k);
  __syncthreads();
  if (threadIdx.x == 0)
    *s_cur = i;  // read again only after the next unit's barriers
}

// The unit loop of a batch stage: thread 0 takes the next unit index from
// the counter, the block finds its instance (last one whose first unit is
// <= the index) and runs body(instance, unit within the instance) with the
// descriptor in shared memory.  Ends when the counter passes `total`.
template <class F>
__device__ __forceinline__ void batch_loop(const BatchInst *__restrict__ inst,
                                           int n, int stage, uint32_t total,
                                           unsigned *counter, F body)
{
  __shared__ uint32_t s_first[kBatchMax + 1];
  __shared__ uint32_t s_u;
  __shared__ int s_cur;
  __shared__ BatchInst s_b;
  for (int i = threadIdx.x; i < n; i += kThreads)
    s_first[i] = __ldg(&inst[i].first[stage]);
  if (threadIdx.x == 0)
  {
    s_first[n] = total;
    s_cur = -1;
  }
  for (;;)
  {
    __syncthreads();  // the previous unit is done with shared memory
    if (threadIdx.x == 0)
      s_u = atomicAdd(counter, 1u);
    __syncthreads();
    const uint32_t u = s_u;
    if (u >= total)
      return;
    int lo = 0, hi = n;  // s_first[lo] <= u < s_first[hi]
    while (hi - lo > 1)
    {
      const int mid = (lo + hi) >> 1;
      if (s_first[mid] <= u)
        lo = mid;
      else
        hi = mid;
    }
    batch_load(inst, lo, &s_b, &s_cur);
    body(lo, u - s_first[lo], s_b);
  }
}

__global__ void __launch_bounds__(kThreads)
    k_batch_prepare(const BatchInst *__restrict__ inst, int n, uint32_t total,
                    unsigned *counter, const __grid_constant__ BatchIo io)
{
  batch_loop(inst, n, kBatchPrepare, total, counter,
             [&](int i, uint32_t u, const BatchInst &b) {
               const int rpb = kThreads / b.tpr;
               const uint32_t nyb = (b.g.G[1] + rpb - 1) / rpb;
               const uint32_t Z = b.g.G[2];
               const int yb = (int)(u % nyb), z = (int)((u / nyb) % Z);
               const int c = (int)(u / (nyb * Z));
               if (b.sens)
                 prepare_unit<true>(yb, z, c, io.in[i], b.sens, b.deapo, b.g,
                                    0, b.signs, b.tpr, b.grid);
               else
                 prepare_unit<false>(yb, z, c, io.in[i], nullptr, b.deapo,
                                     b.g, 0, b.signs, b.tpr, b.grid);
             });
}

template <int DIM, int KS>
__device__ __forceinline__ void batch_interp_unit(const BatchInst &b,
                                                  uint32_t u, float2 *out,
                                                  float2 *smem)
{
  const uint32_t ng = (b.C + b.fwd_cg - 1) / b.fwd_cg;
  forward_interp_unit<DIM, KS>(b.items[u / ng], (int)(u % ng), b.traj, b.di,
                               b.dens, b.grid, b.g, b.lut, b.M, b.C,
                               b.signs ? 0 : 1, b.g.fft_scale, out, smem,
                               b.fwd_cg);
}

// One launch per dimensionality (its own unit list); 8 footprint slots
// (kernel widths up to 7) for every instance, so that each launch holds a
// single instantiation of the interpolation.
template <int DIM>
__global__ void __launch_bounds__(kThreads, 3)
    k_batch_interp(const BatchInst *__restrict__ inst, int n, uint32_t total,
                   unsigned *counter, const __grid_constant__ BatchIo io)
{
  extern __shared__ float2 smem[];
  batch_loop(inst, n, DIM == 2 ? kBatchInterp : kBatchInterp3, total, counter,
             [&](int i, uint32_t u, const BatchInst &b) {
               batch_interp_unit<DIM, kBatchSlots>(b, u, io.out[i], smem);
             });
}

__global__ void __launch_bounds__(kThreads)
    k_batch_gather(const BatchInst *__restrict__ inst, int n, uint32_t total,
                   unsigned *counter, const __grid_constant__ BatchIo io)
{
  batch_loop(inst, n, kBatchGather, total, counter,
             [&](int i, uint32_t u, const BatchInst &b) {
               const uint32_t nj = (b.M + kGatherSamples - 1) / kGatherSamples;
               gather_inv_unit((int)(u % nj), (int)(u / nj), io.in[i],
                               b.di_inv, b.dens, b.M, b.C, b.CP, b.ks);
             });
}

__host__ __device__ constexpr size_t batch_spread_smem()
{
  size_t m = SpmmSmem<1, 1>::bytes;
  m = m > SpmmSmem<2, 1>::bytes ? m : SpmmSmem<2, 1>::bytes;
  m = m > SpmmSmem<4, 2>::bytes ? m : SpmmSmem<4, 2>::bytes;
  m = m > SpmmSmem<8, 2>::bytes ? m : SpmmSmem<8, 2>::bytes;
  m = m > SpmmSmem<16, 2>::bytes ? m : SpmmSmem<16, 2>::bytes;
  m = m > SpmmSmem<32, 2>::bytes ? m : SpmmSmem<32, 2>::bytes;
  return m;
}

__global__ void __launch_bounds__(kThreads, 3)
    k_batch_spread(const BatchInst *__restrict__ inst, int n, uint32_t total,
                   unsigned *counter)
{
  __shared__ __align__(16) unsigned char sm[batch_spread_smem()];
  batch_loop(inst, n, kBatchSpread, total, counter,
             [&](int, uint32_t u, const BatchInst &b) {
               const uint32_t rows = (uint32_t)b.g.G[1] * b.g.G[2];
               const uint32_t nch = (b.g.G[0] + kSpmmCells - 1) / kSpmmCells;
               const int row = (int)(u % rows);
               const int ch = (int)((u / rows) % nch);
               const int grp = (int)(u / (rows * nch));
#define GN_BSPMM(CGV, VV)                                                      \
  adjoint_spmm_unit<CGV, VV>(row, ch, grp, b.w_rows, b.w_nz, b.ks, b.CP, b.g,  \
                             b.C, 1, b.grid, sm)
               switch (b.spmm_cg)
               {
               case 1: GN_BSPMM(1, 1); break;
               case 2: GN_BSPMM(2, 1); break;
               case 4: GN_BSPMM(4, 2); break;
               case 8: GN_BSPMM(8, 2); break;
               case 16: GN_BSPMM(16, 2); break;
               default: GN_BSPMM(32, 2); break;
               }
#undef GN_BSPMM
             });
}

__global__ void __launch_bounds__(kThreads)
    k_batch_finish(const BatchInst *__restrict__ inst, int n, uint32_t total,
                   unsigned *counter, const __grid_constant__ BatchIo io)
{
  batch_loop(inst, n, kBatchFinish, total, counter,
             [&](int i, uint32_t u, const BatchInst &b) {
               const long long p = (long long)u * kThreads + threadIdx.x;
               if (p >= b.g.img_count)
                 return;
               if (b.sens)
                 finish_pixel<true>(p, b.grid, b.deapo, b.sens, b.g, b.C, 2,
                                    0, io.out[i]);
               else
                 finish_pixel<false>(p, b.grid, b.deapo, nullptr, b.g, b.C, 2,
                                     0, io.out[i]);
             });
}
}  // namespace

int spmm_coil_group(int C) { return C > 16 ? 32 : pow2_at_least(C); }

bool gridding_supported(const Geo &g, std::string &why)
{
  if (g.sw > kMaxSectorWidth)
  {
    why = "sector width above 32 is not supported";
    return false;
  }
  if (forward_smem_bytes(g, 1) > 200 * 1024)
  {
    why = "sector tile exceeds shared memory (3-D sector width too large)";
    return false;
  }
  return true;
}

int forward_coil_group(int C, int dim, int pad)
{
  int cg = C > 8 ? 8 : pow2_at_least(C);
  // keep the tile + halo within shared memory
  const size_t cells = dim == 3 ? (size_t)pad * pad * pad : (size_t)pad * pad;
  while (cg > 1 && cells * (cg + 1) * sizeof(float2) > 160 * 1024)
    cg >>= 1;
  if (dim == 2)
    cg = C > 16 ? 32 : pow2_at_least(C);
  return cg;
}

size_t forward_smem_bytes(const Geo &g, int cg)
{
  const size_t cells = g.dim == 3 ? (size_t)g.pad * g.pad * g.pad
                                  : (size_t)g.pad * g.pad;
  const int ks = g.kw + 1 <= 4 ? 4 : 8;
  return cells * (cg + 1) * sizeof(float2) +
         (size_t)kThreads * (g.dim + g.dim * ks) * 4 + 8 + (size_t)g.pad * 16;
}

void launch_gather_kspace_inv(const float2 *kspace, const uint32_t *inv,
                              const float *dens_sorted, uint32_t M, int C,
                              int CP, float2 *ks, cudaStream_t s)
{
  if (!M)
    return;
  dim3 grd((M + kGatherSamples - 1) / kGatherSamples,
           (CP + kGatherCoils - 1) / kGatherCoils);
  k_gather_kspace_inv<<<grd, kThreads, 0, s>>>(kspace, inv, dens_sorted, M,
                                               C, CP, ks);
  GN_LAUNCH_CHECK("gather k-space (original order)");
}

void launch_invert_permutation(const uint32_t *idx, uint32_t M,
                               uint32_t *inv, cudaStream_t s)
{
  if (!M)
    return;
  k_invert<<<grid_for(M, 256, 8192), 256, 0, s>>>(idx, M, inv);
  GN_LAUNCH_CHECK("invert permutation");
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


void launch_adjoint_spmm(const uint32_t *row_off, const uint2 *nz,
                         const float2 *ks, int CP, const Geo &g, int C,
                         bool shift, float2 *grid, cudaStream_t s)
{
  const int cg = spmm_coil_group(C);
  dim3 grd(g.G[1] * g.G[2], (g.G[0] + kSpmmCells - 1) / kSpmmCells,
           (C + cg - 1) / cg);
#define GN_SPMM(CGV, VV)                                                       \
  k_adjoint_spmm<CGV, VV><<<grd, kThreads, 0, s>>>(row_off, nz, ks, CP, g, C, \
                                                   shift ? 1 : 0, grid)
  switch (cg)
  {
  case 1: GN_SPMM(1, 1); break;
  case 2: GN_SPMM(2, 1); break;
  case 4: GN_SPMM(4, 2); break;
  case 8: GN_SPMM(8, 2); break;
  case 16: GN_SPMM(16, 2); break;
  default: GN_SPMM(32, 2); break;
  }
#undef GN_SPMM
  GN_LAUNCH_CHECK("adjoint spmm");
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
                            bool image_grid, float2 *grid, cudaStream_t s,
                            bool signs)
{
  const int X = image_grid ? g.N[0] : g.G[0];
  const int Y = image_grid ? g.N[1] : g.G[1];
  const int Z = image_grid ? g.N[2] : g.G[2];
  // threads per row: 16-byte stores of cell pairs (single cells for odd
  // rows), at most 64 threads so that short rows still fill the block
  const int work = (X & 1) == 0 ? X / 2 : X;
  const int tpr = work >= 64 ? 64 : (work > 0 ? work : 1);
  const int rpb = kThreads / tpr;
  for (int c0 = 0; c0 < C; c0 += 65535)
  {
    const dim3 grd((unsigned)((Y + rpb - 1) / rpb), (unsigned)Z,
                   (unsigned)std::min(C - c0, 65535));
    if (sens)
      k_forward_prepare<true><<<grd, kThreads, 0, s>>>(
          image, sens, deapo, g, c0, image_grid, signs ? 1 : 0, tpr, grid);
    else
      k_forward_prepare<false><<<grd, kThreads, 0, s>>>(
          image, nullptr, deapo, g, c0, image_grid, signs ? 1 : 0, tpr,
          grid);
  }
  GN_LAUNCH_CHECK("forward prepare");
}

void launch_forward_interp(const FwdItem *items, int n_items,
                           const float *traj_sorted, const uint32_t *idx,
                           const float *dens_sorted, const float2 *grid,
                           const Geo &g, const float *lut, uint32_t M, int C,
                           bool shift, float scale, float2 *out,
                           cudaStream_t s, int tile_coils)
{
  if (n_items <= 0)
    return;
  int cg = forward_coil_group(C, g.dim, g.pad);
  if (tile_coils > 0)
  {  // tuned tile shape, reduced until it fits in shared memory
    cg = tile_coils > 32 ? 32 : tile_coils;
    while (cg > 1 && forward_smem_bytes(g, cg) > 200 * 1024)
      cg >>= 1;
  }
#define GN_FWD(D, CGV)                                                         \
  if (slots_for(g) == 4)                                                       \
    fwd_dispatch<D, CGV, 4>(items, n_items, traj_sorted, idx, dens_sorted,    \
                            grid, g, lut, M, C, shift, scale, out, s);        \
  else                                                                         \
    fwd_dispatch<D, CGV, 8>(items, n_items, traj_sorted, idx, dens_sorted,    \
                            grid, g, lut, M, C, shift, scale, out, s)
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


using tma::EncodeTiledFn;
using tma::encode_fn;

bool forward_pairs(const Geo &g, int tile_coils)
{
  // 3-D, the z transform with tensor-copy tiles (every axis <= 256), kernel
  // width <= 3 (four footprint slots), tiles of four coils, two pairs of
  // tiles within three blocks' shared memory per SM
  if (g.dim != 3 || slots_for(g) != 4 || !encode_fn())
    return false;
  for (int a = 0; a < 3; ++a)
    if (g.G[a] > 256 || g.G[a] < 16)
      return false;
  if (tile_coils > 0 && tile_coils != 4)
    return false;
  const size_t tile = (size_t)pair_tile_stride(g.pad) * 16;
  return 2 * tile + 64 <= 74 * 1024;
}

// One block per work item: the bank group (16-byte unit mod 8) of each
// sample's first footprint cell in the coil-pair tile, then the samples
// dealt round-robin over the eight groups: position = the samples of lower
// rank within their group, plus those of equal rank in lower groups.  Each
// run of eight lanes then holds eight groups while all of them have
// samples left.  Only the lanes' order changes: every sample's arithmetic
// is the same in any position.
template <int KS>
__global__ void __launch_bounds__(kThreads)
    k_forward_lane_order(const FwdItem *__restrict__ items,
                         const float *__restrict__ traj, uint32_t M, Geo g,
                         const float *__restrict__ lut,
                         uint32_t *__restrict__ order)
{
  __shared__ unsigned char s_bank[kFwdItemSamples];
  __shared__ int s_cnt[8];
  const FwdItem it = items[blockIdx.x];
  const int n = it.end - it.begin;
  int sa[3];
  split_sector(it.sector, g, sa);
  if (threadIdx.x < 8)
    s_cnt[threadIdx.x] = 0;
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += kThreads)
  {
    int l0[3];
    for (int a = 0; a < 3; ++a)
    {
      int l[KS];
      float w[KS];
      const int nn = compact_axis<KS>(
          __ldg(traj + (size_t)a * M + it.begin + k), a, sa[a], g, lut, l, w);
      l0[a] = nn ? l[0] : 0;
    }
    const int bank = ((l0[2] * g.pad + l0[1]) * g.pad + l0[0]) & 7;
    s_bank[k] = (unsigned char)bank;
    atomicAdd(&s_cnt[bank], 1);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += kThreads)
  {
    const int b = s_bank[k];
    int rank = 0;
    for (int u = 0; u < k; ++u)
      rank += s_bank[u] == b;
    int pos = 0;
    for (int q = 0; q < 8; ++q)
      pos += min(s_cnt[q], rank) + (q < b && s_cnt[q] > rank);
    order[it.begin + pos] = (uint32_t)(it.begin + k);
  }
}

void build_forward_lane_order(const FwdItem *items, int n_items,
                              const float *traj_sorted, uint32_t M,
                              const Geo &g, const float *lut, uint32_t *order,
                              cudaStream_t s)
{
  if (n_items <= 0)
    return;
  if (slots_for(g) == 4)
    k_forward_lane_order<4><<<(unsigned)n_items, kThreads, 0, s>>>(
        items, traj_sorted, M, g, lut, order);
  else
    k_forward_lane_order<8><<<(unsigned)n_items, kThreads, 0, s>>>(
        items, traj_sorted, M, g, lut, order);
  GN_LAUNCH_CHECK("forward lane order");
}

bool launch_forward_interp_tma(const FwdItem *items, int n_items,
                               const float *traj_sorted, const uint32_t *idx,
                               const float *dens_sorted, const float2 *grid,
                               const Geo &g, const float *lut, uint32_t M,
                               int C, float scale, float2 *out,
                               tma::CopyWait cw, cudaStream_t s,
                               int tile_coils, bool paired,
                               const uint32_t *lane_order)
{
  if (n_items <= 0)
    return true;
  if (paired)
  {  // coil-pair grid: every coil group of an item in one block, a ring of
     // two tile buffers, three blocks per SM
    EncodeTiledFn enc = encode_fn();
    if (!enc)
      return false;
    const int pad = g.pad;
    const int pairs = (C + 1) / 2;
    CUtensorMap tm;
    // the coil of a pair and x merged into one axis of 2 G_x values: a box
    // row is a tile row of both coils (2 pad x 8 bytes), not one cell
    cuuint64_t dims[4] = {2 * (cuuint64_t)g.G[0], (cuuint64_t)g.G[1],
                          (cuuint64_t)g.G[2], (cuuint64_t)pairs};
    cuuint64_t strides[3];
    strides[0] = 2 * sizeof(float2) * (cuuint64_t)g.G[0];
    strides[1] = strides[0] * g.G[1];
    strides[2] = strides[1] * g.G[2];
    cuuint32_t box[4] = {2 * (cuuint32_t)pad, (cuuint32_t)pad,
                         (cuuint32_t)pad, 2};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    if (enc(&tm, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4, const_cast<float2 *>(grid),
            dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      throw Error(kInternal, "coil-pair grid tensor map rejected");
    const int nbuf = 2;
    const size_t tile = (size_t)pair_tile_stride(pad) * sizeof(float4);
    const size_t smem2 = (size_t)nbuf * tile + 8 * nbuf + 16;
    auto k = k_forward_tma_groups<4, 4, 3>;
    GN_CUDA(cudaFuncSetAttribute(
        k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
    k<<<(unsigned)n_items, kThreads, smem2, s>>>(
        tm, items, lane_order, traj_sorted, idx, dens_sorted, grid, g, lut, M,
        C, nbuf, scale, out, cw);
    GN_LAUNCH_CHECK("forward interpolation (coil-pair tiles, all groups)");
    return true;
  }
  EncodeTiledFn enc = encode_fn();
  if (!enc || (g.G[0] & 1))
    return false;
  const int pad = g.pad;
  const int PX = (pad + 2) & ~1;  // pad + 1 rounded up to even
  // coils per tile: a power of two, at most C (the box stays inside the
  // coil extent) and at most 4 in 3-D (64 KB tiles, three blocks per SM)
  const int cmax = std::min(C, tile_coils > 0
                                   ? std::min(tile_coils, g.dim == 3 ? 4 : 32)
                                   : (g.dim == 3 ? 4 : 32));
  int cg = 1;
  while (cg * 2 <= cmax)
    cg <<= 1;
  const int PZ = g.dim == 3 ? pad : 1;
  const size_t tile = (size_t)cg * PZ * pad * PX * sizeof(float2);
  const size_t smem = tile + 16;
  if (smem > 200 * 1024 || PX > 256 || pad > 256)
    return false;
  CUtensorMap tm;
  cuuint64_t dims[4], strides[3];
  cuuint32_t box[4], estr[4] = {1, 1, 1, 1};
  const int rank = g.dim + 1;
  dims[0] = g.G[0];
  dims[1] = g.G[1];
  strides[0] = (cuuint64_t)g.G[0] * sizeof(float2);
  box[0] = PX;
  box[1] = pad;
  if (g.dim == 3)
  {
    dims[2] = g.G[2];
    dims[3] = C;
    strides[1] = strides[0] * g.G[1];
    strides[2] = strides[1] * g.G[2];
    box[2] = pad;
    box[3] = cg;
  }
  else
  {
    dims[2] = C;
    strides[1] = strides[0] * g.G[1];
    box[2] = cg;
  }
  if (enc(&tm, CU_TENSOR_MAP_DATA_TYPE_UINT64, rank,
          const_cast<float2 *>(grid), dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
          CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return false;
  const int ks = slots_for(g);
  const dim3 grd((unsigned)n_items, (unsigned)((C + cg - 1) / cg));
#define GN_TMA(D, CGV, KSV)                                                    \
  {                                                                            \
    auto k = k_forward_tma<D, CGV, KSV>;                                       \
    if (smem > 48 * 1024)                                                      \
      GN_CUDA(cudaFuncSetAttribute(                                            \
          k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));         \
    k<<<grd, kThreads, smem, s>>>(tm, items, traj_sorted, idx, dens_sorted,    \
                                  grid, g, lut, M, C, PX, scale, out, cw);     \
  }
#define GN_TMA_KS(D, CGV)                                                      \
  if (ks == 4)                                                                 \
    GN_TMA(D, CGV, 4)                                                          \
  else                                                                         \
    GN_TMA(D, CGV, 8)
  if (g.dim == 3)
  {
    switch (cg)
    {
    case 1: GN_TMA_KS(3, 1); break;
    case 2: GN_TMA_KS(3, 2); break;
    default: GN_TMA_KS(3, 4); break;
    }
  }
  else
  {
    switch (cg)
    {
    case 1: GN_TMA_KS(2, 1); break;
    case 2: GN_TMA_KS(2, 2); break;
    case 4: GN_TMA_KS(2, 4); break;
    case 8: GN_TMA_KS(2, 8); break;
    case 16: GN_TMA_KS(2, 16); break;
    default: GN_TMA_KS(2, 32); break;
    }
  }
#undef GN_TMA_KS
#undef GN_TMA
  GN_LAUNCH_CHECK("forward interpolation (tensor-copy tiles)");
  return true;
}


int spmm_xfft_coils(int L) { return xfft_max_coils(L); }

bool launch_adjoint_spmm_xfft(const uint32_t *row_off, const uint2 *nz,
                              const float2 *ks, int CP, const Geo &g, int C,
                              const float2 *roots_x, float2 *out,
                              cudaStream_t s)
{
  const int L = g.G[0];
  if (L < 16 || L > 1024 || (L & (L - 1)) || g.shift_inv[0] != L / 2)
    return false;
  const int cgmax = spmm_xfft_coils(L);
  // the spread's coil group must divide the k-space lane count CP
  int cg = spmm_coil_group(C);
  if (cg > cgmax)
    cg = cgmax;
  if (CP % cg)
    return false;
  const dim3 grd((unsigned)((long long)g.G[1] * g.G[2]),
                 (unsigned)((C + cg - 1) / cg));
  bool ok = true;
  auto go = [&](auto lc, auto cgc, auto vc) {
    constexpr int LL = decltype(lc)::value;
    constexpr int CGV = decltype(cgc)::value;
    constexpr int VV = decltype(vc)::value;
    if constexpr (CGV > xfft_max_coils(LL))
    {  // never selected (the coil group is capped above)
      ok = false;
      return;
    }
    else
    {
      constexpr int NU = kWarps * (32 / (CGV / VV));
      const size_t smem = XfftLayout<CGV, LL>::smem(NU);
      if (smem > 220 * 1024)
      {
        ok = false;
        return;
      }
      auto k = k_adjoint_spmm_xfft<CGV, VV, LL>;
      GN_CUDA(cudaFuncSetAttribute(
          k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k<<<grd, kThreads, smem, s>>>(row_off, nz, ks, CP, g, C, roots_x, out);
    }
  };
  using I = std::integral_constant<int, 1>;
  using I2 = std::integral_constant<int, 2>;
  auto with_cg = [&](auto lc) {
    switch (cg)
    {
    case 1: go(lc, std::integral_constant<int, 1>(), I()); break;
    case 2: go(lc, std::integral_constant<int, 2>(), I()); break;
    case 4: go(lc, std::integral_constant<int, 4>(), I2()); break;
    case 8: go(lc, std::integral_constant<int, 8>(), I2()); break;
    case 16: go(lc, std::integral_constant<int, 16>(), I2()); break;
    default: go(lc, std::integral_constant<int, 32>(), I2()); break;
    }
  };
  switch (L)
  {
  case 16: with_cg(std::integral_constant<int, 16>()); break;
  case 32: with_cg(std::integral_constant<int, 32>()); break;
  case 64: with_cg(std::integral_constant<int, 64>()); break;
  case 128: with_cg(std::integral_constant<int, 128>()); break;
  case 256: with_cg(std::integral_constant<int, 256>()); break;
  case 512: with_cg(std::integral_constant<int, 512>()); break;
  default: with_cg(std::integral_constant<int, 1024>()); break;
  }
  if (!ok)
    return false;
  GN_LAUNCH_CHECK("adjoint spread with x transform");
  return true;
}

// --------------------------------------------------------------------------
// batches (host side)
// --------------------------------------------------------------------------
void batch_configure(BatchInst &b, int tile_coils)
{
  const Geo &g = b.g;
  b.spmm_cg = spmm_coil_group(b.C);
  b.CP = (b.C + b.spmm_cg - 1) / b.spmm_cg * b.spmm_cg;
  b.slots = kBatchSlots;
  int cg = forward_coil_group(b.C, g.dim, g.pad);
  if (tile_coils > 0)
    cg = tile_coils > 32 ? 32 : pow2_at_least(tile_coils);
  if (g.dim == 3 && cg > 8)
    cg = 8;
  b.fwd_cg = cg;
  // tiles within 72 KB keep three blocks of the interpolation stage per SM
  while (b.fwd_cg > 1 && batch_interp_smem(b) > 72 * 1024)
    b.fwd_cg >>= 1;
  const int X = g.G[0];
  const int work = (X & 1) == 0 ? X / 2 : X;
  b.tpr = work >= 64 ? 64 : (work > 0 ? work : 1);
}

void batch_units(const BatchInst &b, uint32_t units[kBatchStages])
{
  const Geo &g = b.g;
  const uint32_t rpb = kThreads / b.tpr;
  units[kBatchPrepare] =
      (uint32_t)((g.G[1] + rpb - 1) / rpb) * g.G[2] * (uint32_t)b.C;
  const uint32_t interp =
      (uint32_t)b.n_items * (uint32_t)((b.C + b.fwd_cg - 1) / b.fwd_cg);
  units[kBatchInterp] = g.dim == 2 ? interp : 0;
  units[kBatchInterp3] = g.dim == 3 ? interp : 0;
  units[kBatchGather] = (uint32_t)((b.M + kGatherSamples - 1) / kGatherSamples) *
                        (uint32_t)((b.CP + kGatherCoils - 1) / kGatherCoils);
  units[kBatchSpread] =
      (uint32_t)g.G[1] * g.G[2] *
      (uint32_t)((g.G[0] + kSpmmCells - 1) / kSpmmCells) *
      (uint32_t)((b.C + b.spmm_cg - 1) / b.spmm_cg);
  units[kBatchFinish] = (uint32_t)((g.img_count + kThreads - 1) / kThreads);
}

size_t batch_interp_smem(const BatchInst &b)
{
  const Geo &g = b.g;
  const size_t cells =
      g.dim == 3 ? (size_t)g.pad * g.pad * g.pad : (size_t)g.pad * g.pad;
  return cells * (b.fwd_cg + 1) * sizeof(float2) +
         (size_t)kThreads * (g.dim + g.dim * kBatchSlots) * 4 + 8 +
         (size_t)g.pad * 16;
}

namespace
{
// persistent blocks: as many as are resident on the device at once
template <typename K>
unsigned resident_blocks(K kernel, size_t smem)
{
  int dev = 0, sms = 0, per_sm = 0;
  GN_CUDA(cudaGetDevice(&dev));
  GN_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  GN_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel,
                                                        kThreads, smem));
  return (unsigned)std::max(1, sms * std::max(1, per_sm));
}
}  // namespace

unsigned launch_batch_stage(int stage, const BatchInst *inst, int n,
                            uint32_t total, const BatchIo *io,
                            unsigned *counter, size_t interp_smem,
                            cudaStream_t s)
{
  if (total == 0 || n <= 0)
    return 0;
  if (n > kBatchMax)
    throw Error(kInvalidArgument, "too many instances in a batch");
  unsigned nb = 0;
  switch (stage)
  {
  case kBatchPrepare:
    nb = std::min<unsigned>(total, resident_blocks(k_batch_prepare, 0));
    k_batch_prepare<<<nb, kThreads, 0, s>>>(inst, n, total, counter, *io);
    break;
  case kBatchInterp:
    set_smem(k_batch_interp<2>, interp_smem);
    nb = std::min<unsigned>(total,
                            resident_blocks(k_batch_interp<2>, interp_smem));
    k_batch_interp<2><<<nb, kThreads, interp_smem, s>>>(inst, n, total,
                                                        counter, *io);
    break;
  case kBatchInterp3:
    set_smem(k_batch_interp<3>, interp_smem);
    nb = std::min<unsigned>(total,
                            resident_blocks(k_batch_interp<3>, interp_smem));
    k_batch_interp<3><<<nb, kThreads, interp_smem, s>>>(inst, n, total,
                                                        counter, *io);
    break;
  case kBatchGather:
    nb = std::min<unsigned>(total, resident_blocks(k_batch_gather, 0));
    k_batch_gather<<<nb, kThreads, 0, s>>>(inst, n, total, counter, *io);
    break;
  case kBatchSpread:
    nb = std::min<unsigned>(total, resident_blocks(k_batch_spread, 0));
    k_batch_spread<<<nb, kThreads, 0, s>>>(inst, n, total, counter);
    break;
  default:
    nb = std::min<unsigned>(total, resident_blocks(k_batch_finish, 0));
    k_batch_finish<<<nb, kThreads, 0, s>>>(inst, n, total, counter, *io);
    break;
  }
  GN_LAUNCH_CHECK("batch stage");
  return nb;
}

}  // namespace gnufft
