// Separable, pruned Cartesian transforms fused with the image-space stages
// (see fftpass.cuh).  Index maps per axis (G grid, N image, crop c = the
// upstream crop offset, s = floor(G/2) the INVERSE fftshift):
//   forward  FFT input n holds image pixel (n + s - c) mod G when < N
//   adjoint  FFT output k holds image pixel (k - c - s) mod G when < N
// (the upstream pad -> fftshift and fftshift -> crop,
// gpuNUFFT_operator.cpp:1178-1215 and 775-806).
#include "fftpass.cuh"

#include <algorithm>
#include <cmath>
#include <type_traits>

#include "devutil.hpp"
#include "fftcore.cuh"
#include "tma.cuh"

namespace gnufft
{
namespace
{
using namespace fftcore;

// --------------------------------------------------------------------------
// column passes: lines along a strided axis, columns contiguous
// --------------------------------------------------------------------------
// src: planes of src_rows x ncols, dst: planes of dst_rows x ncols.  FFT
// input n reads source row (n + in_add) mod L when < in_count (else zero);
// FFT output k goes to row (k + out_add) mod L when < out_count.
template <int L, bool INV>
__global__ void __launch_bounds__(Shape<L>::CT)
    k_fft_cols(const float2 *__restrict__ src, float2 *__restrict__ dst,
               long long ncols, int src_rows, int dst_rows, int in_add,
               int in_count, int out_add, int out_count,
               const float2 *__restrict__ roots,
               const uint2 *__restrict__ colrange)
{
  using S = Shape<L>;
  extern __shared__ float2 sm[];
  float2 *tw = sm;
  float2 *Ybase = sm + L;
  load_roots(tw, roots, L);
  const int cl = threadIdx.x % S::TC, lt = threadIdx.x / S::TC;
  const long long col = (long long)blockIdx.x * S::TC + cl;
  const long long plane = blockIdx.y;
  // optional output row range of the column (rows outside are not needed)
  uint2 cr = make_uint2(0u, 0xFFFFFFFFu);
  if (colrange && col < ncols)
    cr = __ldg(colrange + col);
  const bool on = col < ncols && cr.x <= cr.y;
  // exchange slots of the block's columns interleaved: slot * TC + column
  float2 *Y = Ybase + cl;
  const float2 *sp = src + plane * src_rows * ncols + col;
  float2 *dp = dst + plane * dst_rows * ncols + col;
  __syncthreads();
  float2 w[Rm<L>::V / 2];
  load_reg_roots<L>(w, tw);
  if (lt < S::R2)
  {
    float2 a[S::R1];
#pragma unroll
    for (int j = 0; j < S::R1; ++j)
    {
      const int r = (lt + S::R2 * j + in_add) & (L - 1);
      a[j] = (on && r < in_count) ? __ldg(sp + (long long)r * ncols)
                                  : make_float2(0.f, 0.f);
    }
    stage1<L, INV, S::TC>(a, lt, w, tw, Y);
  }
  __syncthreads();
  if (lt < S::R1)
  {
    float2 b[S::R2];
    stage2<L, INV, S::TC>(b, lt, w, Y);
    if (on)
    {
#pragma unroll
      for (int k2 = 0; k2 < S::R2; ++k2)
      {
        const int r = (lt + S::R1 * k2 + out_add) & (L - 1);
        if (r < out_count && (unsigned)r >= cr.x && (unsigned)r <= cr.y)
          dp[(long long)r * ncols] = b[k2];
      }
    }
  }
}

// --------------------------------------------------------------------------
// column passes with tensor-copy (TMA) tiles
// --------------------------------------------------------------------------
// A persistent block walks its tiles of TC adjacent columns (tile t: plane
// t / n_ct, columns (t % n_ct) * TC ...) through two shared-memory buffers:
// the copy of its next tile is in flight while the current one is
// transformed.  The transform runs in place in the tile: a stage-1 thread
// reads the rows of its residue class mod R2 and writes its twiddled
// outputs back into rows of the same class (row k1 * R2 + residue), so no
// thread overwrites a row another thread still has to read; after a
// barrier, stage-2 thread k1 reads row k1 * R2 + ((u + in_add) mod R2) for
// every stage-1 index u.  A tile row is TC * 8 = 128 bytes, so each warp
// access covers whole rows (no bank conflicts, no padding).  The arithmetic
// is that of k_fft_cols.
template <int L> struct ColTma
{
  using S = Shape<L>;
  static_assert(S::TC * 8 == 128, "tile rows of 128 bytes");
  static constexpr size_t tile_bytes = (size_t)L * S::TC * sizeof(float2);
  static size_t smem()
  {
    return 2 * tile_bytes + (size_t)L * sizeof(float2) + 2 * 8 + 16;
  }
};

// One thread: expect the tile's bytes on `bar` and issue its copies (boxes
// of box_rows rows starting at rows 0, box_rows, ...).
__device__ __forceinline__ void col_tile_issue(const CUtensorMap *tmap,
                                               uint32_t dst, uint32_t bar,
                                               int col0, int plane,
                                               int box_rows, int ncopy,
                                               uint32_t bytes)
{
  tma::mbar_expect_tx(bar, bytes);
  for (int q = 0; q < ncopy; ++q)
    tma::copy_3d(dst + (uint32_t)(q * box_rows) * 128u, tmap, col0,
                 q * box_rows, plane, bar);
}

// The in-place transform of column cl of tile B; returns the stage-2
// outputs of thread lt (< R1) in b (outputs k = lt + R1 * k2).
// Tile position of (row r, column lane cl): rows of TC columns, or (PAIRS)
// two planes of L rows x TC / 2 columns (lanes cl < TC / 2 in the first).
template <int L, bool PAIRS>
__device__ __forceinline__ int col_pos(int r, int cl)
{
  constexpr int TC = Shape<L>::TC;
  if constexpr (PAIRS)
    return ((cl / (TC / 2)) * L + r) * (TC / 2) + cl % (TC / 2);
  else
    return r * TC + cl;
}

template <int L, bool INV, bool PAIRS = false>
__device__ __forceinline__ void col_tile_fft(float2 *B, int cl, int lt,
                                             int in_add, int in_count,
                                             const float2 (&w)[Rm<L>::V / 2],
                                             const float2 *tw,
                                             float2 (&b)[Shape<L>::R2])
{
  using S = Shape<L>;
  if (lt < S::R2)
  {
    float2 a[S::R1];
#pragma unroll
    for (int j = 0; j < S::R1; ++j)
    {
      const int r = (lt + S::R2 * j + in_add) & (L - 1);
      a[j] = r < in_count ? B[col_pos<L, PAIRS>(r, cl)] : make_float2(0.f, 0.f);
    }
    reg_fft<S::R1, Rm<L>::V, INV>(a, w);
    const int rho = (lt + in_add) & (S::R2 - 1);
#pragma unroll
    for (int k1 = 0; k1 < S::R1; ++k1)
    {
      float2 v = a[k1];
      if (k1 != 0)
      {
        float2 r = tw[(lt * k1) & (L - 1)];
        if (INV)
          r.y = -r.y;
        v = cmul(v, r);
      }
      B[col_pos<L, PAIRS>(k1 * S::R2 + rho, cl)] = v;
    }
  }
  __syncthreads();
  if (lt < S::R1)
  {
#pragma unroll
    for (int u = 0; u < S::R2; ++u)
      b[u] = B[col_pos<L, PAIRS>(lt * S::R2 + ((u + in_add) & (S::R2 - 1)),
                                  cl)];
    reg_fft<S::R2, Rm<L>::V, INV>(b, w);
  }
}

// The same transform for two adjacent columns 2 cp, 2 cp + 1 of a tile of
// TC-column rows (one 16-byte shared access per row and stage for both,
// one twiddle load for both).  Outputs k = lt + R1 * k2 in b0 / b1.
template <int L, bool INV>
__device__ __forceinline__ void col_tile_fft2(float2 *B, int cp, int lt,
                                              int in_add, int in_count,
                                              const float2 (&w)[Rm<L>::V / 2],
                                              const float2 *tw,
                                              float2 (&b0)[Shape<L>::R2],
                                              float2 (&b1)[Shape<L>::R2])
{
  using S = Shape<L>;
  constexpr int TP = S::TC / 2;  // column pairs per tile row
  float4 *B4 = reinterpret_cast<float4 *>(B);
  if (lt < S::R2)
  {
    float2 a0[S::R1], a1[S::R1];
#pragma unroll
    for (int j = 0; j < S::R1; ++j)
    {
      const int r = (lt + S::R2 * j + in_add) & (L - 1);
      const float4 v =
          r < in_count ? B4[r * TP + cp] : make_float4(0.f, 0.f, 0.f, 0.f);
      a0[j] = make_float2(v.x, v.y);
      a1[j] = make_float2(v.z, v.w);
    }
    reg_fft<S::R1, Rm<L>::V, INV>(a0, w);
    reg_fft<S::R1, Rm<L>::V, INV>(a1, w);
    const int rho = (lt + in_add) & (S::R2 - 1);
#pragma unroll
    for (int k1 = 0; k1 < S::R1; ++k1)
    {
      float2 v0 = a0[k1], v1 = a1[k1];
      if (k1 != 0)
      {
        float2 r = tw[(lt * k1) & (L - 1)];
        if (INV)
          r.y = -r.y;
        v0 = cmul(v0, r);
        v1 = cmul(v1, r);
      }
      B4[(k1 * S::R2 + rho) * TP + cp] = make_float4(v0.x, v0.y, v1.x, v1.y);
    }
  }
  __syncthreads();
  if (lt < S::R1)
  {
#pragma unroll
    for (int u = 0; u < S::R2; ++u)
    {
      const float4 v =
          B4[(lt * S::R2 + ((u + in_add) & (S::R2 - 1))) * TP + cp];
      b0[u] = make_float2(v.x, v.y);
      b1[u] = make_float2(v.z, v.w);
    }
    reg_fft<S::R2, Rm<L>::V, INV>(b0, w);
    reg_fft<S::R2, Rm<L>::V, INV>(b1, w);
  }
}

// Tile t of a pass over `planes` planes of n_ct column tiles (PAIRED 0:
// plane t / n_ct, columns (t % n_ct) * TC ...).  PAIRED > 0: a tile holds
// TC / 2 columns of both planes (coils) of a pair; output element (plane c,
// row r, column col) goes to ((c / 2) * dst_rows * ncols + r * ncols + col)
// * 2 + c % 2, i.e. coil pairs interleaved (the layout the 3-D forward
// interpolation reads two coils of a cell from with one 16-byte load), and
// every warp store covers TC / 2 whole pairs.  Tile t: pair t / n_ct,
// column tile t % n_ct (n_ct counted in TC / 2 columns).  Tile layouts in
// shared memory: PAIRED 0, rows of TC columns of one plane; PAIRED 1, the
// two coils as two planes of L rows x TC / 2 columns (two 3-D boxes; the
// second plane of an odd last pair is an out-of-range box, zero fill; the
// two planes' rows share banks); PAIRED 2, one 4-D box (columns, coil in
// pair, rows, pair) that interleaves the coils' half rows, so that tile row
// r holds TC / 2 columns of the first coil, then of the second -- the
// layout of PAIRED 0, read without bank conflicts.  `tail` (PAIRED 2)
// covers an odd last coil (pair tail_pl) with a one-coil map whose second
// coil is out of range (zero fill).  CPT 2 (PAIRED 2 only): each thread
// runs two adjacent columns of one coil (col_tile_fft2), half the threads.
template <int L, bool INV, int PAIRED, int CPT = 1>
__global__ void __launch_bounds__(Shape<L>::CT / CPT, 3)
    k_fft_cols_tma(const __grid_constant__ CUtensorMap tmap,
                   const __grid_constant__ CUtensorMap tail, long long tail_pl,
                   float2 *__restrict__ dst, long long ncols, FastDiv n_ct,
                   int n_tiles, int box_rows, int ncopy, int dst_rows,
                   int in_add, int in_count, int out_add, int out_count,
                   const float2 *__restrict__ roots,
                   const uint2 *__restrict__ colrange,
                   const uint32_t *__restrict__ tiles, tma::CopyWait cw)
{
  using S = Shape<L>;
  using T = ColTma<L>;
  constexpr int TC = S::TC;
  extern __shared__ __align__(128) unsigned char smraw[];
  float2 *buf = reinterpret_cast<float2 *>(smraw);
  float2 *tw = buf + 2 * L * TC;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(tw + L);
  int &s_fail = *reinterpret_cast<int *>(mbar + 2);
  const uint32_t bar0 = tma::smem_addr(mbar);
  const uint32_t buf0 = tma::smem_addr(buf);
  const uint32_t bytes = (uint32_t)(ncopy * box_rows) * 128u;
  const int stride = gridDim.x;
  constexpr int CW = PAIRED ? TC / 2 : TC;  // columns per tile
  auto tile = [&](int t, int &pl, int &ct) {
    pl = (int)n_ct.div((uint32_t)t);
    ct = t - pl * (int)n_ct.d;
    if (tiles)
      ct = (int)__ldg(tiles + ct);
  };
  auto issue = [&](int t, int b) {
    int pl, ct;
    tile(t, pl, ct);
    const uint32_t dst = buf0 + (uint32_t)b * (uint32_t)T::tile_bytes;
    const uint32_t bar = bar0 + 8u * (uint32_t)b;
    if (PAIRED == 2)
    {  // both coils of pair pl, half rows interleaved
      tma::mbar_expect_tx(bar, bytes);
      if (pl == tail_pl)
        tma::copy_4d(dst, &tail, (int)ct * CW, 0, 0, 0, bar);
      else
        tma::copy_4d(dst, &tmap, (int)ct * CW, 0, 0, (int)pl, bar);
    }
    else if (PAIRED == 1)
    {  // both planes of pair pl, each into its own L rows
      tma::mbar_expect_tx(bar, bytes);  // two boxes of half the columns
      tma::copy_3d(dst, &tmap, (int)ct * CW, 0, (int)(2 * pl), bar);
      tma::copy_3d(dst + (uint32_t)(L * CW * sizeof(float2)), &tmap,
                   (int)ct * CW, 0, (int)(2 * pl + 1), bar);
    }
    else
      col_tile_issue(&tmap, dst, bar, (int)ct * TC, (int)pl, box_rows, ncopy,
                     bytes);
  };
  if (threadIdx.x == 0)
  {
    s_fail = 0;
    tma::mbar_init(bar0);
    tma::mbar_init(bar0 + 8u);
    tma::mbar_init_fence();
    if (blockIdx.x < n_tiles)
      issue(blockIdx.x, 0);
    if (blockIdx.x + stride < n_tiles)
      issue(blockIdx.x + stride, 1);
  }
  load_roots(tw, roots, L);
  __syncthreads();
  float2 w[Rm<L>::V / 2];
  load_reg_roots<L>(w, tw);
  static_assert(CPT == 1 || (CPT == 2 && PAIRED == 2), "column pairs");
  // CPT 2 (interleaved coil pairs): thread (cl = column pair, lt) runs tile
  // columns 2 cl, 2 cl + 1, two adjacent grid columns of one coil
  const int cl = threadIdx.x % (TC / CPT), lt = threadIdx.x / (TC / CPT);
  int i = 0;
  for (int t = blockIdx.x; t < n_tiles; t += stride, ++i)
  {
    const int b = i & 1;
    if (threadIdx.x == 0 &&
        !tma::mbar_wait_bounded(bar0 + 8u * (uint32_t)b,
                                (uint32_t)(i >> 1) & 1u, cw.polls))
      s_fail = 1;
    __syncthreads();
    if (s_fail)
    {  // a copy did not complete: report it and give the copies in flight
       // (this tile's, the next one's) a bounded wait before returning
      if (threadIdx.x == 0)
      {
        atomicExch(cw.err, 1);
        tma::mbar_wait_bounded(bar0 + 8u * (uint32_t)b, (uint32_t)(i >> 1) & 1u);
        if (t + stride < n_tiles)
          tma::mbar_wait_bounded(bar0 + 8u * (uint32_t)(b ^ 1),
                                 (uint32_t)((i + 1) >> 1) & 1u);
      }
      return;
    }
    int pl, ct;
    tile(t, pl, ct);
    const int q = cl * CPT;  // first tile column of the thread
    const long long plane = PAIRED ? 2LL * pl + q / CW : pl;
    const long long col = (long long)ct * CW + q % CW;
    const long long psz = (long long)dst_rows * ncols;
    float2 *dp = PAIRED ? dst + ((plane >> 1) * psz + col) * 2 + (plane & 1)
                        : dst + plane * psz + col;
    const long long rs = PAIRED ? 2 * ncols : ncols;
    if constexpr (CPT == 1)
    {
      uint2 cr = make_uint2(0u, 0xFFFFFFFFu);
      if (colrange && col < ncols)
        cr = __ldg(colrange + col);
      const bool on = col < ncols && cr.x <= cr.y;
      float2 bv[S::R2];
      col_tile_fft<L, INV, PAIRED == 1>(buf + (size_t)b * L * TC, cl, lt,
                                        in_add, in_count, w, tw, bv);
      if (lt < S::R1 && on)
      {
#pragma unroll
        for (int k2 = 0; k2 < S::R2; ++k2)
        {
          const int r = (lt + S::R1 * k2 + out_add) & (L - 1);
          if (r < out_count && (unsigned)r >= cr.x && (unsigned)r <= cr.y)
            dp[(long long)r * rs] = bv[k2];
        }
      }
    }
    else
    {  // columns col, col + 1 (ncols is even, so both or neither exist)
      uint2 cr0 = make_uint2(0u, 0xFFFFFFFFu), cr1 = cr0;
      if (colrange && col < ncols)
      {
        cr0 = __ldg(colrange + col);
        cr1 = __ldg(colrange + col + 1);
      }
      float2 b0[S::R2], b1[S::R2];
      col_tile_fft2<L, INV>(buf + (size_t)b * L * TC, cl, lt, in_add,
                            in_count, w, tw, b0, b1);
      if (lt < S::R1 && col < ncols)
      {
#pragma unroll
        for (int k2 = 0; k2 < S::R2; ++k2)
        {
          const int r = (lt + S::R1 * k2 + out_add) & (L - 1);
          if (r < out_count && (unsigned)r >= cr0.x && (unsigned)r <= cr0.y)
            dp[(long long)r * rs] = b0[k2];
          if (r < out_count && (unsigned)r >= cr1.x && (unsigned)r <= cr1.y)
            dp[(long long)r * rs + 2] = b1[k2];  // next column, same coil
        }
      }
    }
    tma::fence_proxy_async();  // the in-place writes before the refill
    __syncthreads();           // buffer b is free
    if (threadIdx.x == 0 && t + 2 * stride < n_tiles)
      issue(t + 2 * stride, b);
  }
}

// --------------------------------------------------------------------------
// last adjoint pass along a strided axis, fused with the image stages
// --------------------------------------------------------------------------
// Columns contiguous (TC per block); each block runs every coil of its
// columns in turn: inverse DFT, crop + shift (output k holds image index
// (k + out_add) mod L when < n_out), 1/sqrt(Ng), deapodization and the
// conj(S) coil sum in coil order (or per-coil outputs).  src: coil c,
// row r, column col at c * coil_stride + r * ncols + col; image pixel of
// output row n and column col: n * ncols + col.
template <int L, bool SENS>
__global__ void __launch_bounds__(Shape<L>::CT, L <= 256 ? 3 : 1)
    k_fft_cols_sum(const float2 *__restrict__ src, long long ncols,
                   long long coil_stride, const float *__restrict__ deapo,
                   const float2 *__restrict__ sens, int n_out, long long N,
                   int C, int coils_per_block, int out_add, float scale,
                   int stage, int accumulate,
                   const float2 *__restrict__ roots, float2 *__restrict__ out,
                   float2 *__restrict__ partial)
{
  using S = Shape<L>;
  extern __shared__ float2 sm[];
  float2 *tw = sm;
  float2 *Ybase = sm + L;
  load_roots(tw, roots, L);
  const int cl = threadIdx.x % S::TC, lt = threadIdx.x / S::TC;
  const long long col = (long long)blockIdx.x * S::TC + cl;
  const bool on = col < ncols;
  float2 *Y = Ybase + cl;
  __syncthreads();
  float2 w[Rm<L>::V / 2];
  load_reg_roots<L>(w, tw);
  float2 acc[S::R2];
#pragma unroll
  for (int k2 = 0; k2 < S::R2; ++k2)
    acc[k2] = make_float2(0.f, 0.f);
  const int c0 = blockIdx.y * coils_per_block;
  const int c1 = min(C, c0 + coils_per_block);
  for (int c = c0; c < c1; ++c)
  {
    if (lt < S::R2)
    {
      const float2 *sp = src + (long long)c * coil_stride + col;
      float2 a[S::R1];
#pragma unroll
      for (int j = 0; j < S::R1; ++j)
        a[j] = on ? __ldg(sp + (long long)(lt + S::R2 * j) * ncols)
                  : make_float2(0.f, 0.f);
      stage1<L, true, S::TC>(a, lt, w, tw, Y);
    }
    __syncthreads();
    if (lt < S::R1 && on)
    {
      float2 b[S::R2];
      stage2<L, true, S::TC>(b, lt, w, Y);
#pragma unroll
      for (int k2 = 0; k2 < S::R2; ++k2)
      {
        const int n = (lt + S::R1 * k2 + out_add) & (L - 1);
        if (n >= n_out)
          continue;
        const long long px = (long long)n * ncols + col;
        // crop -> FFT scaling -> deapodization (gpuNUFFT_operator.cpp:
        // 800-819)
        float2 v = make_float2(__fmul_rn(b[k2].x, scale),
                               __fmul_rn(b[k2].y, scale));
        if (stage == 2)
        {
          const float d = __ldg(deapo + px);
          v.x = __fmul_rn(v.x, d);
          v.y = __fmul_rn(v.y, d);
        }
        if (SENS && stage == 2)
        {  // conj(S) * v, running coil sum (std_gpuNUFFT_kernels.cu:158-218)
          const float2 sv = __ldg(sens + c * N + px);
          const float2 t = cmul_conj(v, sv);
          acc[k2].x = __fadd_rn(acc[k2].x, t.x);
          acc[k2].y = __fadd_rn(acc[k2].y, t.y);
        }
        else
          out[c * N + px] = v;
      }
    }
    __syncthreads();
  }
  if (SENS && stage == 2 && lt < S::R1 && on)
  {
#pragma unroll
    for (int k2 = 0; k2 < S::R2; ++k2)
    {
      const int n = (lt + S::R1 * k2 + out_add) & (L - 1);
      if (n >= n_out)
        continue;
      const long long px = (long long)n * ncols + col;
      if (partial)
      {  // one coil group of several: summed in group order afterwards
        partial[blockIdx.y * N + px] = acc[k2];
        continue;
      }
      float2 r = acc[k2];
      if (accumulate)
      {
        const float2 o = out[px];
        r = make_float2(o.x + r.x, o.y + r.y);
      }
      out[px] = r;
    }
  }
}

// The same pass with the coil combine (stage 2, maps) on tensor-copy
// tiles.  A persistent block walks its units (unit u: TC adjacent columns
// (u / groups) * TC ..., coil group u % groups) and in each unit its coils
// in order.  Per coil, two copies bring the column tile (L rows x TC
// columns) and the coil-map tile (n_out rows x TC columns) into one of two
// stages, so that the copies of the next coil (or of the next unit's first
// coil) are in flight while the current one is transformed in place (as in
// k_fft_cols_tma).  Deapodization is read once per unit.  Arithmetic and
// coil order are those of k_fft_cols_sum, so both give the same results.
template <int L> struct SumTma
{
  using S = Shape<L>;
  static constexpr uint32_t src_bytes = (uint32_t)(L * S::TC * sizeof(float2));
  __host__ __device__ static uint32_t sens_bytes(int n_out)
  {
    return (uint32_t)(n_out * S::TC * sizeof(float2));
  }
  static size_t smem(int n_out)
  {
    return 2 * ((size_t)src_bytes + sens_bytes(n_out)) +
           (size_t)L * sizeof(float2) + 2 * 8 + 16;
  }
};

template <int L>
__global__ void __launch_bounds__(Shape<L>::CT, 2)
    k_fft_cols_sum_tma(const __grid_constant__ CUtensorMap src_map,
                       const __grid_constant__ CUtensorMap sens_map,
                       long long ncols, int n_units, FastDiv groups,
                       int cpb, int C, const float *__restrict__ deapo,
                       int n_out, long long N, int out_add, float scale,
                       int accumulate, const float2 *__restrict__ roots,
                       float2 *__restrict__ out, float2 *__restrict__ partial,
                       tma::CopyWait cw)
{
  using S = Shape<L>;
  using T = SumTma<L>;
  constexpr int TC = S::TC;
  extern __shared__ __align__(128) unsigned char smraw[];
  float2 *src_t = reinterpret_cast<float2 *>(smraw);  // 2 x L x TC
  float2 *sens_t = src_t + 2 * L * TC;                 // 2 x n_out x TC
  float2 *tw = sens_t + 2 * (size_t)n_out * TC;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(tw + L);
  int &s_fail = *reinterpret_cast<int *>(mbar + 2);
  const uint32_t bar0 = tma::smem_addr(mbar);
  const uint32_t src0 = tma::smem_addr(src_t);
  const uint32_t sens0 = tma::smem_addr(sens_t);
  const uint32_t sens_bytes = T::sens_bytes(n_out);
  // job cursor: unit u, coil c of the unit's coils [c0, c1)
  struct Cur
  {
    int u, ct, g;  // unit, its column tile and coil group
    int c, c1;     // coil, end of the group's coils
  };
  auto start = [&](int u) {
    Cur k;
    k.u = u;
    k.ct = (int)groups.div((uint32_t)u);
    k.g = u - k.ct * (int)groups.d;
    k.c = k.g * cpb;
    k.c1 = min(C, k.c + cpb);
    return k;
  };
  auto next = [&](Cur k) {
    if (++k.c >= k.c1)
      k = start(k.u + gridDim.x);
    return k;
  };
  auto issue = [&](const Cur &k, int b) {
    const uint32_t bar = bar0 + 8u * (uint32_t)b;
    const int col0 = k.ct * TC;
    tma::mbar_expect_tx(bar, T::src_bytes + sens_bytes);
    tma::copy_3d(src0 + (uint32_t)b * T::src_bytes, &src_map, col0, 0, k.c,
                 bar);
    tma::copy_3d(sens0 + (uint32_t)b * sens_bytes, &sens_map, col0, 0, k.c,
                 bar);
  };
  Cur ic = start(blockIdx.x);  // the next job to copy (uniform)
  if (threadIdx.x == 0)
  {
    s_fail = 0;
    tma::mbar_init(bar0);
    tma::mbar_init(bar0 + 8u);
    tma::mbar_init_fence();
    if (ic.u < n_units)
      issue(ic, 0);
  }
  ic = next(ic);
  if (threadIdx.x == 0 && ic.u < n_units)
    issue(ic, 1);
  ic = next(ic);
  load_roots(tw, roots, L);
  __syncthreads();
  float2 w[Rm<L>::V / 2];
  load_reg_roots<L>(w, tw);
  const int cl = threadIdx.x % TC, lt = threadIdx.x / TC;
  float2 acc[S::R2];
  float d[S::R2];
  long long i = 0;
  for (Cur cc = start(blockIdx.x); cc.u < n_units; ++i)
  {
    const int b = (int)(i & 1);
    if (threadIdx.x == 0 &&
        !tma::mbar_wait_bounded(bar0 + 8u * (uint32_t)b,
                                (uint32_t)(i >> 1) & 1u, cw.polls))
      s_fail = 1;
    __syncthreads();
    const Cur nx = next(cc);
    if (s_fail)
    {  // a copy did not complete: report it and give the copies in flight
       // (this job's, the next one's) a bounded wait before returning
      if (threadIdx.x == 0)
      {
        atomicExch(cw.err, 1);
        tma::mbar_wait_bounded(bar0 + 8u * (uint32_t)b,
                               (uint32_t)(i >> 1) & 1u);
        if (nx.u < n_units)
          tma::mbar_wait_bounded(bar0 + 8u * (uint32_t)(b ^ 1),
                                 (uint32_t)((i + 1) >> 1) & 1u);
      }
      return;
    }
    const long long col = (long long)cc.ct * TC + cl;
    const bool on = col < ncols && lt < S::R1;
    if (cc.c == cc.g * cpb)
    {  // the unit's first coil: its deapodization, a zero sum
#pragma unroll
      for (int k2 = 0; k2 < S::R2; ++k2)
      {
        const int n = (lt + S::R1 * k2 + out_add) & (L - 1);
        d[k2] = (on && n < n_out) ? __ldg(deapo + (long long)n * ncols + col)
                                  : 0.f;
        acc[k2] = make_float2(0.f, 0.f);
      }
    }
    float2 bv[S::R2];
    col_tile_fft<L, true, false>(src_t + (size_t)b * L * TC, cl, lt, 0, L, w,
                                 tw, bv);
    if (on)
    {
      const float2 *st = sens_t + (size_t)b * n_out * TC;
#pragma unroll
      for (int k2 = 0; k2 < S::R2; ++k2)
      {
        const int n = (lt + S::R1 * k2 + out_add) & (L - 1);
        if (n >= n_out)
          continue;
        // crop -> FFT scaling -> deapodization -> conj(S) * v, running coil
        // sum (gpuNUFFT_operator.cpp:800-819, std_gpuNUFFT_kernels.cu:
        // 158-218)
        float2 v = make_float2(__fmul_rn(bv[k2].x, scale),
                               __fmul_rn(bv[k2].y, scale));
        v.x = __fmul_rn(v.x, d[k2]);
        v.y = __fmul_rn(v.y, d[k2]);
        const float2 sv = st[n * TC + cl];
        const float2 t = cmul_conj(v, sv);
        acc[k2].x = __fadd_rn(acc[k2].x, t.x);
        acc[k2].y = __fadd_rn(acc[k2].y, t.y);
      }
    }
    tma::fence_proxy_async();  // the in-place writes before the refill
    __syncthreads();           // stage b is free
    if (threadIdx.x == 0 && ic.u < n_units)
      issue(ic, b);
    ic = next(ic);
    if (nx.u != cc.u && on)
    {  // the unit's last coil: its sum (or the group's partial sum)
#pragma unroll
      for (int k2 = 0; k2 < S::R2; ++k2)
      {
        const int n = (lt + S::R1 * k2 + out_add) & (L - 1);
        if (n >= n_out)
          continue;
        const long long px = (long long)n * ncols + col;
        if (partial)
        {
          partial[cc.g * N + px] = acc[k2];
          continue;
        }
        float2 r = acc[k2];
        if (accumulate)
        {
          const float2 o = out[px];
          r = make_float2(o.x + r.x, o.y + r.y);
        }
        out[px] = r;
      }
    }
    cc = nx;
  }
}

__global__ void k_sum_coil_groups(const float2 *__restrict__ partial,
                                  int groups, long long N, int accumulate,
                                  float2 *__restrict__ out)
{
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < N;
       p += (long long)gridDim.x * blockDim.x)
  {
    float2 r = make_float2(0.f, 0.f);
    for (int k = 0; k < groups; ++k)
    {
      const float2 v = partial[k * N + p];
      r.x += v.x;
      r.y += v.y;
    }
    if (accumulate)
    {
      const float2 o = out[p];
      r = make_float2(o.x + r.x, o.y + r.y);
    }
    out[p] = r;
  }
}

// --------------------------------------------------------------------------
// forward rows: sens multiply, deapodization, pad + shift, DFT along x
// --------------------------------------------------------------------------
// One line per (image row, coil), coil fastest: a block's lines share image
// rows, so the image is read once per block.  Output A[c][row][k],
// rows = N_y * N_z.
template <int L, bool SENS>
__global__ void __launch_bounds__(kFftThreads, L <= 256 ? 4 : 1)
    k_fft_rows_fwd(const float2 *__restrict__ image,
                   const float2 *__restrict__ sens,
                   const float *__restrict__ deapo, int Nx, long long rows,
                   long long N, int C, int in_add, int out_add,
                   const float2 *__restrict__ roots, float2 *__restrict__ A)
{
  using S = Shape<L>;
  extern __shared__ float2 sm[];
  float2 *tw = sm;
  load_roots(tw, roots, L);
  const int line = threadIdx.x / S::T, lt = threadIdx.x % S::T;
  const long long ln = (long long)blockIdx.x * S::NL + line;
  const bool on = ln < rows * C;
  const long long row = on ? ln / C : 0;
  const int c = on ? (int)(ln - row * C) : 0;
  float2 *Y = sm + L + line * S::R1 * S::YP;
  const long long rbase = row * Nx;
  __syncthreads();
  float2 w[Rm<L>::V / 2];
  load_reg_roots<L>(w, tw);
  if (lt < S::R2)
  {
    // FFT input n = lt + R2 j holds image x (n + in_add) mod L when < Nx
    float2 a[S::R1];
#pragma unroll
    for (int j = 0; j < S::R1; ++j)
    {
      const int xp = (lt + S::R2 * j + in_add) & (L - 1);
      float2 v = make_float2(0.f, 0.f);
      if (on && xp < Nx)
      {
        const long long px = rbase + xp;
        if (SENS)
        {  // sensMulKernel, then deapodization (std_gpuNUFFT_kernels.cu)
          const float2 x = __ldg(image + px);
          const float2 s = __ldg(sens + c * N + px);
          v = cmul(x, s);
        }
        else
          v = __ldg(image + c * N + px);
        const float d = __ldg(deapo + px);
        v.x = __fmul_rn(v.x, d);
        v.y = __fmul_rn(v.y, d);
      }
      a[j] = v;
    }
    stage1<L, false, 1>(a, lt, w, tw, Y);
  }
  __syncthreads();
  if (lt < S::R1 && on)
  {
    float2 b[S::R2];
    stage2<L, false, 1>(b, lt, w, Y);
    float2 *out = A + ((long long)c * rows + row) * L;
#pragma unroll
    for (int k2 = 0; k2 < S::R2; ++k2)
      out[(lt + S::R1 * k2 + out_add) & (L - 1)] = b[k2];
  }
}

// The same pass on tensor-copy tiles (at least NL coils, N_x <= 256, N_x a
// multiple of 4): a persistent block walks its jobs (job j: image row
// j / n_cc, coils (j % n_cc) * NL ..., one line per coil) through two
// stages.  Per job one tensor copy brings the NL coil rows (the maps with
// SENS, else the per-coil images; coils past C are out of range, zero
// fill) and untiled copies bring the image row (SENS) and the
// deapodization row, so that the copies of the job after next are in
// flight while the current one is transformed: a stage is refilled as soon
// as the first DFT stage, its only reader, is done.  Arithmetic is that of
// k_fft_rows_fwd, so both give the same results.
struct RowsTma
{
  static __host__ __device__ uint32_t up128(uint32_t v)
  {
    return (v + 127u) & ~127u;
  }
  // per stage: coil rows, image row, deapodization row
  static __host__ __device__ uint32_t coil_bytes(int NL, int Nx)
  {
    return up128((uint32_t)(NL * Nx * 8));
  }
  static __host__ __device__ uint32_t img_bytes(int Nx)
  {
    return up128((uint32_t)(Nx * 8));
  }
  static __host__ __device__ uint32_t stage_bytes(int NL, int Nx)
  {
    return coil_bytes(NL, Nx) + img_bytes(Nx) + up128((uint32_t)(Nx * 4));
  }
};

template <int L, bool SENS>
__global__ void __launch_bounds__(kFftThreads, 3)
    k_fft_rows_fwd_tma(const __grid_constant__ CUtensorMap coil_map,
                       const float2 *__restrict__ image,
                       const float *__restrict__ deapo, int Nx,
                       long long rows, int C, int n_jobs, FastDiv n_cc,
                       int in_add, int out_add,
                       const float2 *__restrict__ roots,
                       float2 *__restrict__ A, tma::CopyWait cw)
{
  using S = Shape<L>;
  constexpr int NL = S::NL;
  extern __shared__ __align__(128) unsigned char smraw[];
  const uint32_t cb = RowsTma::coil_bytes(NL, Nx);
  const uint32_t ib = RowsTma::img_bytes(Nx);
  const uint32_t sb = RowsTma::stage_bytes(NL, Nx);
  float2 *tw = reinterpret_cast<float2 *>(smraw + 2 * sb);
  float2 *Ybase = tw + L;
  uint64_t *mbar = reinterpret_cast<uint64_t *>(Ybase + NL * S::R1 * S::YP);
  int &s_fail = *reinterpret_cast<int *>(mbar + 2);
  const uint32_t bar0 = tma::smem_addr(mbar);
  const uint32_t st0 = tma::smem_addr(smraw);
  const uint32_t tx = (uint32_t)(NL * Nx * 8) + (SENS ? (uint32_t)(Nx * 8) : 0u) +
                      (uint32_t)(Nx * 4);
  const int stride = gridDim.x;
  auto issue = [&](int j, int b) {
    const long long r = n_cc.div((uint32_t)j);
    const int c0 = (j - (int)r * (int)n_cc.d) * NL;
    const uint32_t dst = st0 + (uint32_t)b * sb;
    const uint32_t bar = bar0 + 8u * (uint32_t)b;
    tma::mbar_expect_tx(bar, tx);
    tma::copy_2d(dst, &coil_map, (int)(r * Nx), c0, bar);
    if (SENS)
      tma::copy_bulk(dst + cb, image + r * Nx, (uint32_t)(Nx * 8), bar);
    tma::copy_bulk(dst + cb + ib, deapo + r * Nx, (uint32_t)(Nx * 4), bar);
  };
  if (threadIdx.x == 0)
  {
    s_fail = 0;
    tma::mbar_init(bar0);
    tma::mbar_init(bar0 + 8u);
    tma::mbar_init_fence();
    if (blockIdx.x < n_jobs)
      issue(blockIdx.x, 0);
    if (blockIdx.x + stride < n_jobs)
      issue(blockIdx.x + stride, 1);
  }
  load_roots(tw, roots, L);
  __syncthreads();
  float2 w[Rm<L>::V / 2];
  load_reg_roots<L>(w, tw);
  const int line = threadIdx.x / S::T, lt = threadIdx.x % S::T;
  float2 *Y = Ybase + line * S::R1 * S::YP;
  int i = 0;
  for (int j = blockIdx.x; j < n_jobs; j += stride, ++i)
  {
    const int b = i & 1;
    if (threadIdx.x == 0 &&
        !tma::mbar_wait_bounded(bar0 + 8u * (uint32_t)b,
                                (uint32_t)(i >> 1) & 1u, cw.polls))
      s_fail = 1;
    __syncthreads();  // also: the previous job's exchange reads are done
    if (s_fail)
    {  // a copy did not complete: report it and give the copies in flight
       // (this job's, the next one's) a bounded wait before returning
      if (threadIdx.x == 0)
      {
        atomicExch(cw.err, 1);
        tma::mbar_wait_bounded(bar0 + 8u * (uint32_t)b,
                               (uint32_t)(i >> 1) & 1u);
        if (j + stride < n_jobs)
          tma::mbar_wait_bounded(bar0 + 8u * (uint32_t)(b ^ 1),
                                 (uint32_t)((i + 1) >> 1) & 1u);
      }
      return;
    }
    const long long row = n_cc.div((uint32_t)j);
    const int c = (j - (int)row * (int)n_cc.d) * NL + line;
    const unsigned char *stg = smraw + (size_t)b * sb;
    const float2 *crow = reinterpret_cast<const float2 *>(stg) + line * Nx;
    const float2 *img = reinterpret_cast<const float2 *>(stg + cb);
    const float *dea = reinterpret_cast<const float *>(stg + cb + ib);
    if (lt < S::R2)
    {
      // FFT input n = lt + R2 j holds image x (n + in_add) mod L when < Nx
      float2 a[S::R1];
#pragma unroll
      for (int q = 0; q < S::R1; ++q)
      {
        const int xp = (lt + S::R2 * q + in_add) & (L - 1);
        float2 v = make_float2(0.f, 0.f);
        if (xp < Nx)
        {
          if (SENS)
          {  // sensMulKernel, then deapodization (std_gpuNUFFT_kernels.cu)
            const float2 x = img[xp];
            const float2 sv = crow[xp];
            v = cmul(x, sv);
          }
          else
            v = crow[xp];
          const float d = dea[xp];
          v.x = __fmul_rn(v.x, d);
          v.y = __fmul_rn(v.y, d);
        }
        a[q] = v;
      }
      stage1<L, false, 1>(a, lt, w, tw, Y);
    }
    __syncthreads();  // stage b read; exchange written
    if (threadIdx.x == 0 && j + 2 * stride < n_jobs)
      issue(j + 2 * stride, b);
    if (lt < S::R1 && c < C)
    {
      float2 bv[S::R2];
      stage2<L, false, 1>(bv, lt, w, Y);
      float2 *out = A + ((long long)c * rows + row) * L;
#pragma unroll
      for (int k2 = 0; k2 < S::R2; ++k2)
        out[(lt + S::R1 * k2 + out_add) & (L - 1)] = bv[k2];
    }
  }
}

// --------------------------------------------------------------------------
// adjoint rows: inverse DFT along x, crop + shift, scale, deapodization,
// conj(sens) coil sum
// --------------------------------------------------------------------------
// Per-coil outputs (stage 1, or no maps): one line per (row, coil), coil
// fastest.
template <int L>
__global__ void __launch_bounds__(kFftThreads, L <= 256 ? 3 : 1)
    k_fft_rows_adj_coils(const float2 *__restrict__ A,
                         const float *__restrict__ deapo, int Nx,
                         long long rows, long long N, int C, int out_add,
                         float scale, int stage,
                         const float2 *__restrict__ roots,
                         float2 *__restrict__ out)
{
  using S = Shape<L>;
  extern __shared__ float2 sm[];
  float2 *tw = sm;
  load_roots(tw, roots, L);
  const int line = threadIdx.x / S::T, lt = threadIdx.x % S::T;
  const long long ln = (long long)blockIdx.x * S::NL + line;
  const bool on = ln < rows * C;
  const long long row = on ? ln / C : 0;
  const int c = on ? (int)(ln - row * C) : 0;
  float2 *Y = sm + L + line * S::R1 * S::YP;
  __syncthreads();
  float2 w[Rm<L>::V / 2];
  load_reg_roots<L>(w, tw);
  if (lt < S::R2 && on)
  {
    const float2 *in = A + ((long long)c * rows + row) * L;
    float2 a[S::R1];
#pragma unroll
    for (int j = 0; j < S::R1; ++j)
      a[j] = __ldg(in + lt + S::R2 * j);
    stage1<L, true, 1>(a, lt, w, tw, Y);
  }
  __syncthreads();
  if (lt < S::R1 && on)
  {
    float2 b[S::R2];
    stage2<L, true, 1>(b, lt, w, Y);
#pragma unroll
    for (int k2 = 0; k2 < S::R2; ++k2)
    {
      // FFT output k = lt + R1 k2 holds image x (k + out_add) mod L
      const int xp = (lt + S::R1 * k2 + out_add) & (L - 1);
      if (xp >= Nx)
        continue;
      const long long px = row * Nx + xp;
      // crop -> FFT scaling -> deapodization (gpuNUFFT_operator.cpp:800-819)
      float2 v = make_float2(__fmul_rn(b[k2].x, scale),
                             __fmul_rn(b[k2].y, scale));
      if (stage == 2)
      {
        const float d = __ldg(deapo + px);
        v.x = __fmul_rn(v.x, d);
        v.y = __fmul_rn(v.y, d);
      }
      out[c * N + px] = v;
    }
  }
}

// With maps (stage 2): the block owns RPB image rows and runs their coils
// in chunks of CPC (lines = RPB x CPC); each chunk's conj(S) * v terms go
// through shared memory and are added to the rows' running sums in coil
// order, so the sum order is fixed.
template <int L>
__global__ void __launch_bounds__(kFftThreads, L <= 256 ? 3 : 1)
    k_fft_rows_adj_sum(const float2 *__restrict__ A,
                       const float *__restrict__ deapo,
                       const float2 *__restrict__ sens, int Nx, long long rows,
                       long long N, int C, int cpc, int out_add, float scale,
                       int accumulate, const float2 *__restrict__ roots,
                       float2 *__restrict__ out)
{
  using S = Shape<L>;
  extern __shared__ float2 sm[];
  float2 *tw = sm;
  float2 *Ybase = sm + L;                       // exchange, then terms
  float2 *accS = Ybase + S::NL * S::R1 * S::YP;  // [rpb][Nx] running sums
  load_roots(tw, roots, L);
  const int rpb = S::NL / cpc;
  const int line = threadIdx.x / S::T, lt = threadIdx.x % S::T;
  const int rl = line / cpc, cl = line - rl * cpc;
  const long long row = (long long)blockIdx.x * rpb + rl;
  const bool row_on = row < rows;
  float2 *Y = Ybase + line * S::R1 * S::YP;
  float2 *term = Ybase + (size_t)line * Nx;  // aliases the exchange area
  for (int i = threadIdx.x; i < rpb * Nx; i += kFftThreads)
    accS[i] = make_float2(0.f, 0.f);
  __syncthreads();
  float2 w[Rm<L>::V / 2];
  load_reg_roots<L>(w, tw);
  for (int c0 = 0; c0 < C; c0 += cpc)
  {
    const int c = c0 + cl;
    const bool on = row_on && c < C;
    if (lt < S::R2 && on)
    {
      const float2 *in = A + ((long long)c * rows + row) * L;
      float2 a[S::R1];
#pragma unroll
      for (int j = 0; j < S::R1; ++j)
        a[j] = __ldg(in + lt + S::R2 * j);
      stage1<L, true, 1>(a, lt, w, tw, Y);
    }
    __syncthreads();
    float2 b[S::R2];
    if (lt < S::R1 && on)
      stage2<L, true, 1>(b, lt, w, Y);
    __syncthreads();  // the exchange area becomes the term area
    if (lt < S::R1)
    {
#pragma unroll
      for (int k2 = 0; k2 < S::R2; ++k2)
      {
        const int xp = (lt + S::R1 * k2 + out_add) & (L - 1);
        if (xp >= Nx)
          continue;
        float2 t = make_float2(0.f, 0.f);
        if (on)
        {
          const long long px = row * Nx + xp;
          // crop -> FFT scaling -> deapodization -> conj(S) * v
          // (gpuNUFFT_operator.cpp:800-843, std_gpuNUFFT_kernels.cu:158-218)
          float2 v = make_float2(__fmul_rn(b[k2].x, scale),
                                 __fmul_rn(b[k2].y, scale));
          const float d = __ldg(deapo + px);
          v.x = __fmul_rn(v.x, d);
          v.y = __fmul_rn(v.y, d);
          const float2 s = __ldg(sens + c * N + px);
          t = cmul_conj(v, s);
        }
        term[xp] = t;
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < rpb * Nx; i += kFftThreads)
    {
      const int r = i / Nx, x = i - r * Nx;
      float2 sum = accS[i];
      const int nc = min(cpc, C - c0);
      for (int k = 0; k < nc; ++k)
      {
        const float2 t = Ybase[(size_t)(r * cpc + k) * Nx + x];
        sum.x += t.x;
        sum.y += t.y;
      }
      accS[i] = sum;
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < rpb * Nx; i += kFftThreads)
  {
    const int r = i / Nx, x = i - r * Nx;
    const long long rr = (long long)blockIdx.x * rpb + r;
    if (rr >= rows)
      continue;
    float2 v = accS[i];
    if (accumulate)
    {
      const float2 o = out[rr * Nx + x];
      v = make_float2(o.x + v.x, o.y + v.y);
    }
    out[rr * Nx + x] = v;
  }
}

// --------------------------------------------------------------------------
// dispatch
// --------------------------------------------------------------------------
inline int pos_mod(long long v, int m)
{
  long long r = v % m;
  return (int)(r < 0 ? r + m : r);
}

template <class F> void with_length(int L, F &&f)
{
  switch (L)
  {
  case 16: f(std::integral_constant<int, 16>()); break;
  case 32: f(std::integral_constant<int, 32>()); break;
  case 64: f(std::integral_constant<int, 64>()); break;
  case 128: f(std::integral_constant<int, 128>()); break;
  case 256: f(std::integral_constant<int, 256>()); break;
  case 512: f(std::integral_constant<int, 512>()); break;
  case 1024: f(std::integral_constant<int, 1024>()); break;
  default: throw Error(kInternal, "pruned transform length not supported");
  }
}

template <class K> void set_smem(K kernel, size_t bytes)
{
  if (bytes > 48 * 1024)
    GN_CUDA(cudaFuncSetAttribute(kernel,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)bytes));
}

// Tensor map of planes x rows x columns of complex values (columns
// contiguous), box TC columns x box_rows rows x 1 plane.  False when TMA is
// unavailable or the layout does not meet its alignment rules.
bool col_tensor_map(CUtensorMap &tm, const float2 *base, long long ncols,
                    int rows, long long plane_stride, long long planes, int TC,
                    int box_rows)
{  // TC: columns per box (a multiple of 2)
  tma::EncodeTiledFn enc = tma::encode_fn();
  if (!enc || (ncols & 1) || (plane_stride & 1) ||
      (reinterpret_cast<uintptr_t>(base) & 15))
    return false;
  cuuint64_t dims[3] = {(cuuint64_t)ncols, (cuuint64_t)rows,
                        (cuuint64_t)planes};
  cuuint64_t strides[2] = {(cuuint64_t)ncols * sizeof(float2),
                           (cuuint64_t)plane_stride * sizeof(float2)};
  cuuint32_t box[3] = {(cuuint32_t)TC, (cuuint32_t)box_rows, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  return enc(&tm, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3,
             const_cast<float2 *>(base), dims, strides, box, estr,
             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
             CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tensor maps of the coil-pair tiles with interleaved half rows: 4-D
// (columns, coil in pair, rows, pair), box CW columns x 2 coils x box_rows
// rows x 1 pair, so that the box lands in shared memory as rows of CW
// columns of the first coil followed by CW of the second.  `tm` covers the
// planes / 2 whole pairs; with an odd plane count, `tail` covers the last
// plane as a pair whose second coil is out of range (zero fill).  False
// when TMA is unavailable or rejects the layout.
bool col_pair_tensor_maps(CUtensorMap &tm, CUtensorMap &tail,
                          const float2 *base, long long ncols, int rows,
                          long long plane_stride, long long planes, int CW,
                          int box_rows)
{
  tma::EncodeTiledFn enc = tma::encode_fn();
  if (!enc || (ncols & 1) || (plane_stride & 1) ||
      (reinterpret_cast<uintptr_t>(base) & 15))
    return false;
  auto make = [&](CUtensorMap &m, const float2 *b, long long coils,
                  long long pairs) {
    cuuint64_t dims[4] = {(cuuint64_t)ncols, (cuuint64_t)coils,
                          (cuuint64_t)rows, (cuuint64_t)pairs};
    cuuint64_t strides[3] = {(cuuint64_t)plane_stride * sizeof(float2),
                             (cuuint64_t)ncols * sizeof(float2),
                             (cuuint64_t)(2 * plane_stride) * sizeof(float2)};
    cuuint32_t box[4] = {(cuuint32_t)CW, 2, (cuuint32_t)box_rows, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    return enc(&m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 4,
               const_cast<float2 *>(b), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  const long long pairs = planes / 2;
  if (planes & 1)
  {
    if (!make(tail, base + (planes - 1) * plane_stride, 1, 1))
      return false;
    if (pairs == 0)
    {
      tm = tail;
      return true;
    }
  }
  if (!make(tm, base, 2, pairs))
    return false;
  if (!(planes & 1))
    tail = tm;
  return true;
}

// Persistent blocks of the tensor-copy passes: three per SM.
unsigned persistent_blocks(long long work)
{
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long cap = 3LL * sms;
  return (unsigned)(work < cap ? work : cap);
}

template <bool INV>
void cols(int L, const float2 *src, float2 *dst, long long ncols,
          int src_rows, int dst_rows, long long planes, int in_add,
          int in_count, int out_add, int out_count, const float2 *roots,
          cudaStream_t s, const uint2 *colrange = nullptr,
          tma::CopyWait wait = tma::CopyWait(), bool paired = false,
          const uint32_t *tiles = nullptr, long long n_list = 0,
          int list_cols = 0)
{
  bool done = false;
  if (wait.err && L <= 256)
    with_length(L, [&](auto lc) {
      constexpr int LL = decltype(lc)::value;
      if constexpr (LL <= 256)
      {
        using S = Shape<LL>;
        const int box_rows = src_rows < 256 ? src_rows : 256;
        const int ncopy = (src_rows + box_rows - 1) / box_rows;
        // paired: boxes of TC / 2 columns of one plane, two per tile
        const int cw = paired ? S::TC / 2 : S::TC;
        if (paired && ncopy != 1)
          return;
        CUtensorMap tm, tail;
        long long tail_pl = -1;
        // paired: interleaved half rows (one 4-D box) where the tensor
        // maps take that layout, else two planes
        int mode = 0;
        if (paired &&
            col_pair_tensor_maps(tm, tail, src, ncols, src_rows,
                                 (long long)src_rows * ncols, planes, cw,
                                 box_rows))
        {
          mode = 2;
          if (planes & 1)
            tail_pl = planes / 2;
        }
        else
        {
          if (!col_tensor_map(tm, src, ncols, src_rows,
                              (long long)src_rows * ncols, planes, cw,
                              box_rows))
            return;
          tail = tm;
          mode = paired ? 1 : 0;
        }
        // a list of the column tiles to transform (paired, same width)
        const bool listed = paired && tiles && list_cols == cw;
        const long long n_ct = listed ? n_list : (ncols + cw - 1) / cw;
        if (n_ct == 0)
        {
          done = true;  // no column carries a range: nothing to write
          return;
        }
        const long long n_tiles = n_ct * (paired ? (planes + 1) / 2 : planes);
        if (n_tiles >= (1LL << 31) - 2LL * persistent_blocks(n_tiles))
          return;  // tile indices are 31-bit
        auto launch = [&](auto k, int threads) {
          set_smem(k, ColTma<LL>::smem());
          k<<<persistent_blocks(n_tiles), threads, ColTma<LL>::smem(), s>>>(
              tm, tail, tail_pl, dst, ncols, FastDiv((uint32_t)n_ct),
              (int)n_tiles, box_rows, ncopy,
              dst_rows, in_add, in_count, out_add, out_count, roots, colrange,
              listed ? tiles : nullptr, wait);
        };
        // the interleaved coil-pair pass (twice the lines of the others,
        // bound by instruction issue) runs two adjacent columns per thread;
        // the plain passes, closer to the DRAM bound, keep the warps of one
        // column per thread
        if (mode == 2)
          launch(k_fft_cols_tma<LL, INV, 2, 2>, S::CT / 2);
        else if (mode == 1)
          launch(k_fft_cols_tma<LL, INV, 1>, S::CT);
        else
          launch(k_fft_cols_tma<LL, INV, 0>, S::CT);
        GN_LAUNCH_CHECK("pruned column transform (tensor-copy tiles)");
        done = true;
      }
    });
  if (done)
    return;
  if (paired)
    throw Error(kInternal, "interleaved coil pairs need the tensor-copy pass");
  with_length(L, [&](auto lc) {
    constexpr int LL = decltype(lc)::value;
    using S = Shape<LL>;
    auto k = k_fft_cols<LL, INV>;
    set_smem(k, S::col_smem());
    if (planes > 65535)
      throw Error(kNotSupported, "too many planes for the pruned transform");
    const dim3 grid((unsigned)((ncols + S::TC - 1) / S::TC),
                    (unsigned)planes);
    k<<<grid, S::CT, S::col_smem(), s>>>(src, dst, ncols, src_rows,
                                          dst_rows, in_add, in_count, out_add,
                                          out_count, roots, colrange);
    GN_LAUNCH_CHECK("pruned column transform");
  });
}

// The coil-combining last adjoint pass on tensor-copy tiles, where it
// applies: lengths up to 256, two blocks per SM, layouts the tensor maps
// take.  False (nothing launched) otherwise.
template <int L>
bool launch_cols_sum_tma(const float2 *src, long long ncols,
                         long long coil_stride, const float *deapo,
                         const float2 *sens, int n_out, long long N, int C,
                         int groups, int cpb, int out_add, float scale,
                         int accumulate, const float2 *roots, float2 *out,
                         float2 *partial, tma::CopyWait cw, cudaStream_t s)
{
  if constexpr (L > 256)
    return false;
  else
  {
    using S = Shape<L>;
    const size_t smem = SumTma<L>::smem(n_out);
    if (!cw.err || smem > 113 * 1024 || n_out > L || (N & 1))
      return false;
    CUtensorMap src_map, sens_map;
    if (!col_tensor_map(src_map, src, ncols, L, coil_stride, C, S::TC, L) ||
        !col_tensor_map(sens_map, sens, ncols, n_out, N, C, S::TC, n_out))
      return false;
    const long long nb = (ncols + S::TC - 1) / S::TC;
    const long long n_units = nb * groups;
    if (n_units >= (1LL << 30))
      return false;  // unit indices are 31-bit
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long blocks = n_units < 2LL * sms ? n_units : 2LL * sms;
    auto k = k_fft_cols_sum_tma<L>;
    set_smem(k, smem);
    k<<<(unsigned)blocks, S::CT, smem, s>>>(
        src_map, sens_map, ncols, (int)n_units, FastDiv((uint32_t)groups),
        cpb, C, deapo, n_out, N,
        out_add, scale, accumulate, roots, out, partial, cw);
    GN_LAUNCH_CHECK("pruned adjoint last pass (tensor-copy tiles)");
    return true;
  }
}

// The forward row pass on tensor-copy tiles, where it applies (see
// k_fft_rows_fwd_tma); false (nothing launched) otherwise.
template <int L>
bool launch_rows_fwd_tma(const float2 *image, const float2 *sens,
                         const float *deapo, int Nx, long long rows,
                         long long N, int C, int in_add, int out_add,
                         const float2 *roots, float2 *A, tma::CopyWait cw,
                         cudaStream_t s)
{
  if constexpr (L > 256)
    return false;
  else
  {
    using S = Shape<L>;
    constexpr int NL = S::NL;
    const float2 *coils = sens ? sens : image;
    tma::EncodeTiledFn enc = tma::encode_fn();
    if (!enc || !cw.err || C < NL || Nx > 256 || Nx > L || (Nx & 3) ||
        (reinterpret_cast<uintptr_t>(image) & 15) ||
        (reinterpret_cast<uintptr_t>(coils) & 15) ||
        (reinterpret_cast<uintptr_t>(deapo) & 15))
      return false;
    const size_t smem = 2 * (size_t)RowsTma::stage_bytes(NL, Nx) +
                        (size_t)L * sizeof(float2) +
                        (size_t)NL * S::R1 * S::YP * sizeof(float2) + 2 * 8 +
                        16;
    if (smem > 113 * 1024)
      return false;
    // coil rows: (pixel, coil), box N_x pixels x NL coils
    CUtensorMap tm;
    cuuint64_t dims[2] = {(cuuint64_t)N, (cuuint64_t)C};
    cuuint64_t strides[1] = {(cuuint64_t)N * sizeof(float2)};
    cuuint32_t box[2] = {(cuuint32_t)Nx, (cuuint32_t)NL};
    cuuint32_t estr[2] = {1, 1};
    if (enc(&tm, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2,
            const_cast<float2 *>(coils), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
    const int n_cc = (C + NL - 1) / NL;
    const long long n_jobs = rows * n_cc;
    if (n_jobs >= (1LL << 30))
      return false;  // job indices are 31-bit
    auto launch = [&](auto k) {
      set_smem(k, smem);
      int dev = 0, sms = 148, per_sm = 1;
      if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
              &per_sm, k, kFftThreads, smem) != cudaSuccess ||
          per_sm < 1)
        per_sm = 1;
      const long long cap = (long long)per_sm * sms;
      k<<<(unsigned)(n_jobs < cap ? n_jobs : cap), kFftThreads, smem, s>>>(
          tm, image, deapo, Nx, rows, C, (int)n_jobs, FastDiv((uint32_t)n_cc),
          in_add, out_add, roots, A, cw);
    };
    if (sens)
      launch(k_fft_rows_fwd_tma<L, true>);
    else
      launch(k_fft_rows_fwd_tma<L, false>);
    GN_LAUNCH_CHECK("pruned forward rows (tensor-copy tiles)");
    return true;
  }
}

}  // namespace

bool pruned_fft_supported(const Geo &g)
{
  for (int a = 0; a < g.dim; ++a)
  {
    const int G = g.G[a];
    if (G < 16 || G > 1024 || (G & (G - 1)))
      return false;
  }
  return true;
}

void fft_roots(int L, std::vector<float2> &tab)
{
  tab.resize(L);
  const double two_pi = 6.283185307179586476925286766559;
  for (int j = 0; j < L; ++j)
  {
    const double ang = -two_pi * (double)j / (double)L;
    tab[j] = make_float2((float)std::cos(ang), (float)std::sin(ang));
  }
}

size_t pruned_scratch_a(const Geo &g, int C)
{
  return (size_t)C * g.N[2] * g.N[1] * g.G[0];
}

size_t pruned_scratch_b(const Geo &g, int C)
{
  return g.dim == 3 ? (size_t)C * g.N[2] * g.G[1] * g.G[0] : 0;
}

void launch_pruned_forward(const float2 *image, const float2 *sens,
                           const float *deapo, const Geo &g, int C,
                           const float2 *const roots[3], float2 *tmp_a,
                           float2 *tmp_b, float2 *grid, cudaStream_t s,
                           const uint2 *zrange, tma::CopyWait cw,
                           bool paired, const uint32_t *ztiles, int n_ztiles,
                           int ztile_cols)
{
  const long long N = g.img_count;
  const long long rows = (long long)g.N[1] * g.N[2];
  // x: image rows -> A [C][N_z][N_y][G_x]
  with_length(g.G[0], [&](auto lc) {
    constexpr int LL = decltype(lc)::value;
    using S = Shape<LL>;
    const long long nb = (rows * C + S::NL - 1) / S::NL;
    const int in_add = pos_mod((long long)g.shift_inv[0] - g.crop[0], g.G[0]);
    // the FORWARD fftshift: frequency k is stored at (k - ceil(G/2)) mod G
    const int out_add = pos_mod(-(long long)g.shift_fwd[0], g.G[0]);
    if (launch_rows_fwd_tma<LL>(image, sens, deapo, g.N[0], rows, N, C,
                                in_add, out_add, roots[0], tmp_a, cw, s))
      return;
    if (sens)
    {
      auto k = k_fft_rows_fwd<LL, true>;
      set_smem(k, S::smem());
      k<<<(unsigned)nb, kFftThreads, S::smem(), s>>>(
          image, sens, deapo, g.N[0], rows, N, C, in_add, out_add, roots[0],
          tmp_a);
    }
    else
    {
      auto k = k_fft_rows_fwd<LL, false>;
      set_smem(k, S::smem());
      k<<<(unsigned)nb, kFftThreads, S::smem(), s>>>(
          image, sens, deapo, g.N[0], rows, N, C, in_add, out_add, roots[0],
          tmp_a);
    }
    GN_LAUNCH_CHECK("pruned forward rows");
  });
  // y: A -> (3-D) B [C][N_z][G_y][G_x] or (2-D) the grid
  float2 *ydst = g.dim == 3 ? tmp_b : grid;
  cols<false>(g.G[1], tmp_a, ydst, g.G[0], g.N[1], g.G[1],
              (long long)C * g.N[2],
              pos_mod((long long)g.shift_inv[1] - g.crop[1], g.G[1]), g.N[1],
              pos_mod(-(long long)g.shift_fwd[1], g.G[1]), g.G[1], roots[1],
              s, nullptr, cw);
  if (g.dim == 3)  // z: B -> grid
    cols<false>(g.G[2], tmp_b, grid, (long long)g.G[1] * g.G[0], g.N[2],
                g.G[2], C,
                pos_mod((long long)g.shift_inv[2] - g.crop[2], g.G[2]),
                g.N[2], pos_mod(-(long long)g.shift_fwd[2], g.G[2]), g.G[2],
                roots[2], s, zrange, cw, paired, ztiles, n_ztiles,
                ztile_cols);
}

void launch_pruned_adjoint(const float2 *grid, const float *deapo,
                           const float2 *sens, const Geo &g, int C, int stage,
                           int accumulate, const float2 *const roots[3],
                           float2 *tmp_a, float2 *tmp_b, float2 *out,
                           cudaStream_t s)
{
  const long long N = g.img_count;
  const long long rows = (long long)g.N[1] * g.N[2];
  const float2 *ysrc = grid;
  if (g.dim == 3)
  {  // z: grid -> B [C][N_z][G_y][G_x]
    cols<true>(g.G[2], grid, tmp_b, (long long)g.G[1] * g.G[0], g.G[2],
               g.N[2], C, 0, g.G[2],
               pos_mod(-(long long)g.crop[2] - g.shift_inv[2], g.G[2]),
               g.N[2], roots[2], s);
    ysrc = tmp_b;
  }
  // y: -> A [C][N_z][N_y][G_x]
  cols<true>(g.G[1], ysrc, tmp_a, g.G[0], g.G[1], g.N[1],
             (long long)C * g.N[2], 0, g.G[1],
             pos_mod(-(long long)g.crop[1] - g.shift_inv[1], g.G[1]), g.N[1],
             roots[1], s);
  // x + image stages
  with_length(g.G[0], [&](auto lc) {
    constexpr int LL = decltype(lc)::value;
    using S = Shape<LL>;
    const int out_add =
        pos_mod(-(long long)g.crop[0] - g.shift_inv[0], g.G[0]);
    if (sens != nullptr && stage == 2)
    {
      int cpc = 1;
      while (cpc < C && cpc < S::NL)
        cpc <<= 1;
      const int rpb = S::NL / cpc;
      const size_t smem =
          S::smem() + (size_t)rpb * g.N[0] * sizeof(float2);
      auto k = k_fft_rows_adj_sum<LL>;
      set_smem(k, smem);
      k<<<(unsigned)((rows + rpb - 1) / rpb), kFftThreads, smem, s>>>(
          tmp_a, deapo, sens, g.N[0], rows, N, C, cpc, out_add, g.fft_scale,
          accumulate, roots[0], out);
    }
    else
    {
      auto k = k_fft_rows_adj_coils<LL>;
      set_smem(k, S::smem());
      k<<<(unsigned)((rows * C + S::NL - 1) / S::NL), kFftThreads, S::smem(),
          s>>>(tmp_a, deapo, g.N[0], rows, N, C, out_add, g.fft_scale, stage,
               roots[0], out);
    }
    GN_LAUNCH_CHECK("pruned adjoint rows");
  });
}


void launch_pruned_adjoint_xfirst(const float2 *xrows, const float *deapo,
                                  const float2 *sens, const Geo &g, int C,
                                  int stage, int accumulate,
                                  const float2 *const roots[3],
                                  float2 *tmp_b, float2 *part, float2 *out,
                                  cudaStream_t s, tma::CopyWait cw)
{
  const long long N = g.img_count;
  const float2 *src = xrows;
  long long ncols = g.N[0];
  int ax = 1;  // the axis of the last pass
  if (g.dim == 3)
  {  // y: [C][G_z][G_y][N_x] -> [C][G_z][N_y][N_x]
    cols<true>(g.G[1], xrows, tmp_b, g.N[0], g.G[1], g.N[1],
               (long long)C * g.G[2], 0, g.G[1],
               pos_mod(-(long long)g.crop[1] - g.shift_inv[1], g.G[1]),
               g.N[1], roots[1], s, nullptr, cw);
    src = tmp_b;
    ncols = (long long)g.N[1] * g.N[0];
    ax = 2;
  }
  const long long coil_stride = (long long)g.G[ax] * ncols;
  const int out_add =
      pos_mod(-(long long)g.crop[ax] - g.shift_inv[ax], g.G[ax]);
  with_length(g.G[ax], [&](auto lc) {
    constexpr int LL = decltype(lc)::value;
    using S = Shape<LL>;
    const long long nb = (ncols + S::TC - 1) / S::TC;
    // coil groups in separate blocks when the columns alone do not fill
    // the GPU (eight blocks per SM); their coil sums meet in `partial`
    int groups = 1;
    while (groups < C && nb * groups < 148LL * 8)
      groups *= 2;
    if (groups > C)
      groups = C;
    const int cpb = (C + groups - 1) / groups;
    groups = (C + cpb - 1) / cpb;
    const bool combine = sens != nullptr && stage == 2;
    float2 *partial = (combine && groups > 1) ? part : nullptr;
    const dim3 grd((unsigned)nb, (unsigned)groups);
    const bool tiles =
        combine && launch_cols_sum_tma<LL>(src, ncols, coil_stride, deapo,
                                           sens, g.N[ax], N, C, groups, cpb,
                                           out_add, g.fft_scale, accumulate,
                                           roots[ax], out, partial, cw, s);
    if (combine && !tiles)
    {
      auto k = k_fft_cols_sum<LL, true>;
      set_smem(k, S::col_smem());
      k<<<grd, S::CT, S::col_smem(), s>>>(src, ncols, coil_stride, deapo,
                                         sens, g.N[ax], N, C, cpb, out_add,
                                         g.fft_scale, stage, accumulate,
                                         roots[ax], out, partial);
    }
    else if (!combine)
    {
      auto k = k_fft_cols_sum<LL, false>;
      set_smem(k, S::col_smem());
      k<<<grd, S::CT, S::col_smem(), s>>>(src, ncols, coil_stride, deapo,
                                         nullptr, g.N[ax], N, C, cpb, out_add,
                                         g.fft_scale, stage, accumulate,
                                         roots[ax], out, nullptr);
    }
    GN_LAUNCH_CHECK("pruned adjoint last pass");
    if (partial)
    {
      k_sum_coil_groups<<<grid_for(N, 256, 148 * 16), 256, 0, s>>>(
          partial, groups, N, accumulate, out);
      GN_LAUNCH_CHECK("coil-group sum");
    }
  });
}

size_t pruned_scratch_xfirst(const Geo &g, int C)
{
  return g.dim == 3 ? (size_t)C * g.G[2] * g.N[1] * g.N[0] : 0;
}

}  // namespace gnufft
