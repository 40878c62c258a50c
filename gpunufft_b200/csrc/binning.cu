// Plan-time integer kernels: sector assignment, stable radix sort, scans and
// owner candidate lists.  All results are deterministic (no atomics decide
// an order) and integer-exact.
#include "binning.cuh"

#include <algorithm>
#include <vector>

#include "footprint.cuh"

namespace gnufft
{
namespace
{
constexpr int kScanThreads = 256;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_inclusive_scan(uint32_t v)
{
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1)
  {
    uint32_t n = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o)
      v += n;
  }
  return v;
}

// Block-local exclusive scan of a 1024-item tile; block totals to `sums`.
__global__ void __launch_bounds__(kScanThreads)
    k_scan_tile(const uint32_t *__restrict__ in, uint32_t *__restrict__ out,
                uint32_t *__restrict__ sums, size_t n)
{
  __shared__ uint32_t warp_tot[kScanThreads / 32];
  const size_t base = (size_t)blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  uint32_t v[kScanItems];
  uint32_t tsum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i)
  {
    v[i] = (base + i < n) ? in[base + i] : 0u;
    tsum += v[i];
  }
  uint32_t incl = warp_inclusive_scan(tsum);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 31)
    warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0)
  {
    uint32_t w = lane < kScanThreads / 32 ? warp_tot[lane] : 0u;
    uint32_t wi = warp_inclusive_scan(w);
    if (lane < kScanThreads / 32)
      warp_tot[lane] = wi - w;  // exclusive warp offsets
    if (lane == kScanThreads / 32 - 1 && sums)
      sums[blockIdx.x] = wi;
  }
  __syncthreads();
  uint32_t run = warp_tot[warp] + incl - tsum;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i)
  {
    if (base + i < n)
      out[base + i] = run;
    run += v[i];
  }
}

__global__ void k_scan_add(uint32_t *__restrict__ out,
                           const uint32_t *__restrict__ offs, size_t n)
{
  const size_t base = (size_t)blockIdx.x * kScanTile;
  const uint32_t o = offs[blockIdx.x];
  for (int i = threadIdx.x; i < kScanTile; i += blockDim.x)
    if (base + i < n)
      out[base + i] += o;
}

constexpr int kSortThreads = 256;
constexpr int kSortRounds = 16;
constexpr int kSortTile = kSortThreads * kSortRounds;
constexpr int kSortWarps = kSortThreads / 32;

__global__ void __launch_bounds__(kSortThreads)
    k_radix_hist(const uint32_t *__restrict__ keys, size_t n, int shift,
                 uint32_t *__restrict__ hist)
{
  __shared__ uint32_t h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  const size_t base = (size_t)blockIdx.x * kSortTile;
  for (int i = threadIdx.x; i < kSortTile; i += kSortThreads)
    if (base + i < n)
      atomicAdd(&h[(keys[base + i] >> shift) & 255u], 1u);
  __syncthreads();
  hist[(size_t)threadIdx.x * gridDim.x + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter of one 8-bit digit: items keep their input order within a
// digit (block order via the digit-major scan, (round, warp, lane) order
// inside a block).
__global__ void __launch_bounds__(kSortThreads)
    k_radix_scatter(const uint32_t *__restrict__ kin,
                    const uint32_t *__restrict__ vin,
                    uint32_t *__restrict__ kout, uint32_t *__restrict__ vout,
                    size_t n, int shift, const uint32_t *__restrict__ offs)
{
  __shared__ uint32_t run[256];
  __shared__ uint32_t wcnt[kSortWarps][256];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  run[tid] = offs[(size_t)tid * gridDim.x + blockIdx.x];
  const size_t base = (size_t)blockIdx.x * kSortTile;
  for (int r = 0; r < kSortRounds; ++r)
  {
    for (int i = tid; i < kSortWarps * 256; i += kSortThreads)
      (&wcnt[0][0])[i] = 0;
    __syncthreads();
    const size_t j = base + (size_t)r * kSortThreads + tid;
    const bool valid = j < n;
    const uint32_t k = valid ? kin[j] : 0u;
    const uint32_t d = (k >> shift) & 255u;
    const unsigned peers =
        __match_any_sync(0xffffffffu, valid ? d : 0xffffffffu);
    const int rank = __popc(peers & ((1u << lane) - 1u));
    if (valid && lane == __ffs(peers) - 1)
      wcnt[warp][d] = __popc(peers);
    __syncthreads();
    {
      uint32_t acc = run[tid];
#pragma unroll
      for (int w = 0; w < kSortWarps; ++w)
      {
        uint32_t c = wcnt[w][tid];
        wcnt[w][tid] = acc;
        acc += c;
      }
      run[tid] = acc;
    }
    __syncthreads();
    if (valid)
    {
      const uint32_t pos = wcnt[warp][d] + rank;
      kout[pos] = k;
      vout[pos] = vin[j];
    }
    __syncthreads();
  }
}

__global__ void k_count_keys(const uint32_t *__restrict__ keys, size_t n,
                             uint32_t *__restrict__ counts)
{
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    atomicAdd(&counts[keys[i]], 1u);
}

__global__ void k_assign(const float *__restrict__ traj, uint32_t M, Geo g,
                         uint32_t *__restrict__ sector)
{
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < M;
       i += (size_t)gridDim.x * blockDim.x)
  {
    uint32_t s = 0, stride = 1;
    for (int a = 0; a < g.dim; ++a)
    {
      uint32_t sa = sector_of_axis(traj[(size_t)a * M + i], g.Gf[a],
                                   (float)g.sw);
      s += sa * stride;
      stride *= (uint32_t)g.S[a];
    }
    sector[i] = s;
  }
}

__global__ void k_gather(const float *__restrict__ traj,
                         const float *__restrict__ dens,
                         const uint32_t *__restrict__ idx, uint32_t M, int dim,
                         float *__restrict__ traj_sorted,
                         float *__restrict__ dens_sorted)
{
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < M;
       t += (size_t)gridDim.x * blockDim.x)
  {
    const uint32_t j = idx[t];
    for (int a = 0; a < dim; ++a)
      traj_sorted[(size_t)a * M + t] = traj[(size_t)a * M + j];
    if (dens)
      dens_sorted[t] = dens[j];
  }
}

__device__ __forceinline__ void split_sector(uint32_t s, const Geo &g,
                                             int *sa)
{
  sa[0] = (int)(s % (uint32_t)g.S[0]);
  uint32_t r = s / (uint32_t)g.S[0];
  sa[1] = (int)(r % (uint32_t)g.S[1]);
  sa[2] = (int)(r / (uint32_t)g.S[1]);
}

// Every (cell, weight) of the footprint of sorted sample t.
template <bool FILL>
__global__ void k_interp_pairs(const float *__restrict__ traj_sorted,
                               const uint32_t *__restrict__ sector_sorted,
                               uint32_t M, Geo g, const float *__restrict__ lut,
                               uint32_t *__restrict__ count,
                               const uint32_t *__restrict__ pos,
                               uint32_t *__restrict__ keys,
                               uint32_t *__restrict__ ids,
                               uint2 *__restrict__ pairs)
{
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < M;
       t += (size_t)gridDim.x * blockDim.x)
  {
    int sa[3];
    split_sector(sector_sorted[t], g, sa);
    int cell[3][kSlots];
    float w[3][kSlots];
    int n[3] = {1, 1, 1};
    cell[2][0] = 0;
    w[2][0] = 1.0f;
    for (int a = 0; a < g.dim; ++a)
      n[a] = axis_footprint(traj_sorted[(size_t)a * M + t], a, sa[a], g, lut,
                            cell[a], w[a]);
    if (!FILL)
    {
      count[t] = (uint32_t)(n[0] * n[1] * n[2]);
      continue;
    }
    uint32_t p = pos[t];
    for (int z = 0; z < n[2]; ++z)
      for (int y = 0; y < n[1]; ++y)
      {
        // upstream weight order: (K[z] * K[y]) * K[x]
        const float wzy = g.dim == 3 ? __fmul_rn(w[2][z], w[1][y]) : w[1][y];
        const uint32_t rowc =
            ((uint32_t)cell[2][z] * (uint32_t)g.G[1] + (uint32_t)cell[1][y]) *
            (uint32_t)g.G[0];
        for (int x = 0; x < n[0]; ++x)
        {
          keys[p] = rowc + (uint32_t)cell[0][x];
          ids[p] = p;
          pairs[p] = make_uint2((uint32_t)t,
                                __float_as_uint(__fmul_rn(wzy, w[0][x])));
          ++p;
        }
      }
  }
}

__global__ void k_gather_pairs(const uint32_t *__restrict__ ids,
                               const uint2 *__restrict__ pairs, size_t n,
                               uint2 *__restrict__ out)
{
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = pairs[ids[i]];
}

int bits_for(uint32_t max_value)
{
  int b = 1;
  while (b < 32 && (max_value >> b) != 0)
    ++b;
  return b;
}
}  // namespace

size_t scan_scratch_elems(size_t n)
{
  const size_t nb = (n + kScanTile - 1) / kScanTile;
  return nb <= 1 ? 0 : nb + scan_scratch_elems(nb);
}

void scan_exclusive(const uint32_t *in, uint32_t *out, size_t n,
                    cudaStream_t s, uint32_t *scratch)
{
  if (n == 0)
    return;
  const size_t nb = (n + kScanTile - 1) / kScanTile;
  if (nb == 1)
  {
    k_scan_tile<<<1, kScanThreads, 0, s>>>(in, out, nullptr, n);
    GN_LAUNCH_CHECK("scan");
    return;
  }
  DeviceBuffer own;
  if (!scratch)
  {
    own.reset(scan_scratch_elems(n) * sizeof(uint32_t));
    scratch = own.as<uint32_t>();
  }
  uint32_t *sums = scratch;  // this level's block sums, then the next level's
  k_scan_tile<<<(unsigned)nb, kScanThreads, 0, s>>>(in, out, sums, n);
  GN_LAUNCH_CHECK("scan");
  scan_exclusive(sums, sums, nb, s, sums + nb);
  k_scan_add<<<(unsigned)nb, kScanThreads, 0, s>>>(out, sums, n);
  GN_LAUNCH_CHECK("scan add");
  if (own.get())
    GN_CUDA(cudaStreamSynchronize(s));  // `own` is released on return
}

void sort_pairs(const uint32_t *keys_in, const uint32_t *vals_in,
                uint32_t *keys_out, uint32_t *vals_out, size_t n, int key_bits,
                cudaStream_t s)
{
  if (n == 0)
    return;
  if (n >= (1ull << 32))
    throw Error(kNotSupported, "more than 2^32 items to sort");
  const int passes = (key_bits + 7) / 8;
  const unsigned nb = (unsigned)((n + kSortTile - 1) / kSortTile);
  // one allocation: histograms, their scan scratch, ping-pong keys / values
  const size_t nh = (size_t)256 * nb, nsc = scan_scratch_elems(nh);
  const size_t off_tk = (nh + nsc + 63) / 64 * 64;  // 256-byte aligned
  const size_t off_tv = off_tk + (n + 63) / 64 * 64;
  DeviceBuffer work((off_tv + n) * sizeof(uint32_t));
  uint32_t *hist = work.as<uint32_t>(), *scratch = hist + nh;
  uint32_t *tk = hist + off_tk, *tv = hist + off_tv;
  // ping-pong so that the last pass lands in *_out
  const uint32_t *ki = keys_in, *vi = vals_in;
  for (int p = 0; p < passes; ++p)
  {
    const bool to_out = ((passes - 1 - p) % 2) == 0;
    uint32_t *ko = to_out ? keys_out : tk;
    uint32_t *vo = to_out ? vals_out : tv;
    k_radix_hist<<<nb, kSortThreads, 0, s>>>(ki, n, 8 * p, hist);
    GN_LAUNCH_CHECK("radix hist");
    scan_exclusive(hist, hist, nh, s, scratch);
    k_radix_scatter<<<nb, kSortThreads, 0, s>>>(ki, vi, ko, vo, n, 8 * p,
                                                hist);
    GN_LAUNCH_CHECK("radix scatter");
    ki = ko;
    vi = vo;
  }
  GN_CUDA(cudaStreamSynchronize(s));  // `work` is released on return
}

void histogram_offsets(const uint32_t *keys, size_t n, uint32_t bins,
                       uint32_t *offsets, cudaStream_t s)
{
  GN_CUDA(cudaMemsetAsync(offsets, 0, (size_t)(bins + 1) * sizeof(uint32_t),
                          s));
  if (n)
  {
    k_count_keys<<<grid_for(n, 256, 4096), 256, 0, s>>>(keys, n, offsets);
    GN_LAUNCH_CHECK("count keys");
  }
  scan_exclusive(offsets, offsets, (size_t)bins + 1, s);
}

void assign_sectors(const float *traj, uint32_t M, const Geo &g,
                    uint32_t *sector, cudaStream_t s)
{
  if (!M)
    return;
  k_assign<<<grid_for(M, 256, 8192), 256, 0, s>>>(traj, M, g, sector);
  GN_LAUNCH_CHECK("assign sectors");
}

void gather_sorted(const float *traj, const float *dens, const uint32_t *idx,
                   uint32_t M, int dim, float *traj_sorted, float *dens_sorted,
                   cudaStream_t s)
{
  if (!M)
    return;
  k_gather<<<grid_for(M, 256, 8192), 256, 0, s>>>(traj, dens, idx, M, dim,
                                                  traj_sorted, dens_sorted);
  GN_LAUNCH_CHECK("gather sorted");
}

size_t build_interp_matrix(const float *traj_sorted,
                           const uint32_t *sector_sorted, uint32_t M,
                           const Geo &g, const float *lut,
                           DeviceBuffer &row_off, DeviceBuffer &nz,
                           cudaStream_t s)
{
  const uint32_t G = (uint32_t)g.grid_count;
  row_off.reset((size_t)(G + 1) * sizeof(uint32_t));
  if (M == 0)
  {
    GN_CUDA(cudaMemsetAsync(row_off.get(), 0, (size_t)(G + 1) * 4, s));
    nz.reset(sizeof(uint2));
    return 0;
  }
  const size_t nsc = scan_scratch_elems((size_t)M + 1);
  DeviceBuffer count(((size_t)M + 1 + nsc) * sizeof(uint32_t));
  GN_CUDA(cudaMemsetAsync(count.get(), 0, (size_t)(M + 1) * 4, s));
  const unsigned nb = grid_for(M, 256, 8192);
  k_interp_pairs<false><<<nb, 256, 0, s>>>(traj_sorted, sector_sorted, M, g,
                                           lut, count.as<uint32_t>(), nullptr,
                                           nullptr, nullptr, nullptr);
  GN_LAUNCH_CHECK("interp count");
  scan_exclusive(count.as<uint32_t>(), count.as<uint32_t>(), (size_t)M + 1,
                 s, count.as<uint32_t>() + M + 1);
  uint32_t total = 0;
  GN_CUDA(cudaMemcpyAsync(&total, count.as<uint32_t>() + M, sizeof(uint32_t),
                          cudaMemcpyDeviceToHost, s));
  GN_CUDA(cudaStreamSynchronize(s));
  const size_t n = total;
  DeviceBuffer keys(n * 4 + 4), ids(n * 4 + 4), pairs(n * 8 + 8);
  k_interp_pairs<true><<<nb, 256, 0, s>>>(
      traj_sorted, sector_sorted, M, g, lut, nullptr, count.as<uint32_t>(),
      keys.as<uint32_t>(), ids.as<uint32_t>(), pairs.as<uint2>());
  GN_LAUNCH_CHECK("interp fill");
  count.release();
  DeviceBuffer skeys(n * 4 + 4), sids(n * 4 + 4);
  sort_pairs(keys.as<uint32_t>(), ids.as<uint32_t>(), skeys.as<uint32_t>(),
             sids.as<uint32_t>(), n, bits_for(G ? G - 1 : 0), s);
  keys.release();
  ids.release();
  nz.reset(n * 8 + 8);
  k_gather_pairs<<<grid_for(n, 256, 8192), 256, 0, s>>>(
      sids.as<uint32_t>(), pairs.as<uint2>(), n, nz.as<uint2>());
  GN_LAUNCH_CHECK("interp gather");
  histogram_offsets(skeys.as<uint32_t>(), n, G, row_off.as<uint32_t>(), s);
  GN_CUDA(cudaStreamSynchronize(s));
  return n;
}


namespace
{
// Range of z (grid cells with at least one interpolation weight) per (y, x)
// column, widened by one cell each way; empty columns keep lo > hi.
__global__ void k_col_ranges(const uint32_t *__restrict__ row_off, int G0,
                             int G1, int G2, uint2 *__restrict__ range)
{
  const long long n = (long long)G0 * G1 * G2;
  for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n;
       c += (long long)gridDim.x * blockDim.x)
  {
    if (row_off[c + 1] == row_off[c])
      continue;
    const long long col = c % ((long long)G0 * G1);
    const int z = (int)(c / ((long long)G0 * G1));
    atomicMin(&range[col].x, (unsigned)max(z - 1, 0));
    atomicMax(&range[col].y, (unsigned)min(z + 1, G2 - 1));
  }
}
}  // namespace

void build_column_ranges(const uint32_t *row_off, const Geo &g,
                         DeviceBuffer &range, DeviceBuffer &tiles,
                         int &n_tiles, cudaStream_t s)
{
  const size_t cols = (size_t)g.G[0] * g.G[1];
  range.reset(cols * sizeof(uint2));
  std::vector<uint2> h(cols, make_uint2(0xFFFFFFFFu, 0u));
  GN_CUDA(cudaMemcpyAsync(range.get(), h.data(), cols * sizeof(uint2),
                          cudaMemcpyHostToDevice, s));
  k_col_ranges<<<grid_for(g.grid_count, 256, 148 * 64), 256, 0, s>>>(
      row_off, g.G[0], g.G[1], g.G[2], range.as<uint2>());
  GN_LAUNCH_CHECK("column ranges");
  GN_CUDA(cudaMemcpyAsync(h.data(), range.get(), cols * sizeof(uint2),
                          cudaMemcpyDeviceToHost, s));
  GN_CUDA(cudaStreamSynchronize(s));
  // tiles of kColTile adjacent columns with at least one range
  std::vector<uint32_t> list;
  const size_t nt = (cols + kColTile - 1) / kColTile;
  for (size_t t = 0; t < nt; ++t)
  {
    bool any = false;
    for (size_t c = t * kColTile; c < std::min(cols, (t + 1) * kColTile); ++c)
      any = any || h[c].x <= h[c].y;
    if (any)
      list.push_back((uint32_t)t);
  }
  n_tiles = (int)list.size();
  tiles.reset(std::max<size_t>(list.size(), 1) * sizeof(uint32_t));
  if (!list.empty())
    GN_CUDA(cudaMemcpyAsync(tiles.get(), list.data(),
                            list.size() * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, s));
  GN_CUDA(cudaStreamSynchronize(s));
}

}  // namespace gnufft
