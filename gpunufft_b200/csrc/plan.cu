// Plan (one per trajectory) and the C ABI declared in include/gpunufft_b200.h.
//
// Plan creation restates the upstream factory
// (gpuNUFFT_operator_factory.cpp:450-553): sector assignment, sort by
// sector, sorted coordinates / density, sector offsets, centers, balanced
// processing order and the deapodization function -- and adds the owner
// candidate lists and work items used by this library's kernels.  All tables
// stay resident on the device, together with the sensitivity maps, the
// kernel lookup table and cached cuFFT plans.
//
// Calls restate GpuNUFFTOperator::performGpuNUFFTAdj / performForwardGpuNUFFT
// (gpuNUFFT_operator.cpp:370-1294) with all coils of a call in one pass.
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cufft.h>
#include <cuda_runtime.h>

#include "../../include/gpunufft_b200.h"
#include "binning.cuh"
#include "capi.hpp"
#include "devutil.hpp"
#include "fftpass.cuh"
#include "footprint.cuh"
#include "geometry.hpp"
#include "gridding.cuh"
#include "hostcopy.hpp"
#include "planview.hpp"
#include "tma.cuh"
#include "trajgrad.cuh"

using namespace gnufft;

namespace
{
thread_local std::string g_last_error;

// Samples per forward work item.
constexpr int kFwdPayload = kFwdItemSamples;

// Mirrors the upstream IndPair (gpuNUFFT_types.hpp:33-49): compared by the
// second member only, so libstdc++'s std::sort produces the upstream order.
struct SectorPair
{
  uint32_t first, second;
  bool operator<(const SectorPair &o) const { return second < o.second; }
  bool operator>(const SectorPair &o) const { return second > o.second; }
};

const char *kVersion = "gpunufft_b200 0.1.0 (sm_100a)";

}  // namespace

struct gnufft_plan
{
  gnufft_desc desc{};
  Geo g{};
  int dim = 2;
  uint32_t M = 0;
  cudaStream_t stream = nullptr;
  bool texture = false;
  bool plain = false;
  int fwd_tile_coils = 0;  // 0: automatic
  bool pruned = false;     // separable pruned transforms instead of cuFFT
  // cuFFT grids even along every axis: the forward folds its shift into the
  // prepare pass as signs and reads sector tiles by tensor copies
  bool fwd_signs = false;
  int *copy_err_h = nullptr;  // set by a tile copy that timed out (mapped)
  int *copy_err_d = nullptr;
  long long copy_polls = tma::kMbarSpin;  // first wait of a tile copy
  size_t mem_limit = 0;  // scratch cap of a call (0: the free memory)
  // TEXTURE operators: the lookup table as a filtered texture
  cudaArray_t lut_array = nullptr;
  cudaTextureObject_t lut_tex = 0;

  // host copies of the exported tables
  std::vector<float> lut_h, deapo_h;
  std::vector<uint32_t> sdc_h, centers_h, order_h;
  bool has_dens = false;

  // resident device tables
  DeviceBuffer lut, traj_sorted, di, sec_sorted, dens_sorted;
  DeviceBuffer fwd_items, fwd_order, deapo, sens;
  DeviceBuffer di_inv;  // sorted position of every original sample
  DeviceBuffer w_rows, w_nz;  // interpolation matrix, CSR by grid cell
  DeviceBuffer dlut;          // kernel derivative table (trajectory gradient)
  DeviceBuffer roots[3];      // DFT roots per axis (pruned transforms)
  DeviceBuffer zrange;        // per (y, x) column: z rows with weights
  DeviceBuffer ztiles;        // column tiles holding a z range
  int n_ztiles = 0;
  float dlut_mult = 0.f;
  size_t nnz = 0;
  int n_fwd_items = 0;
  uint32_t sens_coils = 0;
  std::vector<float2> sens_h;

  // per-call scratch (grow-only)
  DeviceBuffer ks, grid, stage_in, stage_out, one_sens, fft_a, fft_b;
  std::map<int, cufftHandle> fft;

  // timing
  bool timing = false;
  cudaEvent_t ev[8] = {};  // start / end of prepare, gridding, fft, finish
  gnufft_stage_times times{};
  uint32_t launches = 0;

  ~gnufft_plan()
  {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(desc.device);
    if (stream)
      cudaStreamSynchronize(stream);
    for (auto &kv : fft)
      cufftDestroy(kv.second);
    for (auto &e : ev)
      if (e)
        cudaEventDestroy(e);
    if (stream)
      cudaStreamDestroy(stream);
    if (copy_err_h)
      cudaFreeHost(copy_err_h);
    if (lut_tex)
      cudaDestroyTextureObject(lut_tex);
    if (lut_array)
      cudaFreeArray(lut_array);
    if (prev >= 0)
      cudaSetDevice(prev);
  }

  size_t device_bytes() const
  {
    const DeviceBuffer *bufs[] = {&lut,         &traj_sorted, &di,
                                  &sec_sorted,  &dens_sorted,
                                  &fwd_items,   &fwd_order,   &deapo,
                                  &sens,
                                  &di_inv,
                                  &w_rows,      &w_nz,
                                  &ks,          &grid,        &stage_in,
                                  &stage_out,   &one_sens,    &fft_a,
                                  &fft_b,       &dlut,        &roots[0],
                                  &roots[1],    &roots[2],    &zrange,
                                  &ztiles};
    size_t s = 0;
    for (auto *b : bufs)
      s += b->bytes();
    return s;
  }

  cufftHandle fft_plan(int batch)
  {
    auto it = fft.find(batch);
    if (it != fft.end())
      return it->second;
    cufftHandle h;
    int n[3];
    if (dim == 3)
    {
      n[0] = g.G[2];
      n[1] = g.G[1];
      n[2] = g.G[0];
    }
    else
    {
      n[0] = g.G[1];
      n[1] = g.G[0];
    }
    check_cufft(cufftPlanMany(&h, dim, n, nullptr, 1, (int)g.grid_count,
                              nullptr, 1, (int)g.grid_count, CUFFT_C2C, batch),
                "cufftPlanMany");
    fft[batch] = h;
    return h;
  }

  void mark(int i, cudaStream_t s)
  {
    if (timing)
      GN_CUDA(cudaEventRecord(ev[i], s));
  }
};

namespace
{
template <class T> void upload(DeviceBuffer &b, const T *h, size_t n,
                               cudaStream_t s)
{
  b.reset(std::max<size_t>(n, 1) * sizeof(T));
  if (n)
    GN_CUDA(cudaMemcpyAsync(b.get(), h, n * sizeof(T), cudaMemcpyHostToDevice,
                            s));
}

template <class T> void download(std::vector<T> &h, const DeviceBuffer &b,
                                 size_t n, cudaStream_t s)
{
  h.resize(n);
  if (n)
    GN_CUDA(cudaMemcpyAsync(h.data(), b.get(), n * sizeof(T),
                            cudaMemcpyDeviceToHost, s));
}

void validate_desc(const gnufft_desc *d)
{
  if (!d)
    throw Error(kInvalidArgument, "descriptor is NULL");
  if (d->operator_type < 0 || d->operator_type > 3)
    throw Error(kInvalidArgument, "unknown operator type");
  if (d->n_samples == 0)
    throw Error(kInvalidArgument, "trajectory has no samples");
}

// computeProcessingOrder (gpuNUFFT_operator_factory.cpp:74-126): sectors by
// count descending (same libstdc++ std::sort on the same input, so the same
// order), split into MAXIMUM_PAYLOAD chunks.
void processing_order(const std::vector<uint32_t> &sdc,
                      std::vector<uint32_t> &order)
{
  std::vector<SectorPair> cps;
  for (size_t i = 0; i + 1 < sdc.size(); i++)
    cps.push_back(SectorPair{(uint32_t)i, sdc[i + 1] - sdc[i]});
  std::sort(cps.begin(), cps.end(), std::greater<SectorPair>());
  order.clear();
  for (auto &p : cps)
  {
    if (p.second == 0)
      break;
    order.push_back(p.first);
    order.push_back(0);
    int remaining = (int)p.second;
    uint32_t off = 1;
    while (remaining - (int)kUpstreamPayload > 0)
    {
      remaining -= kUpstreamPayload;
      order.push_back(p.first);
      order.push_back((off++) * kUpstreamPayload);
    }
  }
}

// computeSectorCenters / 2D (gpuNUFFT_operator_factory.cpp:207-270)
void sector_centers(const Geo &g, std::vector<uint32_t> &c)
{
  c.clear();
  const uint32_t half = (uint32_t)(g.sw >> 1);
  for (int z = 0; z < (g.dim == 3 ? g.S[2] : 1); ++z)
    for (int y = 0; y < g.S[1]; ++y)
      for (int x = 0; x < g.S[0]; ++x)
      {
        c.push_back((uint32_t)x * g.sw + half);
        c.push_back((uint32_t)y * g.sw + half);
        if (g.dim == 3)
          c.push_back((uint32_t)z * g.sw + half);
      }
}

void build_items(gnufft_plan &p)
{
  const int S = p.g.n_sectors;
  std::vector<FwdItem> fitems;
  for (int s = 0; s < S; ++s)
  {
    const uint32_t b = p.sdc_h[s], e = p.sdc_h[s + 1];
    for (uint32_t k = b; k < e; k += kFwdPayload)
      fitems.push_back(
          FwdItem{s, (int)k, (int)std::min<uint32_t>(e, k + kFwdPayload), 0});
  }
  // sector order: consecutive blocks take neighbouring tiles, whose halos
  // overlap, so much of a tile comes from L2
  p.n_fwd_items = (int)fitems.size();
  upload(p.fwd_items, fitems.data(), fitems.size(), p.stream);
}

// The TEXTURE operators read their kernel table through the texture unit:
// a 1-D array with normalised coordinates, linear filtering and clamp
// addressing, the sampler state the upstream gives its 2-D table
// (std_gpuNUFFT_kernels.cu:49-60; that table is the outer product of the 1-D
// one, so per-axis fetches give the same filtered weights).
void make_lut_texture(gnufft_plan &p)
{
  const cudaChannelFormatDesc fd = cudaCreateChannelDesc<float>();
  GN_CUDA(cudaMallocArray(&p.lut_array, &fd, (size_t)p.g.lut_len, 0));
  GN_CUDA(cudaMemcpy2DToArrayAsync(
      p.lut_array, 0, 0, p.lut_h.data(), p.lut_h.size() * sizeof(float),
      p.lut_h.size() * sizeof(float), 1, cudaMemcpyHostToDevice, p.stream));
  cudaResourceDesc rd;
  std::memset(&rd, 0, sizeof(rd));
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = p.lut_array;
  cudaTextureDesc td;
  std::memset(&td, 0, sizeof(td));
  td.addressMode[0] = cudaAddressModeClamp;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 1;
  GN_CUDA(cudaCreateTextureObject(&p.lut_tex, &rd, &td, nullptr));
  GN_CUDA(cudaStreamSynchronize(p.stream));
  p.g.lut_tex = (unsigned long long)p.lut_tex;
}

void init_common(gnufft_plan &p, const gnufft_desc *d)
{
  validate_desc(d);
  p.desc = *d;
  p.texture = d->operator_type == GNUFFT_TEXTURE ||
              d->operator_type == GNUFFT_BALANCED_TEXTURE;
  p.plain = (d->flags & GNUFFT_FLAG_PLAIN) != 0;
  {
    const uint32_t code = (d->flags & GNUFFT_FLAG_FWD_TILE_MASK) >> 8;
    if (code > 6)
      throw Error(kInvalidArgument, "forward tile coil count out of range");
    p.fwd_tile_coils = code ? 1 << (code - 1) : 0;
  }
  std::string err;
  if (!make_geo(d->img_dims, d->osf, d->kernel_width, d->sector_width,
                p.texture, p.g, err))
    throw Error(kInvalidArgument, err);
  if (!gridding_supported(p.g, err))
    throw Error(kNotSupported, err);
  p.pruned = !p.plain && !(d->flags & GNUFFT_FLAG_CUFFT) &&
             pruned_fft_supported(p.g);
  p.fwd_signs = !p.pruned && !p.plain;
  for (int a = 0; a < p.g.dim; ++a)
    p.fwd_signs = p.fwd_signs && p.g.G[a] % 2 == 0;
  if (p.pruned || p.fwd_signs)
  {
    GN_CUDA(cudaHostAlloc(reinterpret_cast<void **>(&p.copy_err_h),
                          sizeof(int), cudaHostAllocMapped));
    *p.copy_err_h = 0;
    GN_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void **>(&p.copy_err_d),
                                     p.copy_err_h, 0));
  }
  p.dim = p.g.dim;
  p.M = d->n_samples;
  if ((size_t)p.M * (p.dim + 2) >= (1ull << 31))
    throw Error(kNotSupported, "too many samples");
  GN_CUDA(cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking));
  p.lut_h.resize(p.g.lut_len);
  kernel_lut_fill(p.lut_h.data(), p.g.lut_len, (int)d->kernel_width, d->osf);
  upload(p.lut, p.lut_h.data(), p.lut_h.size(), p.stream);
  if (p.texture)
    make_lut_texture(p);
  compute_deapo(p.g, p.lut_h.data(), p.deapo_h);
  sector_centers(p.g, p.centers_h);
}

void set_sens_host(gnufft_plan &p, const void *sens, uint32_t n_coils)
{
  if (!sens || n_coils == 0)
  {
    p.sens_coils = 0;
    p.sens_h.clear();
    p.sens.release();
    return;
  }
  const size_t n = (size_t)n_coils * p.g.img_count;
  const float2 *s = static_cast<const float2 *>(sens);
  // only the plain flow (maps copied per coil per call, like the upstream)
  // needs a host copy; the other plans copy from the caller's buffer (the
  // callers synchronise the plan's stream before they return)
  if (p.plain)
    p.sens_h.assign(s, s + n);
  else
    p.sens_h.clear();
  // keep the device buffer when it is large enough (no free / malloc, which
  // would synchronise the device, when maps are swapped between requests)
  p.sens.ensure(n * sizeof(float2));
  copy_host_to_device(p.sens.get(), p.plain ? p.sens_h.data() : s,
                      n * sizeof(float2), p.stream);
  p.sens_coils = n_coils;
}

void finish_tables(gnufft_plan &p)
{
  // interpolation matrix (adjoint) and forward work items
  p.nnz = build_interp_matrix(p.traj_sorted.as<float>(),
                              p.sec_sorted.as<uint32_t>(), p.M, p.g,
                              p.lut.as<float>(), p.w_rows, p.w_nz, p.stream);
  build_items(p);
  if (p.dim == 3 && forward_pairs(p.g, 0))
  {
    p.fwd_order.reset((size_t)p.M * sizeof(uint32_t));
    build_forward_lane_order(p.fwd_items.as<FwdItem>(), p.n_fwd_items,
                             p.traj_sorted.as<float>(), p.M, p.g,
                             p.lut.as<float>(), p.fwd_order.as<uint32_t>(),
                             p.stream);
  }
  p.di_inv.reset((size_t)p.M * sizeof(uint32_t) + 4);
  launch_invert_permutation(p.di.as<uint32_t>(), p.M, p.di_inv.as<uint32_t>(),
                            p.stream);
  if (p.pruned && p.dim == 3)
    build_column_ranges(p.w_rows.as<uint32_t>(), p.g, p.zrange, p.ztiles,
                        p.n_ztiles, p.stream);
  processing_order(p.sdc_h, p.order_h);
  upload(p.deapo, p.deapo_h.data(), p.deapo_h.size(), p.stream);
  GN_CUDA(cudaStreamSynchronize(p.stream));
}

void create_plan(gnufft_plan &p, const gnufft_desc *d, const float *traj,
                 const float *dens, const void *sens)
{
  if (!traj)
    throw Error(kInvalidArgument, "trajectory is NULL");
  init_common(p, d);
  const uint32_t M = p.M;
  const int dim = p.dim;
  cudaStream_t s = p.stream;

  DeviceBuffer traj_d, dens_d, sec, iota;
  upload(traj_d, traj, (size_t)dim * M, s);
  if (dens)
  {
    upload(dens_d, dens, M, s);
    p.has_dens = true;
  }
  sec.reset((size_t)M * sizeof(uint32_t));
  assign_sectors(traj_d.as<float>(), M, p.g, sec.as<uint32_t>(), s);

  p.di.reset((size_t)M * sizeof(uint32_t));
  p.sec_sorted.reset((size_t)M * sizeof(uint32_t));
  if (d->flags & GNUFFT_FLAG_REFERENCE_ORDER)
  {
    // the upstream's own order: std::sort of (index, sector) pairs
    // (sortVector, gpuNUFFT_operator_factory.cpp:56-72)
    std::vector<uint32_t> sec_h;
    download(sec_h, sec, M, s);
    GN_CUDA(cudaStreamSynchronize(s));
    std::vector<SectorPair> v(M);
    for (uint32_t i = 0; i < M; ++i)
      v[i] = SectorPair{i, sec_h[i]};
    std::sort(v.begin(), v.end());
    std::vector<uint32_t> di_h(M), ss_h(M);
    for (uint32_t i = 0; i < M; ++i)
    {
      di_h[i] = v[i].first;
      ss_h[i] = v[i].second;
    }
    GN_CUDA(cudaMemcpyAsync(p.di.get(), di_h.data(), M * sizeof(uint32_t),
                            cudaMemcpyHostToDevice, s));
    GN_CUDA(cudaMemcpyAsync(p.sec_sorted.get(), ss_h.data(),
                            M * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    GN_CUDA(cudaStreamSynchronize(s));
  }
  else
  {
    std::vector<uint32_t> io(M);
    for (uint32_t i = 0; i < M; ++i)
      io[i] = i;
    upload(iota, io.data(), M, s);
    int bits = 1;
    while (bits < 32 && ((uint32_t)(p.g.n_sectors - 1) >> bits))
      ++bits;
    sort_pairs(sec.as<uint32_t>(), iota.as<uint32_t>(),
               p.sec_sorted.as<uint32_t>(), p.di.as<uint32_t>(), M, bits, s);
  }
  p.traj_sorted.reset((size_t)dim * M * sizeof(float));
  if (dens)
    p.dens_sorted.reset((size_t)M * sizeof(float));
  gather_sorted(traj_d.as<float>(), dens ? dens_d.as<float>() : nullptr,
                p.di.as<uint32_t>(), M, dim, p.traj_sorted.as<float>(),
                dens ? p.dens_sorted.as<float>() : nullptr, s);
  DeviceBuffer sdc((size_t)(p.g.n_sectors + 1) * sizeof(uint32_t));
  histogram_offsets(p.sec_sorted.as<uint32_t>(), M, (uint32_t)p.g.n_sectors,
                    sdc.as<uint32_t>(), s);
  download(p.sdc_h, sdc, (size_t)p.g.n_sectors + 1, s);
  GN_CUDA(cudaStreamSynchronize(s));
  set_sens_host(p, sens, sens ? d->n_coils : 0);
  finish_tables(p);
}

void load_plan(gnufft_plan &p, const gnufft_desc *d, const float *traj_sorted,
               const uint32_t *di, const uint32_t *sdc,
               const uint32_t *order, uint32_t n_order,
               const uint32_t *centers, const float *dens_sorted,
               const void *sens, const float *deapo)
{
  if (!traj_sorted || !di || !sdc || !centers || !deapo)
    throw Error(kInvalidArgument, "precomputed table is NULL");
  init_common(p, d);
  const uint32_t M = p.M, S = (uint32_t)p.g.n_sectors;
  const int dim = p.dim;
  // validate the tables against the geometry
  if (sdc[0] != 0 || sdc[S] != M)
    throw Error(kInvalidArgument, "sector data count does not span samples");
  for (uint32_t i = 0; i < S; ++i)
    if (sdc[i + 1] < sdc[i])
      throw Error(kInvalidArgument, "sector data count not monotone");
  std::vector<uint8_t> seen(M, 0);
  for (uint32_t i = 0; i < M; ++i)
  {
    if (di[i] >= M || seen[di[i]])
      throw Error(kInvalidArgument, "data indices are not a permutation");
    seen[di[i]] = 1;
  }
  std::vector<uint32_t> my_centers;
  sector_centers(p.g, my_centers);
  if (!std::equal(my_centers.begin(), my_centers.end(), centers))
    throw Error(kInvalidArgument, "sector centers do not match the geometry");
  // every sorted sample must lie in the sector whose range holds it (the
  // kernels place a sample's footprint inside its own sector's tile)
  std::vector<uint32_t> ss(M);
  for (uint32_t sct = 0; sct < S; ++sct)
    for (uint32_t t = sdc[sct]; t < sdc[sct + 1]; ++t)
    {
      uint32_t id = 0, stride = 1;
      for (int a = 0; a < dim; ++a)
      {
        const float c = traj_sorted[(size_t)a * M + t];
        if (!std::isfinite(c))
          throw Error(kInvalidArgument, "trajectory coordinate not finite");
        id += host_sector_of(c, p.g.G[a], p.g.sw) * stride;
        stride *= (uint32_t)p.g.S[a];
      }
      if (id != sct)
        throw Error(kInvalidArgument,
                    "sorted sample " + std::to_string(t) +
                        " does not lie in sector " + std::to_string(sct));
      ss[t] = sct;
    }
  p.sdc_h.assign(sdc, sdc + S + 1);
  p.deapo_h.assign(deapo, deapo + p.g.img_count);
  cudaStream_t s = p.stream;
  upload(p.di, di, M, s);
  upload(p.sec_sorted, ss.data(), M, s);
  upload(p.traj_sorted, traj_sorted, (size_t)dim * M, s);
  if (dens_sorted)
  {
    p.has_dens = true;
    upload(p.dens_sorted, dens_sorted, M, s);
  }
  set_sens_host(p, sens, sens ? d->n_coils : 0);
  finish_tables(p);
  if (order && n_order)
    p.order_h.assign(order, order + 2 * (size_t)n_order);
}

// ------------------------------------------------------------------------
// per-call execution
// ------------------------------------------------------------------------
void check_coils(const gnufft_plan &p, uint32_t C)
{
  if (C == 0)
    throw Error(kInvalidArgument, "n_coils must be positive");
  if (p.sens_coils && C != p.sens_coils)
    throw Error(kInvalidArgument,
                "n_coils differs from the sensitivity map channels");
}

// The error flag and first-wait bound of the plan's tile copies.
tma::CopyWait copy_wait(const gnufft_plan &p)
{
  tma::CopyWait cw;
  cw.err = p.copy_err_d;
  cw.polls = p.copy_polls;
  return cw;
}

// Root tables (once) and grow-only scratch of the pruned transforms.
// A tile copy that did not complete within its bounded wait set the mapped
// flag: report it (once).  Checked at the start of every call (copies of an
// earlier device call) and at the end of the synchronous host calls (their
// own copies).
void check_copy_err(gnufft_plan &p)
{
  if (p.copy_err_h && *(volatile int *)p.copy_err_h)
  {
    *p.copy_err_h = 0;
    throw Error(kCudaError, "a tile copy did not complete within its wait");
  }
}

void ensure_pruned(gnufft_plan &p, uint32_t C, cudaStream_t s)
{
  for (int a = 0; a < p.g.dim; ++a)
    if (!p.roots[a].get())
    {
      std::vector<float2> tab;
      fft_roots(p.g.G[a], tab);
      p.roots[a].reset(tab.size() * sizeof(float2));
      GN_CUDA(cudaMemcpyAsync(p.roots[a].get(), tab.data(),
                              tab.size() * sizeof(float2),
                              cudaMemcpyHostToDevice, s));
      GN_CUDA(cudaStreamSynchronize(s));
    }
  p.fft_a.ensure(pruned_scratch_a(p.g, (int)C) * sizeof(float2));
  p.fft_b.ensure(std::max(pruned_scratch_b(p.g, (int)C),
                          pruned_scratch_xfirst(p.g, (int)C)) *
                 sizeof(float2));
}

std::array<const float2 *, 3> root_ptrs(const gnufft_plan &p)
{
  return {p.roots[0].as<float2>(), p.roots[1].as<float2>(),
          p.roots[2].as<float2>()};
}

// All coils of the call in one pass.
void adjoint_batched(gnufft_plan &p, const float2 *k, float2 *img, uint32_t C,
                     int stage, cudaStream_t s, const float2 *sens,
                     bool accumulate = false)
{
  const Geo &g = p.g;
  const int cg = spmm_coil_group((int)C);
  const int CP = ((int)C + cg - 1) / cg * cg;
  if ((size_t)p.M * CP > 0xFFFFFFFFull)  // 32-bit row offsets in the spread
    throw Error(kNotSupported, "samples x coil lanes exceed 2^32");
  p.ks.ensure((size_t)p.M * CP * sizeof(float2));
  const bool conv = stage == GNUFFT_CONVOLUTION ||
                    stage == GNUFFT_DENSITY_ESTIMATION;
  float2 *grid = img;
  if (!conv)
  {
    p.grid.ensure((size_t)C * g.grid_count * sizeof(float2));
    grid = p.grid.as<float2>();
  }
  p.mark(0, s);
  launch_gather_kspace_inv(k, p.di_inv.as<uint32_t>(),
                           p.has_dens ? p.dens_sorted.as<float>() : nullptr,
                           p.M, (int)C, CP, p.ks.as<float2>(), s);
  p.launches += 1;
  p.mark(1, s);
  p.mark(2, s);
  if (p.pruned && !conv)
  {  // spread whole grid rows with the inverse x transform fused (the grid
     // buffer receives only the cropped x outputs), then y and z
    check_copy_err(p);
    ensure_pruned(p, C, s);
    if (launch_adjoint_spmm_xfft(p.w_rows.as<uint32_t>(), p.w_nz.as<uint2>(),
                                 p.ks.as<float2>(), CP, g, (int)C,
                                 p.roots[0].as<float2>(), grid, s))
    {
      p.launches += 1;
      p.mark(3, s);
      p.mark(4, s);
      launch_pruned_adjoint_xfirst(
          grid, p.deapo.as<float>(),
          stage == GNUFFT_DEAPODIZATION ? sens : nullptr, g, (int)C,
          stage == GNUFFT_FFT ? 1 : 2, accumulate, root_ptrs(p).data(),
          p.fft_b.as<float2>(), p.fft_a.as<float2>(), img, s, copy_wait(p));
      p.launches += g.dim - 1;
      p.mark(5, s);
      p.mark(6, s);
      p.mark(7, s);
      return;
    }
  }
  launch_adjoint_spmm(p.w_rows.as<uint32_t>(), p.w_nz.as<uint2>(),
                      p.ks.as<float2>(), CP, g, (int)C, !conv, grid, s);
  p.launches += 1;
  p.mark(3, s);
  p.mark(4, s);
  if (conv)
  {
    p.mark(5, s);
    p.mark(6, s);
    p.mark(7, s);
    return;
  }
  if (p.pruned)
  {  // inverse transform, crop, scale, deapodization and coil sum fused
    ensure_pruned(p, C, s);
    launch_pruned_adjoint(grid, p.deapo.as<float>(),
                          stage == GNUFFT_DEAPODIZATION ? sens : nullptr, g,
                          (int)C, stage == GNUFFT_FFT ? 1 : 2, accumulate,
                          root_ptrs(p).data(), p.fft_a.as<float2>(),
                          p.fft_b.as<float2>(), img, s);
    p.launches += g.dim + 1;
    p.mark(5, s);
    p.mark(6, s);
    p.mark(7, s);
    return;
  }
  cufftHandle h = p.fft_plan((int)C);
  check_cufft(cufftSetStream(h, s), "cufftSetStream");
  check_cufft(cufftExecC2C(h, (cufftComplex *)grid, (cufftComplex *)grid,
                           CUFFT_INVERSE),
              "cufftExecC2C inverse");
  p.mark(5, s);
  p.mark(6, s);
  launch_adjoint_finish(grid, p.deapo.as<float>(),
                        stage == GNUFFT_DEAPODIZATION ? sens : nullptr, g,
                        (int)C, stage == GNUFFT_FFT ? 1 : 2, accumulate, img,
                        s);
  p.launches += 1;
  p.mark(7, s);
}

void forward_batched(gnufft_plan &p, const float2 *img, float2 *k, uint32_t C,
                     int stage, cudaStream_t s, const float2 *sens)
{
  const Geo &g = p.g;
  if (stage == GNUFFT_DENSITY_ESTIMATION)
  {
    for (int a = 0; a < g.dim; ++a)
      if (g.N[a] != g.G[a])
        throw Error(kNotSupported,
                    "DENSITY_ESTIMATION forward needs grid == image (osf 1)");
  }
  const bool dens_est = stage == GNUFFT_DENSITY_ESTIMATION;
  // 3-D pruned path: the grid holds coil pairs interleaved
  const bool paired = p.pruned && !dens_est && p.copy_err_d &&
                      forward_pairs(g, p.fwd_tile_coils);
  p.grid.ensure((size_t)(paired ? (C + 1) / 2 * 2 : C) * g.grid_count *
                sizeof(float2));
  float2 *grid = p.grid.as<float2>();
  if (p.pruned && !dens_est)
  {  // sens, deapodization, pad, shift and the transform in g.dim passes
    check_copy_err(p);
    ensure_pruned(p, C, s);
    p.mark(0, s);
    p.mark(1, s);
    p.mark(4, s);
    launch_pruned_forward(img, sens, p.deapo.as<float>(), g, (int)C,
                          root_ptrs(p).data(), p.fft_a.as<float2>(),
                          p.fft_b.as<float2>(), grid, s,
                          p.zrange.as<uint2>(), copy_wait(p), paired,
                          p.ztiles.as<uint32_t>(), p.n_ztiles, kColTile);
    p.launches += g.dim;
    p.mark(5, s);
    p.mark(2, s);
    // the grid holds the shifted spectrum: sector tiles are boxes of it
    if (!launch_forward_interp_tma(
            p.fwd_items.as<FwdItem>(), p.n_fwd_items,
            p.traj_sorted.as<float>(), p.di.as<uint32_t>(),
            p.has_dens ? p.dens_sorted.as<float>() : nullptr, grid, g,
            p.lut.as<float>(), p.M, (int)C, g.fft_scale, k, copy_wait(p), s,
            p.fwd_tile_coils, paired, p.fwd_order.as<uint32_t>()))
      launch_forward_interp(
          p.fwd_items.as<FwdItem>(), p.n_fwd_items, p.traj_sorted.as<float>(),
          p.di.as<uint32_t>(),
          p.has_dens ? p.dens_sorted.as<float>() : nullptr, grid, g,
          p.lut.as<float>(), p.M, (int)C, false, g.fft_scale, k, s,
          p.fwd_tile_coils);
    p.launches += 1;
    p.mark(3, s);
    p.mark(6, s);
    p.mark(7, s);
    return;
  }
  const bool signs = p.fwd_signs && !dens_est;
  if (signs)
    check_copy_err(p);
  p.mark(0, s);
  launch_forward_prepare(img, sens, p.deapo.as<float>(), g, (int)C, dens_est,
                         grid, s, signs);
  p.launches += 1;
  p.mark(1, s);
  p.mark(4, s);
  if (!dens_est)
  {
    cufftHandle h = p.fft_plan((int)C);
    check_cufft(cufftSetStream(h, s), "cufftSetStream");
    check_cufft(cufftExecC2C(h, (cufftComplex *)grid, (cufftComplex *)grid,
                             CUFFT_FORWARD),
                "cufftExecC2C forward");
  }
  p.mark(5, s);
  p.mark(2, s);
  // the signed grid holds the FORWARD-shifted spectrum: tiles are boxes
  if (!signs ||
      !launch_forward_interp_tma(
          p.fwd_items.as<FwdItem>(), p.n_fwd_items, p.traj_sorted.as<float>(),
          p.di.as<uint32_t>(),
          p.has_dens ? p.dens_sorted.as<float>() : nullptr, grid, g,
          p.lut.as<float>(), p.M, (int)C, g.fft_scale, k, copy_wait(p), s,
          p.fwd_tile_coils, false))
    launch_forward_interp(
        p.fwd_items.as<FwdItem>(), p.n_fwd_items, p.traj_sorted.as<float>(),
        p.di.as<uint32_t>(),
        (p.has_dens && !dens_est) ? p.dens_sorted.as<float>() : nullptr, grid,
        g, p.lut.as<float>(), p.M, (int)C, !dens_est && !signs,
        dens_est ? 1.0f : g.fft_scale, k, s, p.fwd_tile_coils);
  p.launches += 1;
  p.mark(3, s);
  p.mark(6, s);
  p.mark(7, s);
}

// Trajectory gradient: the forward's prepare + FFT, then the derivative
// interpolation against the k-space weights u [C][M].
void traj_grad(gnufft_plan &p, const float2 *img, const float2 *u, uint32_t C,
               float *out, cudaStream_t s, const float2 *sens)
{
  const Geo &g = p.g;
  if (!p.dlut.get())
  {
    std::vector<float> tab;
    deriv_lut_fill(g, p.desc.osf, kDerivLutLen, tab, p.dlut_mult);
    upload(p.dlut, tab.data(), tab.size(), s);
  }
  p.grid.ensure((size_t)C * g.grid_count * sizeof(float2));
  float2 *grid = p.grid.as<float2>();
  launch_forward_prepare(img, sens, p.deapo.as<float>(), g, (int)C, false,
                         grid, s);
  cufftHandle h = p.fft_plan((int)C);
  check_cufft(cufftSetStream(h, s), "cufftSetStream");
  check_cufft(cufftExecC2C(h, (cufftComplex *)grid, (cufftComplex *)grid,
                           CUFFT_FORWARD),
              "cufftExecC2C forward");
  launch_traj_grad(p.traj_sorted.as<float>(), p.sec_sorted.as<uint32_t>(),
                   p.di.as<uint32_t>(),
                   p.has_dens ? p.dens_sorted.as<float>() : nullptr, grid, g,
                   p.lut.as<float>(), p.dlut.as<float>(), kDerivLutLen,
                   p.dlut_mult, p.M, (int)C, g.fft_scale, u, out, s);
  p.launches += 3;
}

// Device scratch the plan's buffers grow to for calls with C coils
// (forward and adjoint share them): the sorted k-space lanes, the grid and
// the transform passes' buffers (cuFFT's work area counted as one grid).
size_t call_scratch_bytes(const gnufft_plan &p, uint32_t C)
{
  const Geo &g = p.g;
  const size_t G = (size_t)g.grid_count, f2 = sizeof(float2);
  const size_t cg = (size_t)spmm_coil_group((int)C);
  const size_t CP = (C + cg - 1) / cg * cg;
  size_t b = (size_t)p.M * CP * f2 + (size_t)(C + 1) / 2 * 2 * G * f2;
  if (p.pruned)
    b += (pruned_scratch_a(g, (int)C) +
          std::max(pruned_scratch_b(g, (int)C),
                   pruned_scratch_xfirst(g, (int)C))) *
         f2;
  else
    b += (size_t)C * G * f2;
  return b;
}

size_t held_scratch_bytes(const gnufft_plan &p)
{
  return p.ks.bytes() + p.grid.bytes() + p.fft_a.bytes() + p.fft_b.bytes();
}

// Coils per pass so that a pass's scratch fits the plan's memory limit, or
// else the device memory free now (plus what the plan's scratch holds
// already, minus a margin) -- the upstream's concurrent coil count
// (computePossibleConcurrentCoilCount, gpuNUFFT_operator.cpp:327-368),
// for 2-D and 3-D alike.  At least one coil.
uint32_t coils_per_pass(const gnufft_plan &p, uint32_t C)
{
  size_t limit = p.mem_limit;
  if (!limit)
  {
    size_t free_b = 0, total_b = 0;
    GN_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t margin = (size_t)256 << 20;
    const size_t avail = free_b + held_scratch_bytes(p);
    limit = avail > margin ? avail - margin : 0;
  }
  if (call_scratch_bytes(p, C) <= limit)
    return C;
  uint32_t lo = 1, hi = C;  // largest c with scratch(c) <= limit
  while (lo < hi)
  {
    const uint32_t mid = (lo + hi + 1) / 2;
    if (call_scratch_bytes(p, mid) <= limit)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// A batched call in coil passes of at most coils_per_pass coils: k-space,
// maps and per-coil outputs advance by the pass's first coil; the
// coil-combined image (maps, DEAPODIZATION) is summed over the passes.
void adjoint_chunked(gnufft_plan &p, const float2 *k, float2 *img,
                     uint32_t C, int stage, cudaStream_t s)
{
  const uint32_t step = coils_per_pass(p, C);
  const float2 *sens = p.sens.as<float2>();
  const bool combine = stage == GNUFFT_DEAPODIZATION && sens;
  const bool conv = stage == GNUFFT_CONVOLUTION ||
                    stage == GNUFFT_DENSITY_ESTIMATION;
  const size_t per_out = conv ? (size_t)p.g.grid_count
                              : (size_t)p.g.img_count;
  for (uint32_t c0 = 0; c0 < C; c0 += step)
  {
    const uint32_t n = std::min(step, C - c0);
    adjoint_batched(p, k + (size_t)c0 * p.M,
                    combine ? img : img + (size_t)c0 * per_out, n, stage, s,
                    sens ? sens + (size_t)c0 * p.g.img_count : nullptr,
                    combine && c0 > 0);
  }
}

void forward_chunked(gnufft_plan &p, const float2 *img, float2 *k,
                     uint32_t C, int stage, cudaStream_t s)
{
  const uint32_t step = coils_per_pass(p, C);
  const float2 *sens = p.sens.as<float2>();
  const size_t N = (size_t)p.g.img_count;
  for (uint32_t c0 = 0; c0 < C; c0 += step)
  {
    const uint32_t n = std::min(step, C - c0);
    forward_batched(p, sens ? img : img + (size_t)c0 * N,
                    k + (size_t)c0 * p.M, n, stage, s,
                    sens ? sens + (size_t)c0 * N : nullptr);
  }
}

size_t adjoint_out_count(const gnufft_plan &p, uint32_t C, int stage)
{
  if (stage == GNUFFT_CONVOLUTION || stage == GNUFFT_DENSITY_ESTIMATION)
    return (size_t)C * p.g.grid_count;
  if (stage == GNUFFT_DEAPODIZATION && p.sens_coils)
    return (size_t)p.g.img_count;
  return (size_t)C * p.g.img_count;
}

void collect_times(gnufft_plan &p, cudaStream_t s)
{
  p.times.launches = p.launches;
  if (!p.timing)
    return;
  GN_CUDA(cudaStreamSynchronize(s));
  float ms[4] = {0, 0, 0, 0};
  for (int i = 0; i < 4; ++i)
    GN_CUDA(cudaEventElapsedTime(&ms[i], p.ev[2 * i], p.ev[2 * i + 1]));
  p.times.prepare_ms = ms[0];
  p.times.gridding_ms = ms[1];
  p.times.fft_ms = ms[2];
  p.times.finish_ms = ms[3];
}

// One coil per pass, maps copied per coil per call, a synchronisation per
// coil (the upstream flow, gpuNUFFT_operator.cpp:682-843 / 941-1051).
void adjoint_plain(gnufft_plan &p, const float2 *k, float2 *img, uint32_t C,
                   int stage, cudaStream_t s, bool host_io)
{
  const size_t N = p.g.img_count, G = p.g.grid_count;
  const bool conv = stage == GNUFFT_CONVOLUTION ||
                    stage == GNUFFT_DENSITY_ESTIMATION;
  const bool combine = stage == GNUFFT_DEAPODIZATION && p.sens_coils;
  const size_t per_out = conv ? G : N;
  p.stage_in.ensure((size_t)p.M * sizeof(float2));
  p.stage_out.ensure(per_out * sizeof(float2));
  DeviceBuffer acc;
  if (combine)
  {
    acc.reset(N * sizeof(float2));
    GN_CUDA(cudaMemsetAsync(acc.get(), 0, N * sizeof(float2), s));
    p.one_sens.ensure(N * sizeof(float2));
  }
  for (uint32_t c = 0; c < C; ++c)
  {
    const float2 *kc = k + (size_t)c * p.M;
    if (host_io)
    {
      GN_CUDA(cudaMemcpyAsync(p.stage_in.get(), kc, p.M * sizeof(float2),
                              cudaMemcpyHostToDevice, s));
      kc = p.stage_in.as<float2>();
    }
    float2 *oc = host_io ? p.stage_out.as<float2>() : img + c * per_out;
    if (combine)
    {
      // maps copied per coil per call, like the upstream
      GN_CUDA(cudaMemcpyAsync(p.one_sens.get(), p.sens_h.data() + c * N,
                              N * sizeof(float2), cudaMemcpyHostToDevice, s));
      // conj(S_c) * image_c added to the running coil sum
      adjoint_batched(p, kc, acc.as<float2>(), 1, stage, s,
                      p.one_sens.as<float2>(), true);
    }
    else
    {
      adjoint_batched(p, kc, oc, 1, stage, s, nullptr);
      if (host_io)
        GN_CUDA(cudaMemcpyAsync(img + c * per_out, oc,
                                per_out * sizeof(float2),
                                cudaMemcpyDeviceToHost, s));
    }
    GN_CUDA(cudaStreamSynchronize(s));
  }
  if (combine)
    GN_CUDA(cudaMemcpyAsync(img, acc.get(), N * sizeof(float2),
                            host_io ? cudaMemcpyDeviceToHost
                                    : cudaMemcpyDeviceToDevice,
                            s));
  GN_CUDA(cudaStreamSynchronize(s));
}
}  // namespace

// ==========================================================================
// C ABI
// ==========================================================================
namespace gnufft
{
bool plan_view(const gnufft_plan *p, PlanView *v)
{
  if (!p || !v)
    return false;
  v->g = p->g;
  v->M = p->M;
  v->device = p->desc.device;
  v->sens_coils = p->sens_coils;
  v->data_indices = p->di.as<uint32_t>();
  v->dens_sorted = p->has_dens ? p->dens_sorted.as<float>() : nullptr;
  v->w_rows = p->w_rows.as<uint32_t>();
  v->w_nz = p->w_nz.as<uint2>();
  return true;
}

bool plan_tables(gnufft_plan *p, uint32_t n_coils, PlanTables *t)
{
  if (!p || !t)
    return false;
  t->g = p->g;
  t->M = p->M;
  t->device = p->desc.device;
  t->sens_coils = p->sens_coils;
  t->tile_coils = p->fwd_tile_coils;
  t->items = p->fwd_items.as<FwdItem>();
  t->n_items = p->n_fwd_items;
  t->traj_sorted = p->traj_sorted.as<float>();
  t->dens_sorted = p->has_dens ? p->dens_sorted.as<float>() : nullptr;
  t->lut = p->lut.as<float>();
  t->deapo = p->deapo.as<float>();
  t->data_indices = p->di.as<uint32_t>();
  t->inverse_indices = p->di_inv.as<uint32_t>();
  t->w_rows = p->w_rows.as<uint32_t>();
  t->w_nz = p->w_nz.as<uint2>();
  t->sens = p->sens_coils ? p->sens.as<float2>() : nullptr;
  t->fft = p->fft_plan((int)n_coils);
  return true;
}

void set_last_error(const std::string &msg) { g_last_error = msg; }
}  // namespace gnufft

extern "C" {

const char *gnufft_version(void) { return kVersion; }

const char *gnufft_last_error(void) { return g_last_error.c_str(); }

const char *gnufft_status_string(gnufft_status s)
{
  switch (s)
  {
  case GNUFFT_SUCCESS: return "success";
  case GNUFFT_ERROR_INVALID_ARGUMENT: return "invalid argument";
  case GNUFFT_ERROR_OUT_OF_MEMORY: return "out of memory";
  case GNUFFT_ERROR_CUDA: return "CUDA error";
  case GNUFFT_ERROR_CUFFT: return "cuFFT error";
  case GNUFFT_ERROR_NOT_SUPPORTED: return "not supported";
  case GNUFFT_ERROR_INTERNAL: return "internal error";
  }
  return "unknown status";
}

gnufft_status gnufft_plan_create(const gnufft_desc *desc, const float *traj,
                                 const float *dens, const void *sens,
                                 gnufft_plan **plan)
{
  if (!plan)
    return (gnufft_status)fail(kInvalidArgument, "plan pointer is NULL");
  *plan = nullptr;
  return guarded([&] {
    validate_desc(desc);
    DeviceGuard dg(desc->device);
    std::unique_ptr<gnufft_plan> p(new gnufft_plan());
    p->desc.device = desc->device;
    create_plan(*p, desc, traj, dens, sens);
    *plan = p.release();
  });
}

gnufft_status gnufft_plan_load(const gnufft_desc *desc,
                               const float *traj_sorted,
                               const uint32_t *data_indices,
                               const uint32_t *sector_data_count,
                               const uint32_t *processing_order,
                               uint32_t n_order,
                               const uint32_t *sector_centers,
                               const float *dens_sorted, const void *sens,
                               const float *deapo, gnufft_plan **plan)
{
  if (!plan)
    return (gnufft_status)fail(kInvalidArgument, "plan pointer is NULL");
  *plan = nullptr;
  return guarded([&] {
    validate_desc(desc);
    DeviceGuard dg(desc->device);
    std::unique_ptr<gnufft_plan> p(new gnufft_plan());
    p->desc.device = desc->device;
    load_plan(*p, desc, traj_sorted, data_indices, sector_data_count,
              processing_order, n_order, sector_centers, dens_sorted, sens,
              deapo);
    *plan = p.release();
  });
}

gnufft_status gnufft_plan_destroy(gnufft_plan *plan)
{
  return guarded([&] { delete plan; });
}

gnufft_status gnufft_plan_get_info(const gnufft_plan *p,
                                   gnufft_plan_info *info)
{
  if (!p || !info)
    return (gnufft_status)fail(kInvalidArgument, "NULL argument");
  return guarded([&] {
    std::memset(info, 0, sizeof(*info));
    info->dim = (uint32_t)p->dim;
    for (int a = 0; a < 3; ++a)
    {
      const bool used = a < p->dim;
      info->img_dims[a] = used ? (uint32_t)p->g.N[a] : 0;
      info->grid_dims[a] = used ? (uint32_t)p->g.G[a] : 0;
      info->sector_dims[a] = used ? (uint32_t)p->g.S[a] : 0;
    }
    info->n_sectors = (uint32_t)p->g.n_sectors;
    info->n_samples = p->M;
    info->n_coils = p->sens_coils;
    info->kernel_lut_len = (uint32_t)p->g.lut_len;
    info->n_processing_order = (uint32_t)(p->order_h.size() / 2);
    info->has_dens = p->has_dens ? 1 : 0;
    info->device_bytes = p->device_bytes();
  });
}

gnufft_status gnufft_export_tables(const gnufft_plan *p, float *traj_sorted,
                                   uint32_t *data_indices,
                                   uint32_t *sector_data_count,
                                   uint32_t *processing_order,
                                   uint32_t *sector_centers,
                                   float *dens_sorted, float *deapo,
                                   float *kernel_lut)
{
  if (!p)
    return (gnufft_status)fail(kInvalidArgument, "plan is NULL");
  return guarded([&] {
    auto cp = [](auto *dst, const auto &v) {
      if (dst && !v.empty())
        std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
    };
    // the per-sample tables are read from the device (complete since the
    // plan's creation synchronised its stream)
    DeviceGuard dg(p->desc.device);
    auto dl = [](void *dst, const DeviceBuffer &b, size_t bytes) {
      if (dst && bytes)
        GN_CUDA(cudaMemcpy(dst, b.get(), bytes, cudaMemcpyDeviceToHost));
    };
    dl(traj_sorted, p->traj_sorted, (size_t)p->dim * p->M * sizeof(float));
    dl(data_indices, p->di, (size_t)p->M * sizeof(uint32_t));
    cp(sector_data_count, p->sdc_h);
    cp(processing_order, p->order_h);
    cp(sector_centers, p->centers_h);
    if (p->has_dens)
      dl(dens_sorted, p->dens_sorted, (size_t)p->M * sizeof(float));
    cp(deapo, p->deapo_h);
    cp(kernel_lut, p->lut_h);
  });
}

gnufft_status gnufft_set_sens(gnufft_plan *p, const void *sens,
                              uint32_t n_coils)
{
  if (!p)
    return (gnufft_status)fail(kInvalidArgument, "plan is NULL");
  return guarded([&] {
    DeviceGuard dg(p->desc.device);
    GN_CUDA(cudaStreamSynchronize(p->stream));
    set_sens_host(*p, sens, n_coils);
    GN_CUDA(cudaStreamSynchronize(p->stream));
  });
}

gnufft_status gnufft_set_sens_device(gnufft_plan *p, const void *sens,
                                     uint32_t n_coils, void *stream)
{
  if (!p)
    return (gnufft_status)fail(kInvalidArgument, "plan is NULL");
  if (!sens || n_coils == 0)
    return (gnufft_status)fail(kInvalidArgument, "no maps given");
  if (p->plain)
    return (gnufft_status)fail(kNotSupported,
                               "plain plans take host maps (gnufft_set_sens)");
  return guarded([&] {
    DeviceGuard dg(p->desc.device);
    const size_t n = (size_t)n_coils * p->g.img_count;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // the copy is ordered on `stream` only: work on other streams that may
    // still read the previous maps must be ordered before it by the caller
    p->sens.ensure(n * sizeof(float2));
    GN_CUDA(cudaMemcpyAsync(p->sens.get(), sens, n * sizeof(float2),
                            cudaMemcpyDeviceToDevice, s));
    p->sens_h.clear();
    p->sens_coils = n_coils;
  });
}

gnufft_status gnufft_set_memory_limit(gnufft_plan *p, uint64_t bytes)
{
  if (!p)
    return (gnufft_status)fail(kInvalidArgument, "plan is NULL");
  p->mem_limit = (size_t)bytes;
  return GNUFFT_SUCCESS;
}

gnufft_status gnufft_call_scratch_bytes(const gnufft_plan *p,
                                        uint32_t n_coils, uint64_t *bytes)
{
  if (!p || !bytes || !n_coils)
    return (gnufft_status)fail(kInvalidArgument, "invalid argument");
  *bytes = (uint64_t)call_scratch_bytes(*p, n_coils);
  return GNUFFT_SUCCESS;
}

gnufft_status gnufft_set_copy_wait(gnufft_plan *p, int64_t polls)
{
  if (!p)
    return (gnufft_status)fail(kInvalidArgument, "plan is NULL");
  p->copy_polls = polls < 0 ? tma::kMbarSpin : (long long)polls;
  return GNUFFT_SUCCESS;
}

gnufft_status gnufft_plan_check(gnufft_plan *p)
{
  if (!p)
    return (gnufft_status)fail(kInvalidArgument, "plan is NULL");
  return guarded([&] { check_copy_err(*p); });
}

gnufft_status gnufft_set_timing(gnufft_plan *p, int enable)
{
  if (!p)
    return (gnufft_status)fail(kInvalidArgument, "plan is NULL");
  return guarded([&] {
    DeviceGuard dg(p->desc.device);
    if (enable && !p->ev[0])
      for (auto &e : p->ev)
        GN_CUDA(cudaEventCreate(&e));
    p->timing = enable != 0;
  });
}

gnufft_status gnufft_get_stage_times(const gnufft_plan *p,
                                     gnufft_stage_times *t)
{
  if (!p || !t)
    return (gnufft_status)fail(kInvalidArgument, "NULL argument");
  *t = p->times;
  return GNUFFT_SUCCESS;
}

gnufft_status gnufft_adjoint_device(gnufft_plan *p, const void *kspace,
                                    void *image, uint32_t n_coils,
                                    int32_t output, void *stream)
{
  if (!p || !kspace || !image)
    return (gnufft_status)fail(kInvalidArgument, "NULL argument");
  if (output < 0 || output > 3)
    return (gnufft_status)fail(kInvalidArgument, "unknown output stage");
  return guarded([&] {
    DeviceGuard dg(p->desc.device);
    check_coils(*p, n_coils);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    p->launches = 0;
    if (p->plain)
      adjoint_plain(*p, (const float2 *)kspace, (float2 *)image, n_coils,
                    output, s, false);
    else
      adjoint_chunked(*p, (const float2 *)kspace, (float2 *)image, n_coils,
                      output, s);
    collect_times(*p, s);
  });
}

gnufft_status gnufft_forward_device(gnufft_plan *p, const void *image,
                                    void *kspace, uint32_t n_coils,
                                    int32_t output, void *stream)
{
  if (!p || !kspace || !image)
    return (gnufft_status)fail(kInvalidArgument, "NULL argument");
  if (output < 0 || output > 3)
    return (gnufft_status)fail(kInvalidArgument, "unknown output stage");
  return guarded([&] {
    DeviceGuard dg(p->desc.device);
    check_coils(*p, n_coils);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    p->launches = 0;
    if (p->plain)
    {
      const size_t N = p->g.img_count;
      p->one_sens.ensure(N * sizeof(float2));
      for (uint32_t c = 0; c < n_coils; ++c)
      {
        const float2 *ic = (const float2 *)image;
        const float2 *sc = nullptr;
        if (p->sens_coils)
        {
          GN_CUDA(cudaMemcpyAsync(p->one_sens.get(), p->sens_h.data() + c * N,
                                  N * sizeof(float2), cudaMemcpyHostToDevice,
                                  s));
          sc = p->one_sens.as<float2>();
        }
        else
          ic += c * N;
        forward_batched(*p, ic, (float2 *)kspace + (size_t)c * p->M, 1,
                        output, s, sc);
        GN_CUDA(cudaStreamSynchronize(s));
      }
    }
    else
      forward_chunked(*p, (const float2 *)image, (float2 *)kspace, n_coils,
                      output, s);
    collect_times(*p, s);
  });
}

gnufft_status gnufft_adjoint_host(gnufft_plan *p, const void *kspace,
                                  void *image, uint32_t n_coils,
                                  int32_t output)
{
  if (!p || !kspace || !image)
    return (gnufft_status)fail(kInvalidArgument, "NULL argument");
  if (output < 0 || output > 3)
    return (gnufft_status)fail(kInvalidArgument, "unknown output stage");
  return guarded([&] {
    DeviceGuard dg(p->desc.device);
    check_coils(*p, n_coils);
    cudaStream_t s = p->stream;
    p->launches = 0;
    if (p->plain)
    {
      adjoint_plain(*p, (const float2 *)kspace, (float2 *)image, n_coils,
                    output, s, true);
      collect_times(*p, s);
      return;
    }
    const size_t nin = (size_t)n_coils * p->M;
    const size_t nout = adjoint_out_count(*p, n_coils, output);
    p->stage_in.ensure(nin * sizeof(float2));
    p->stage_out.ensure(nout * sizeof(float2));
    copy_host_to_device(p->stage_in.get(), kspace, nin * sizeof(float2), s);
    adjoint_chunked(*p, p->stage_in.as<float2>(), p->stage_out.as<float2>(),
                    n_coils, output, s);
    copy_device_to_host(image, p->stage_out.get(), nout * sizeof(float2), s);
    GN_CUDA(cudaStreamSynchronize(s));
    collect_times(*p, s);
    check_copy_err(*p);  // this call's own tile copies
  });
}

gnufft_status gnufft_forward_host(gnufft_plan *p, const void *image,
                                  void *kspace, uint32_t n_coils,
                                  int32_t output)
{
  if (!p || !kspace || !image)
    return (gnufft_status)fail(kInvalidArgument, "NULL argument");
  if (output < 0 || output > 3)
    return (gnufft_status)fail(kInvalidArgument, "unknown output stage");
  return guarded([&] {
    DeviceGuard dg(p->desc.device);
    check_coils(*p, n_coils);
    cudaStream_t s = p->stream;
    p->launches = 0;
    const size_t nin =
        (p->sens_coils ? 1 : (size_t)n_coils) * (size_t)p->g.img_count;
    const size_t nout = (size_t)n_coils * p->M;
    p->stage_in.ensure(nin * sizeof(float2));
    p->stage_out.ensure(nout * sizeof(float2));
    copy_host_to_device(p->stage_in.get(), image, nin * sizeof(float2), s);
    if (p->plain)
    {
      gnufft_status st = gnufft_forward_device(p, p->stage_in.get(),
                                               p->stage_out.get(), n_coils,
                                               output, s);
      if (st != GNUFFT_SUCCESS)
        throw Error(st, g_last_error);
    }
    else
      forward_chunked(*p, p->stage_in.as<float2>(), p->stage_out.as<float2>(),
                      n_coils, output, s);
    copy_device_to_host(kspace, p->stage_out.get(), nout * sizeof(float2), s);
    GN_CUDA(cudaStreamSynchronize(s));
    collect_times(*p, s);
    check_copy_err(*p);  // this call's own tile copies
  });
}

gnufft_status gnufft_traj_grad_device(gnufft_plan *p, const void *image,
                                      const void *kspace_weights,
                                      uint32_t n_coils, float *grad_traj,
                                      void *stream)
{
  if (!p || !image || !kspace_weights || !grad_traj)
    return (gnufft_status)fail(kInvalidArgument, "NULL argument");
  return guarded([&] {
    DeviceGuard dg(p->desc.device);
    check_coils(*p, n_coils);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    p->launches = 0;
    traj_grad(*p, (const float2 *)image, (const float2 *)kspace_weights,
              n_coils, grad_traj, s, p->sens.as<float2>());
    p->times.launches = p->launches;
  });
}

}  // extern "C"
