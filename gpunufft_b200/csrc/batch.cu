// Batches of independent operators: the C entry points declared in
// include/gpunufft_b200.h (gnufft_batch_*) over the batched stages of
// gridding.cu.  A batch holds one descriptor per instance (the plan's
// tables, the instance's scratch and its first unit of every stage) in
// device memory; a call launches each stage once for all instances and one
// cuFFT call per instance between them.
#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include <cufft.h>
#include <cuda_runtime.h>

#include "../../include/gpunufft_b200.h"
#include "capi.hpp"
#include "devutil.hpp"
#include "gridding.cuh"
#include "planview.hpp"

using namespace gnufft;

struct gnufft_batch
{
  int device = 0;
  uint32_t n = 0;
  std::vector<BatchInst> inst;    // host copies of the descriptors
  std::vector<cufftHandle> fft;   // the plans' cuFFT plans (owned by them)
  DeviceBuffer inst_d, arena, counters;
  uint32_t total[kBatchStages] = {};
  size_t interp_smem = 0;
  BatchIo io{};  // per-call data pointers (kernel parameter)
  // the transforms run on side streams forked from the caller's stream;
  // instances that share a cuFFT plan (frames of one plan) share a side
  // stream, since a plan's work area serves one transform at a time
  std::vector<int> fft_stream;
  std::vector<cudaStream_t> side;
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr;

  ~gnufft_batch()
  {
    for (cudaStream_t st : side)
      cudaStreamDestroy(st);
    for (cudaEvent_t e : join)
      cudaEventDestroy(e);
    if (fork)
      cudaEventDestroy(fork);
  }
};

namespace
{
size_t align256(size_t v) { return (v + 255) / 256 * 256; }

void check_batch(const gnufft_batch *b)
{
  if (!b)
    throw Error(kInvalidArgument, "NULL batch");
}

constexpr int kSideStreams = 8;

// One cuFFT call per instance, spread over the side streams (fork: the
// side streams wait for the caller's stream; join: the caller's stream
// waits for every side stream).  Event records and waits are captured
// into a CUDA graph like the launches.
void run_ffts(gnufft_batch &b, int direction, cudaStream_t s)
{
  GN_CUDA(cudaEventRecord(b.fork, s));
  for (cudaStream_t st : b.side)
    GN_CUDA(cudaStreamWaitEvent(st, b.fork, 0));
  for (uint32_t i = 0; i < b.n; ++i)
  {
    cudaStream_t st = b.side[b.fft_stream[i]];
    check_cufft(cufftSetStream(b.fft[i], st), "cufftSetStream");
    cufftComplex *g = reinterpret_cast<cufftComplex *>(b.inst[i].grid);
    check_cufft(cufftExecC2C(b.fft[i], g, g, direction), "cufftExecC2C");
  }
  for (size_t k = 0; k < b.side.size(); ++k)
  {
    GN_CUDA(cudaEventRecord(b.join[k], b.side[k]));
    GN_CUDA(cudaStreamWaitEvent(s, b.join[k], 0));
  }
}

// Public work units per stage: prepare, interpolation (2-D and 3-D),
// gather, spread, finish.
void public_units(const gnufft_batch &b, uint32_t out[5])
{
  out[0] = b.total[kBatchPrepare];
  out[1] = b.total[kBatchInterp] + b.total[kBatchInterp3];
  out[2] = b.total[kBatchGather];
  out[3] = b.total[kBatchSpread];
  out[4] = b.total[kBatchFinish];
}
}  // namespace

extern "C" {

gnufft_status gnufft_batch_create(gnufft_plan *const *plans,
                                  const uint32_t *n_coils,
                                  uint32_t n_instances, gnufft_batch **out)
{
  if (!plans || !n_coils || !out)
    return (gnufft_status)fail(kInvalidArgument, "NULL argument");
  *out = nullptr;
  if (n_instances == 0 || n_instances > (uint32_t)kBatchMax)
    return (gnufft_status)fail(kInvalidArgument,
                               "a batch holds 1 to 512 instances");
  return guarded([&] {
    PlanView v0;
    if (!plan_view(plans[0], &v0))
      throw Error(kInvalidArgument, "NULL plan");
    auto b = std::make_unique<gnufft_batch>();
    b->device = v0.device;
    b->n = n_instances;
    DeviceGuard dg(b->device);
    b->inst.resize(n_instances);
    b->fft.resize(n_instances);
    std::vector<size_t> grid_off(n_instances), ks_off(n_instances);
    size_t bytes = 0;
    for (uint32_t i = 0; i < n_instances; ++i)
    {
      const std::string who = "instance " + std::to_string(i) + ": ";
      PlanView v;
      if (!plan_view(plans[i], &v))
        throw Error(kInvalidArgument, who + "NULL plan");
      if (v.device != b->device)
        throw Error(kInvalidArgument, who + "plans on different devices");
      const uint32_t C = n_coils[i];
      if (C == 0 || (v.sens_coils && C != v.sens_coils))
        throw Error(kInvalidArgument,
                    who + "n_coils must be positive and match the maps");
      PlanTables t;
      plan_tables(plans[i], C, &t);
      BatchInst &bi = b->inst[i];
      bi = BatchInst{};
      bi.g = t.g;
      bi.M = t.M;
      bi.C = (int)C;
      bi.signs = 0;  // cuFFT of the unsigned grid; the shift is folded in
      bi.n_items = t.n_items;
      bi.items = t.items;
      bi.traj = t.traj_sorted;
      bi.dens = t.dens_sorted;
      bi.lut = t.lut;
      bi.deapo = t.deapo;
      bi.di = t.data_indices;
      bi.di_inv = t.inverse_indices;
      bi.w_rows = t.w_rows;
      bi.w_nz = t.w_nz;
      bi.sens = t.sens;
      batch_configure(bi, t.tile_coils);
      if ((size_t)bi.M * bi.CP > 0xFFFFFFFFull)
        throw Error(kNotSupported, who + "samples x coil lanes exceed 2^32");
      const size_t smem = batch_interp_smem(bi);
      if (smem > 200 * 1024)
        throw Error(kNotSupported,
                    who + "forward tile exceeds shared memory");
      b->interp_smem = std::max(b->interp_smem, smem);
      b->fft[i] = t.fft;
      grid_off[i] = bytes;
      bytes += align256((size_t)C * t.g.grid_count * sizeof(float2));
      ks_off[i] = bytes;
      bytes += align256((size_t)t.M * bi.CP * sizeof(float2));
    }
    b->arena.reset(bytes);
    unsigned char *base = b->arena.as<unsigned char>();
    uint64_t totals[kBatchStages] = {};
    for (uint32_t i = 0; i < n_instances; ++i)
    {
      BatchInst &bi = b->inst[i];
      bi.grid = reinterpret_cast<float2 *>(base + grid_off[i]);
      bi.ks = reinterpret_cast<float2 *>(base + ks_off[i]);
      uint32_t units[kBatchStages];
      batch_units(bi, units);
      for (int st = 0; st < kBatchStages; ++st)
      {
        bi.first[st] = (uint32_t)totals[st];
        totals[st] += units[st];
        // the counter passes the total by up to one unit per block
        if (totals[st] >= 0x7FFFFFFFull)
          throw Error(kNotSupported, "too many work units in one batch");
      }
    }
    for (int st = 0; st < kBatchStages; ++st)
      b->total[st] = (uint32_t)totals[st];
    b->inst_d.reset(n_instances * sizeof(BatchInst));
    GN_CUDA(cudaMemcpy(b->inst_d.get(), b->inst.data(),
                       n_instances * sizeof(BatchInst),
                       cudaMemcpyHostToDevice));
    b->counters.reset(kBatchStages * sizeof(unsigned));
    // side streams for the transforms: one per distinct cuFFT plan, at most
    // kSideStreams
    b->fft_stream.resize(n_instances);
    std::vector<cufftHandle> seen;
    for (uint32_t i = 0; i < n_instances; ++i)
    {
      auto it = std::find(seen.begin(), seen.end(), b->fft[i]);
      const int k = (int)(it - seen.begin());
      if (it == seen.end())
        seen.push_back(b->fft[i]);
      b->fft_stream[i] = k % kSideStreams;
    }
    const int ns = std::min<int>(kSideStreams, (int)seen.size());
    GN_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    for (int k = 0; k < ns; ++k)
    {
      cudaStream_t st;
      GN_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
      b->side.push_back(st);
      cudaEvent_t e;
      GN_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      b->join.push_back(e);
    }
    *out = b.release();
  });
}

gnufft_status gnufft_batch_forward(gnufft_batch *b, const void *const *images,
                                   void *const *kspace, void *stream)
{
  if (!b || !images || !kspace)
    return (gnufft_status)fail(kInvalidArgument, "NULL argument");
  return guarded([&] {
    DeviceGuard dg(b->device);
    for (uint32_t i = 0; i < b->n; ++i)
    {
      if (!images[i] || !kspace[i])
        throw Error(kInvalidArgument,
                    "NULL data pointer of instance " + std::to_string(i));
      b->io.in[i] = static_cast<const float2 *>(images[i]);
      b->io.out[i] = static_cast<float2 *>(kspace[i]);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned *cnt = b->counters.as<unsigned>();
    const BatchInst *inst = b->inst_d.as<BatchInst>();
    GN_CUDA(cudaMemsetAsync(cnt, 0, kBatchStages * sizeof(unsigned), s));
    launch_batch_stage(kBatchPrepare, inst, (int)b->n, b->total[kBatchPrepare],
                       &b->io, cnt + kBatchPrepare, 0, s);
    run_ffts(*b, CUFFT_FORWARD, s);
    launch_batch_stage(kBatchInterp, inst, (int)b->n, b->total[kBatchInterp],
                       &b->io, cnt + kBatchInterp, b->interp_smem, s);
    launch_batch_stage(kBatchInterp3, inst, (int)b->n,
                       b->total[kBatchInterp3], &b->io, cnt + kBatchInterp3,
                       b->interp_smem, s);
  });
}

gnufft_status gnufft_batch_adjoint(gnufft_batch *b, const void *const *kspace,
                                   void *const *images, void *stream)
{
  if (!b || !images || !kspace)
    return (gnufft_status)fail(kInvalidArgument, "NULL argument");
  return guarded([&] {
    DeviceGuard dg(b->device);
    for (uint32_t i = 0; i < b->n; ++i)
    {
      if (!images[i] || !kspace[i])
        throw Error(kInvalidArgument,
                    "NULL data pointer of instance " + std::to_string(i));
      b->io.in[i] = static_cast<const float2 *>(kspace[i]);
      b->io.out[i] = static_cast<float2 *>(images[i]);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned *cnt = b->counters.as<unsigned>();
    const BatchInst *inst = b->inst_d.as<BatchInst>();
    GN_CUDA(cudaMemsetAsync(cnt, 0, kBatchStages * sizeof(unsigned), s));
    launch_batch_stage(kBatchGather, inst, (int)b->n, b->total[kBatchGather],
                       &b->io, cnt + kBatchGather, 0, s);
    launch_batch_stage(kBatchSpread, inst, (int)b->n, b->total[kBatchSpread],
                       &b->io, cnt + kBatchSpread, 0, s);
    run_ffts(*b, CUFFT_INVERSE, s);
    launch_batch_stage(kBatchFinish, inst, (int)b->n, b->total[kBatchFinish],
                       &b->io, cnt + kBatchFinish, 0, s);
  });
}

gnufft_status gnufft_batch_get_info(const gnufft_batch *b,
                                    gnufft_batch_info *info)
{
  if (!b || !info)
    return (gnufft_status)fail(kInvalidArgument, "NULL argument");
  return guarded([&] {
    check_batch(b);
    info->n_instances = b->n;
    public_units(*b, info->units);
    info->kernels_forward = 1 + (b->total[kBatchInterp] > 0) +
                            (b->total[kBatchInterp3] > 0);
    info->kernels_adjoint = 3;
    info->fft_calls = b->n;
    info->device_bytes =
        b->arena.bytes() + b->inst_d.bytes() + b->counters.bytes();
  });
}

gnufft_status gnufft_batch_destroy(gnufft_batch *b)
{
  if (!b)
    return GNUFFT_SUCCESS;
  return guarded([&] {
    DeviceGuard dg(b->device);
    delete b;
  });
}

}  // extern "C"
