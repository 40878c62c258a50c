/*
 * Test-oracle harness around the upstream gpuNUFFT library (built from its
 * own, unmodified sources by oracle/build_ref.sh into oracle/_ref/).
 *
 * This is TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py load it, as the checker / timed reference.
 * The product never links or calls it.
 *
 * Entry points:
 *  - refh_* (CPU only): the upstream kernel LUT (gpuNUFFT_utils.cpp:74-107),
 *    the upstream sector tables computed by the upstream factory with
 *    useGpu=false (gpuNUFFT_operator_factory.cpp:56-270, 450-553 minus the
 *    GPU-only deapodization step), and the upstream CPU gridding routine
 *    gpuNUFFT_cpu (cpu/gpuNUFFT_cpu.cpp:3-159) that its unit tests use.
 *  - refg_* (GPU): the upstream operator created exactly like the upstream
 *    Python binding does (python/gpuNUFFT_operator_python_factory.cpp:70-120),
 *    with or without textures (the texture operators run through the
 *    texture-object stand-ins of oracle/ref_compat.h), and its host-array
 *    adjoint / forward.
 */
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <exception>
#include <stdexcept>
#include <string>
#include <vector>

#include "gpuNUFFT_operator_factory.hpp"
#include "gpuNUFFT_cpu.hpp"

namespace
{
thread_local std::string g_err;

class TableFactory : public gpuNUFFT::GpuNUFFTOperatorFactory
{
 public:
  explicit TableFactory(bool balance)
    : gpuNUFFT::GpuNUFFTOperatorFactory(false, false, balance)
  {
  }
  using gpuNUFFT::GpuNUFFTOperatorFactory::assignSectors;
  using gpuNUFFT::GpuNUFFTOperatorFactory::computeProcessingOrder;
  using gpuNUFFT::GpuNUFFTOperatorFactory::computeSectorCenters;
  using gpuNUFFT::GpuNUFFTOperatorFactory::computeSectorCenters2D;
  using gpuNUFFT::GpuNUFFTOperatorFactory::computeSectorDataCount;
  using gpuNUFFT::GpuNUFFTOperatorFactory::computeTotalSectorCount;
  using gpuNUFFT::GpuNUFFTOperatorFactory::createNewGpuNUFFTOperator;
};

/* gpuNUFFT_operator_factory.cpp:56-72 (sortVector) is a template that the
 * upstream object file does not export, so the harness performs the same
 * call: a vector of upstream IndPair (compared by sector, gpuNUFFT_types.hpp
 * :33-49) sorted with the same libstdc++ std::sort. */
std::vector<gpuNUFFT::IndPair> sort_pairs(const gpuNUFFT::Array<IndType> &a,
                                          uint32_t n)
{
  std::vector<gpuNUFFT::IndPair> v;
  for (IndType i = 0; i < n; i++)
    v.push_back(gpuNUFFT::IndPair(i, a.data[i]));
  std::sort(v.begin(), v.end());
  return v;
}

gpuNUFFT::Dimensions make_dims(uint32_t w, uint32_t h, uint32_t d)
{
  gpuNUFFT::Dimensions dims;
  dims.width = w;
  dims.height = h;
  dims.depth = d;
  return dims;
}
}  // namespace

extern "C" {

const char *refh_last_error(void) { return g_err.c_str(); }

/* Upstream LUT: calculateGrid3KernelSize + load1DKernel (or the linear-
 * interpolation size calculateKernelSizeLinInt when lin != 0).
 * Returns the entry count; writes at most cap entries. */
long refh_kernel_lut(float osf, uint32_t kw, int lin, float *out, long cap)
{
  long n = lin ? calculateKernelSizeLinInt(osf, kw)
               : calculateGrid3KernelSize(osf, kw);
  if (out && cap >= n)
    load1DKernel(out, n, (int)kw, osf);
  return n;
}

/* Sector counts of the upstream factory for these dims: writes per-axis
 * counts to out3 and returns the total. */
uint32_t refh_sector_dims(uint32_t w, uint32_t h, uint32_t d, float osf,
                          uint32_t sw, uint32_t *out3)
{
  gpuNUFFT::Dimensions img = make_dims(w, h, d);
  gpuNUFFT::Dimensions grid = img * osf;
  auto per = [&](uint32_t g) -> uint32_t {
    return g == 0 ? 0 : (uint32_t)std::ceil(static_cast<float>(g) / sw);
  };
  out3[0] = per(grid.width);
  out3[1] = per(grid.height);
  out3[2] = per(grid.depth);
  uint32_t t = 1;
  for (int i = 0; i < 3; ++i)
    t *= out3[i] ? out3[i] : 1;
  return t;
}

/* Upstream factory tables for a trajectory (SoA, dim*M floats), computed
 * with useGpu=false.  Buffers: assigned[M] (per-sample sector id in the
 * ORIGINAL order), data_indices[M], sector_data_count[S+1],
 * centers[dim*S], order[2*cap_order] (balanced only), traj_sorted[dim*M],
 * dens_sorted[M] (if dens != NULL).  Returns the processing-order length
 * (0 when balance == 0) or -1 on error. */
long refh_sector_tables(const float *traj, uint32_t M, uint32_t w, uint32_t h,
                        uint32_t d, float osf, uint32_t kw, uint32_t sw,
                        int balance, const float *dens, uint32_t *assigned,
                        uint32_t *data_indices, uint32_t *sector_data_count,
                        uint32_t *centers, uint32_t *order, long cap_order,
                        float *traj_sorted, float *dens_sorted)
{
  try
  {
    TableFactory f(balance != 0);
    gpuNUFFT::Dimensions img = make_dims(w, h, d);
    gpuNUFFT::GpuNUFFTOperator *op =
        f.createNewGpuNUFFTOperator(kw, sw, osf, img);
    const int dim = op->is2DProcessing() ? 2 : 3;

    std::vector<float> traj_copy(traj, traj + (size_t)dim * M);
    gpuNUFFT::Array<DType> ktraj;
    ktraj.data = traj_copy.data();
    ktraj.dim.length = M;

    gpuNUFFT::Array<IndType> as = f.assignSectors(op, ktraj);
    std::memcpy(assigned, as.data, sizeof(uint32_t) * M);
    std::vector<gpuNUFFT::IndPair> sorted = sort_pairs(as, M);

    // same host gather as the upstream factory's useGpu=false branch
    for (uint32_t i = 0; i < M; i++)
    {
      for (int a = 0; a < dim; ++a)
        traj_sorted[i + (size_t)a * M] =
            traj[sorted[i].first + (size_t)a * M];
      if (dens && dens_sorted)
        dens_sorted[i] = dens[sorted[i].first];
      data_indices[i] = sorted[i].first;
      as.data[i] = sorted[i].second;
    }
    gpuNUFFT::Array<IndType> cnt = f.computeSectorDataCount(op, as);
    std::memcpy(sector_data_count, cnt.data, sizeof(uint32_t) * cnt.count());
    op->setSectorDataCount(cnt);

    long nord = 0;
    if (balance)
    {
      f.computeProcessingOrder(op);
      gpuNUFFT::Array<IndType2> po =
          static_cast<gpuNUFFT::BalancedGpuNUFFTOperator *>(op)
              ->getSectorProcessingOrder();
      nord = (long)po.count();
      if (nord > cap_order)
        throw std::runtime_error("processing order buffer too small");
      for (long i = 0; i < nord; ++i)
      {
        order[2 * i] = po.data[i].x;
        order[2 * i + 1] = po.data[i].y;
      }
    }
    gpuNUFFT::Array<IndType> ctr = dim == 3 ? f.computeSectorCenters(op)
                                            : f.computeSectorCenters2D(op);
    std::memcpy(centers, ctr.data, sizeof(uint32_t) * ctr.count() * 1);
    op->setSectorCenters(ctr);
    free(as.data);
    delete op;  // frees the count / centers / order arrays it was handed
    return nord;
  }
  catch (const std::exception &e)
  {
    g_err = e.what();
    return -1;
  }
}

/* The upstream CPU gridding routine (isotropic 3D adjoint convolution,
 * AoS coords, out-of-grid cells dropped).  All arrays as upstream expects:
 * data[2*M] sorted, crds[3*M] sorted AoS, gdata[2*width^3] accumulated. */
void refh_cpu_gridding(float *data, float *crds, float *gdata, float *kernel,
                       int *sectors, int sector_count, int *sector_centers,
                       int sector_width, int kernel_width, int kernel_count,
                       int width)
{
  gpuNUFFT_cpu(data, crds, gdata, kernel, sectors, sector_count, sector_centers,
               sector_width, kernel_width, kernel_count, width);
}

/* ---------------- GPU side: the upstream operator ------------------------ */

struct RefOp
{
  gpuNUFFT::GpuNUFFTOperator *op;
  std::vector<float2> sens;  // the operator keeps only a pointer
  uint32_t M, C, w, h, d;
  bool has_sens;
};

void *refg_create(const float *traj, uint32_t M, uint32_t w, uint32_t h,
                  uint32_t d, const float *dens, const float *sens_c64,
                  uint32_t n_coils, uint32_t kw, uint32_t sw, float osf,
                  int balance, int textures)
{
  try
  {
    RefOp *r = new RefOp();
    r->M = M;
    r->C = n_coils;
    r->w = w;
    r->h = h;
    r->d = d;
    gpuNUFFT::GpuNUFFTOperatorFactory factory(textures != 0, true,
                                              balance != 0);
    gpuNUFFT::Dimensions img = make_dims(w, h, d);
    const int dim = d == 0 ? 2 : 3;
    std::vector<float> traj_copy(traj, traj + (size_t)dim * M);
    gpuNUFFT::Array<DType> ktraj;
    ktraj.data = traj_copy.data();
    ktraj.dim.length = M;
    std::vector<float> dens_copy;
    gpuNUFFT::Array<DType> densArr;
    if (dens)
    {
      dens_copy.assign(dens, dens + M);
      densArr.data = dens_copy.data();
      densArr.dim.length = M;
    }
    gpuNUFFT::Array<DType2> sensArr;
    r->has_sens = sens_c64 != nullptr;
    if (r->has_sens)
    {
      size_t n = (size_t)img.count() * n_coils;
      r->sens.resize(n);
      std::memcpy(r->sens.data(), sens_c64, n * sizeof(float2));
      sensArr.data = r->sens.data();
      sensArr.dim = img;
      sensArr.dim.channels = n_coils;
    }
    r->op = factory.createGpuNUFFTOperator(ktraj, densArr, sensArr, kw, sw,
                                           osf, img);
    cudaDeviceSynchronize();
    return r;
  }
  catch (const std::exception &e)
  {
    g_err = e.what();
    return nullptr;
  }
}

/* Adjoint with host arrays; output stage as upstream GpuNUFFTOutput. */
int refg_adjoint(void *h, const float *kspace_c64, float *out_c64, int stage)
{
  RefOp *r = static_cast<RefOp *>(h);
  gpuNUFFT::Array<DType2> k;
  k.data = (DType2 *)kspace_c64;
  k.dim.length = r->M;
  k.dim.channels = r->C;
  gpuNUFFT::Array<CufftType> img;
  img.data = (CufftType *)out_c64;
  if (stage == gpuNUFFT::CONVOLUTION || stage == gpuNUFFT::DENSITY_ESTIMATION)
    img.dim = r->op->getGridDims();
  else
    img.dim = r->op->getImageDims();
  img.dim.channels = r->has_sens ? 1 : r->C;
  r->op->performGpuNUFFTAdj(k, img, (gpuNUFFT::GpuNUFFTOutput)stage);
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

int refg_forward(void *h, const float *image_c64, float *kspace_c64, int stage)
{
  RefOp *r = static_cast<RefOp *>(h);
  gpuNUFFT::Array<DType2> img;
  img.data = (DType2 *)image_c64;
  img.dim = r->op->getImageDims();
  img.dim.channels = r->has_sens ? 1 : r->C;
  gpuNUFFT::Array<CufftType> k;
  k.data = (CufftType *)kspace_c64;
  k.dim.length = r->M;
  k.dim.channels = r->C;
  r->op->performForwardGpuNUFFT(img, k, (gpuNUFFT::GpuNUFFTOutput)stage);
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}


void refg_destroy(void *h)
{
  RefOp *r = static_cast<RefOp *>(h);
  if (!r)
    return;
  delete r->op;
  delete r;
}

}  // extern "C"
