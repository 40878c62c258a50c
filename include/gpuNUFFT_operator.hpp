/*
 * gpuNUFFT::GpuNUFFTOperator and its balanced / texture variants for the
 * gpunufft_b200 drop-in: header-only C++ classes over the C ABI in
 * gpunufft_b200.h (link libgpunufft_b200.so; nothing else).
 *
 * Signatures follow the upstream's gpuNUFFT_operator.hpp:92-363,
 * balanced_operator.hpp:13-20, balanced_gpuNUFFT_operator.hpp,
 * texture_gpuNUFFT_operator.hpp and balanced_texture_gpuNUFFT_operator.hpp
 * (andyschwarzl/gpuNUFFT, CUDA/inc), so C++ callers of the upstream compile
 * unchanged.  Differences, all in the direction of the upstream's
 * documented intent:
 *  - errors throw (std::invalid_argument for bad arguments, else
 *    std::runtime_error) where the upstream exits the process;
 *  - CONVOLUTION / FFT outputs of host calls hold every coil;
 *  - the sector tables, trajectory, density weights and geometry are fixed
 *    when the operator is created: their setters throw std::logic_error
 *    (setSens replaces the maps of a live operator, as upstream);
 *  - operators are independent objects (the upstream shares global device
 *    constants between live operators).
 * Operators are created by gpuNUFFT::GpuNUFFTOperatorFactory
 * (gpuNUFFT_operator_factory.hpp).
 */
#ifndef GPUNUFFT_OPERATOR_H_INCLUDED
#define GPUNUFFT_OPERATOR_H_INCLUDED

#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "gpuNUFFT_types.hpp"
#include "gpunufft_b200.h"

namespace gpuNUFFT
{
class GpuNUFFTOperatorFactory;

namespace detail
{
/* A C-ABI status as the exception the C++ API throws. */
inline void check(gnufft_status st)
{
  if (st == GNUFFT_SUCCESS)
    return;
  const char *m = gnufft_last_error();
  const std::string msg = std::string("gpuNUFFT: ") +
                          gnufft_status_string(st) + ": " + (m ? m : "");
  if (st == GNUFFT_ERROR_INVALID_ARGUMENT)
    throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

inline void fixed(const char *what)
{
  throw std::logic_error(std::string("gpuNUFFT: ") + what +
                         " is fixed when the operator is created "
                         "(create a new operator with the factory)");
}
}  // namespace detail

class GpuNUFFTOperator
{
 public:
  virtual ~GpuNUFFTOperator()
  {
    if (plan)
      gnufft_plan_destroy(plan);
    if (!matlabSharedMem)
      for (void *p : owned)
        std::free(p);
  }

  friend class GpuNUFFTOperatorFactory;

  // ---------------------------------------------------------------- setters
  void setOsf(DType) { detail::fixed("the oversampling ratio"); }
  void setKSpaceTraj(Array<DType>) { detail::fixed("the trajectory"); }
  void setSectorCenters(Array<IndType>) { detail::fixed("the sector centers"); }
  void setSectorDataCount(Array<IndType>)
  {
    detail::fixed("the sector data count");
  }
  void setDataIndices(Array<IndType>) { detail::fixed("the data indices"); }
  void setDens(Array<DType>) { detail::fixed("the density compensation"); }
  void setDeapodizationFunction(Array<DType>)
  {
    detail::fixed("the deapodization function");
  }
  void setImageDims(Dimensions) { detail::fixed("the image size"); }
  void setGridSectorDims(Dimensions) { detail::fixed("the sector layout"); }
  /* Replace the sensitivity maps (copied into the operator; sens.data ==
   * NULL removes them). */
  void setSens(Array<DType2> s)
  {
    const IndType ch = s.data ? DEFAULT_VALUE(s.dim.channels) : 0;
    detail::check(gnufft_set_sens(plan, s.data, ch));
    sens = s;
  }

  // ---------------------------------------------------------------- getters
  DType getOsf() { return osf; }
  /* the trajectory in sector-sorted order (structure of arrays) */
  Array<DType> getKSpaceTraj()
  {
    tables();
    return array_of(traj_h, info.n_samples);
  }
  Array<DType2> getSens() { return sens; }
  /* density compensation in sector-sorted order (empty without) */
  Array<DType> getDens()
  {
    tables();
    return array_of(dens_h, info.has_dens ? info.n_samples : 0);
  }
  /* the kernel lookup table */
  Array<DType> getKernel()
  {
    tables();
    return array_of(lut_h, info.kernel_lut_len);
  }
  Array<IndType> getSectorDataCount()
  {
    tables();
    return array_of(sdc_h, info.n_sectors + 1);
  }
  IndType getKernelWidth() { return kernelWidth; }
  IndType getSectorWidth() { return sectorWidth; }
  Dimensions getImageDims() { return imgDims; }
  Dimensions getGridDims() { return imgDims * osf; }
  /* sectors per axis */
  Dimensions getGridSectorDims()
  {
    Dimensions d(info.sector_dims[0], info.sector_dims[1],
                 info.sector_dims[2]);
    return d;
  }
  Dimensions getSectorDims()
  {
    Dimensions d(sectorWidth, sectorWidth, is2DProcessing() ? 0 : sectorWidth);
    return d;
  }
  Array<IndType> getSectorCenters()
  {
    tables();
    return array_of(centers_h, info.dim * info.n_sectors);
  }
  IndType *getSectorCentersData() { return getSectorCenters().data; }
  Array<IndType> getDataIndices()
  {
    tables();
    return array_of(di_h, info.n_samples);
  }
  bool is2DProcessing() { return imgDims.depth == 0; }
  bool is3DProcessing() { return !is2DProcessing(); }
  int getImageDimensionCount() { return is2DProcessing() ? 2 : 3; }

  // ------------------------------------------------------------- operations
  /* Adjoint, host arrays; the result is allocated with calloc (free() it):
   * the image after deapodization (coil-combined with maps). */
  Array<CufftType> performGpuNUFFTAdj(Array<DType2> kspaceData)
  {
    return performGpuNUFFTAdj(kspaceData, DEAPODIZATION);
  }

  virtual void performGpuNUFFTAdj(Array<DType2> kspaceData,
                                  Array<CufftType> &imgData,
                                  GpuNUFFTOutput gpuNUFFTOut = DEAPODIZATION)
  {
    detail::check(gnufft_adjoint_host(plan, kspaceData.data, imgData.data,
                                      DEFAULT_VALUE(kspaceData.dim.channels),
                                      (int32_t)gpuNUFFTOut));
  }

  /* Device arrays, ordered on the legacy default stream. */
  virtual void performGpuNUFFTAdj(GpuArray<DType2> kspaceData_gpu,
                                  GpuArray<CufftType> &imgData_gpu,
                                  GpuNUFFTOutput gpuNUFFTOut = DEAPODIZATION)
  {
    detail::check(gnufft_adjoint_device(
        plan, kspaceData_gpu.data, imgData_gpu.data,
        DEFAULT_VALUE(kspaceData_gpu.dim.channels), (int32_t)gpuNUFFTOut,
        NULL));
  }

  /* Adjoint to the given stage; the result is allocated with calloc:
   * CONVOLUTION / DENSITY_ESTIMATION the grid per coil, otherwise the
   * image (one channel with maps). */
  Array<CufftType> performGpuNUFFTAdj(Array<DType2> kspaceData,
                                      GpuNUFFTOutput gpuNUFFTOut)
  {
    Array<CufftType> img;
    if (gpuNUFFTOut == CONVOLUTION || gpuNUFFTOut == DENSITY_ESTIMATION)
    {
      img.dim = getGridDims();
      img.dim.channels = kspaceData.dim.channels;
    }
    else
    {
      img.dim = getImageDims();
      img.dim.channels = applySensData() ? 1 : kspaceData.dim.channels;
    }
    img.data = (CufftType *)std::calloc(img.count(), sizeof(CufftType));
    if (!img.data)
      throw std::runtime_error("gpuNUFFT: host allocation failed");
    try
    {
      performGpuNUFFTAdj(kspaceData, img, gpuNUFFTOut);
    }
    catch (...)
    {
      std::free(img.data);
      throw;
    }
    return img;
  }

  /* Forward, host arrays; the result is allocated with calloc.  The
   * one-argument form runs the whole forward, like the upstream (whose
   * default output stage CONVOLUTION does not stop a forward early). */
  Array<CufftType> performForwardGpuNUFFT(Array<DType2> imgData)
  {
    return performForwardGpuNUFFT(imgData, CONVOLUTION);
  }

  virtual void
  performForwardGpuNUFFT(Array<DType2> imgData, Array<CufftType> &kspaceData,
                         GpuNUFFTOutput gpuNUFFTOut = DEAPODIZATION)
  {
    detail::check(gnufft_forward_host(
        plan, imgData.data, kspaceData.data,
        DEFAULT_VALUE(kspaceData.dim.channels), forward_stage(gpuNUFFTOut)));
  }

  virtual void
  performForwardGpuNUFFT(GpuArray<DType2> imgData_gpu,
                         GpuArray<CufftType> &kspaceData_gpu,
                         GpuNUFFTOutput gpuNUFFTOut = DEAPODIZATION)
  {
    detail::check(gnufft_forward_device(
        plan, imgData_gpu.data, kspaceData_gpu.data,
        DEFAULT_VALUE(kspaceData_gpu.dim.channels),
        forward_stage(gpuNUFFTOut), NULL));
  }

  Array<CufftType> performForwardGpuNUFFT(Array<DType2> imgData,
                                          GpuNUFFTOutput gpuNUFFTOut)
  {
    Array<CufftType> k;
    k.dim = kSpaceDim;
    k.dim.channels =
        applySensData() ? sens.dim.channels : imgData.dim.channels;
    k.data = (CufftType *)std::calloc(k.count(), sizeof(CufftType));
    if (!k.data)
      throw std::runtime_error("gpuNUFFT: host allocation failed");
    try
    {
      performForwardGpuNUFFT(imgData, k, gpuNUFFTOut);
    }
    catch (...)
    {
      std::free(k.data);
      throw;
    }
    return k;
  }

  bool applyDensComp() { return info.has_dens != 0 && info.n_samples > 1; }
  bool applySensData() { return sens.data != NULL && sens.count() > 1; }
  virtual OperatorType getType() { return operatorType; }

  /* The C-ABI plan behind this operator (for mixing with the C API). */
  gnufft_plan *getPlan() { return plan; }

 protected:
  GpuNUFFTOperator(OperatorType type, IndType kw, IndType sw, DType osf_,
                   Dimensions img, bool shared)
    : operatorType(type), osf(osf_), kernelWidth(kw), sectorWidth(sw),
      imgDims(img), matlabSharedMem(shared), plan(NULL), have_tables(false)
  {
    std::memset(&info, 0, sizeof(info));
  }

  /* the forward has no early stop except DENSITY_ESTIMATION */
  static int32_t forward_stage(GpuNUFFTOutput o)
  {
    return o == DENSITY_ESTIMATION ? (int32_t)DENSITY_ESTIMATION
                                   : (int32_t)DEAPODIZATION;
  }

  void attach(gnufft_plan *p)
  {
    plan = p;
    detail::check(gnufft_plan_get_info(plan, &info));
    kSpaceDim = Dimensions();
    kSpaceDim.length = info.n_samples;
  }

  template <typename T>
  static Array<T> array_of(std::vector<T> &v, size_t n)
  {
    Array<T> a;
    a.data = n ? v.data() : NULL;
    a.dim.length = (IndType)n;
    return a;
  }

  /* host copies of the plan's tables, made on first use */
  void tables()
  {
    if (have_tables)
      return;
    traj_h.resize((size_t)info.dim * info.n_samples);
    di_h.resize(info.n_samples);
    sdc_h.resize((size_t)info.n_sectors + 1);
    order_h.resize(2 * (size_t)info.n_processing_order);
    centers_h.resize((size_t)info.dim * info.n_sectors);
    dens_h.resize(info.has_dens ? info.n_samples : 0);
    lut_h.resize(info.kernel_lut_len);
    detail::check(gnufft_export_tables(
        plan, traj_h.data(), di_h.data(), sdc_h.data(),
        order_h.empty() ? NULL : order_h.data(), centers_h.data(),
        dens_h.empty() ? NULL : dens_h.data(), NULL, lut_h.data()));
    have_tables = true;
  }

  OperatorType operatorType;
  DType osf;
  IndType kernelWidth;
  IndType sectorWidth;
  Dimensions imgDims;
  Dimensions kSpaceDim;
  bool matlabSharedMem;
  gnufft_plan *plan;
  gnufft_plan_info info;
  Array<DType2> sens;
  std::vector<void *> owned;  // precomputed arrays handed over at load
  bool have_tables;
  std::vector<DType> traj_h, dens_h, lut_h;
  std::vector<IndType> di_h, sdc_h, order_h, centers_h;
};

/* Processing-order access of the balanced operators
 * (balanced_operator.hpp:13-20). */
class BalancedOperator
{
 public:
  virtual ~BalancedOperator() {}
  virtual Array<IndType2> getSectorProcessingOrder() = 0;
  virtual void setSectorProcessingOrder(Array<IndType2> order) = 0;
};

class BalancedGpuNUFFTOperator : public GpuNUFFTOperator,
                                 public BalancedOperator
{
 public:
  /* (sector, first sample) pairs, sectors by descending sample count */
  Array<IndType2> getSectorProcessingOrder()
  {
    tables();
    Array<IndType2> a;
    a.data = order_h.empty() ? NULL
                             : reinterpret_cast<IndType2 *>(order_h.data());
    a.dim.length = info.n_processing_order;
    return a;
  }
  void setSectorProcessingOrder(Array<IndType2>)
  {
    detail::fixed("the sector processing order");
  }
  OperatorType getType() { return BALANCED; }
  friend class GpuNUFFTOperatorFactory;

 protected:
  BalancedGpuNUFFTOperator(IndType kw, IndType sw, DType osf_, Dimensions img,
                           bool shared)
    : GpuNUFFTOperator(BALANCED, kw, sw, osf_, img, shared)
  {
  }
};

class TextureGpuNUFFTOperator : public GpuNUFFTOperator
{
 public:
  OperatorType getType() { return TEXTURE; }
  friend class GpuNUFFTOperatorFactory;

 protected:
  TextureGpuNUFFTOperator(OperatorType type, IndType kw, IndType sw,
                          DType osf_, Dimensions img, bool shared)
    : GpuNUFFTOperator(type, kw, sw, osf_, img, shared)
  {
  }
};

class BalancedTextureGpuNUFFTOperator : public TextureGpuNUFFTOperator,
                                        public BalancedOperator
{
 public:
  Array<IndType2> getSectorProcessingOrder()
  {
    tables();
    Array<IndType2> a;
    a.data = order_h.empty() ? NULL
                             : reinterpret_cast<IndType2 *>(order_h.data());
    a.dim.length = info.n_processing_order;
    return a;
  }
  void setSectorProcessingOrder(Array<IndType2>)
  {
    detail::fixed("the sector processing order");
  }
  OperatorType getType() { return BALANCED_TEXTURE; }
  friend class GpuNUFFTOperatorFactory;

 protected:
  BalancedTextureGpuNUFFTOperator(IndType kw, IndType sw, DType osf_,
                                  Dimensions img, bool shared)
    : TextureGpuNUFFTOperator(BALANCED_TEXTURE, kw, sw, osf_, img, shared)
  {
  }
};

}  // namespace gpuNUFFT

#endif  // GPUNUFFT_OPERATOR_H_INCLUDED
