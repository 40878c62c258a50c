/*
 * gpuNUFFT::GpuNUFFTOperatorFactory for the gpunufft_b200 drop-in:
 * header-only, over the C ABI in gpunufft_b200.h.
 *
 * Signatures follow the upstream's gpuNUFFT_operator_factory.hpp:58-172
 * (andyschwarzl/gpuNUFFT, CUDA/inc): createGpuNUFFTOperator with and without
 * density compensation and sensitivity maps, loadPrecomputedGpuNUFFTOperator
 * (the MATLAB 7-array contract), setUseTextures / setBalanceWorkload.  The
 * factory returns a new operator that the caller deletes.  The operator
 * type follows the factory flags as upstream (textures -> TEXTURE /
 * BALANCED_TEXTURE, balancing -> BALANCED / BALANCED_TEXTURE).  useGpu
 * selected where the upstream computes its sector tables; they are
 * computed on the GPU here and are identical either way.
 *
 * Ownership as upstream: arrays handed to createGpuNUFFTOperator stay the
 * caller's (the operator keeps copies; the maps are copied as well); the
 * arrays handed to loadPrecomputedGpuNUFFTOperator are released with
 * free() when the operator is deleted, unless the factory was made with
 * matlabSharedMem = true.  Density weights and maps of at most one element
 * are ignored, as the upstream's applyDensComp / applySensData do.
 */
#ifndef GPUNUFFT_OPERATOR_FACTORY_H_INCLUDED
#define GPUNUFFT_OPERATOR_FACTORY_H_INCLUDED

#include "gpuNUFFT_operator.hpp"

namespace gpuNUFFT
{

class GpuNUFFTOperatorFactory
{
 public:
  GpuNUFFTOperatorFactory(const bool useTextures = true,
                          const bool useGpu = true,
                          bool balanceWorkload = true,
                          bool matlabSharedMem = false)
    : useTextures(useTextures), useGpu(useGpu),
      balanceWorkload(balanceWorkload), matlabSharedMem(matlabSharedMem),
      device(0)
  {
  }

  ~GpuNUFFTOperatorFactory() {}

  GpuNUFFTOperator *createGpuNUFFTOperator(Array<DType> &kSpaceTraj,
                                           const IndType &kernelWidth,
                                           const IndType &sectorWidth,
                                           const DType &osf,
                                           Dimensions &imgDims)
  {
    Array<DType> noDens;
    Array<DType2> noSens;
    return createGpuNUFFTOperator(kSpaceTraj, noDens, noSens, kernelWidth,
                                  sectorWidth, osf, imgDims);
  }

  GpuNUFFTOperator *
  createGpuNUFFTOperator(Array<DType> &kSpaceTraj, Array<DType> &densCompData,
                         const IndType &kernelWidth, const IndType &sectorWidth,
                         const DType &osf, Dimensions &imgDims)
  {
    Array<DType2> noSens;
    return createGpuNUFFTOperator(kSpaceTraj, densCompData, noSens,
                                  kernelWidth, sectorWidth, osf, imgDims);
  }

  GpuNUFFTOperator *
  createGpuNUFFTOperator(Array<DType> &kSpaceTraj, Array<DType> &densCompData,
                         Array<DType2> &sensData, const IndType &kernelWidth,
                         const IndType &sectorWidth, const DType &osf,
                         Dimensions &imgDims)
  {
    if (!kSpaceTraj.data)
      throw std::invalid_argument("gpuNUFFT: trajectory is empty");
    gnufft_desc d = desc(kSpaceTraj.count(), kernelWidth, sectorWidth, osf,
                         imgDims, sensData);
    GpuNUFFTOperator *op = make(kernelWidth, sectorWidth, osf, imgDims);
    gnufft_plan *p = NULL;
    const gnufft_status st = gnufft_plan_create(
        &d, kSpaceTraj.data, dens_of(densCompData),
        d.n_coils ? sensData.data : NULL, &p);
    return finish(op, st, p, sensData);
  }

  /* The MATLAB precomputation contract: sector-sorted trajectory, data
   * indices, sector data count, processing order, sector centers, sorted
   * density weights, maps and deapodization function. */
  GpuNUFFTOperator *loadPrecomputedGpuNUFFTOperator(
      Array<DType> &kSpaceTraj, Array<IndType> &dataIndices,
      Array<IndType> &sectorDataCount, Array<IndType2> &sectorProcessingOrder,
      Array<IndType> &sectorCenters, Array<DType> &densCompData,
      Array<DType2> &sensData, Array<DType> &deapoData,
      const IndType &kernelWidth, const IndType &sectorWidth,
      const DType &osf, Dimensions &imgDims)
  {
    if (!kSpaceTraj.data || !dataIndices.data || !sectorDataCount.data ||
        !sectorCenters.data || !deapoData.data)
      throw std::invalid_argument("gpuNUFFT: precomputed table is empty");
    gnufft_desc d = desc(dataIndices.count(), kernelWidth, sectorWidth, osf,
                         imgDims, sensData);
    GpuNUFFTOperator *op = make(kernelWidth, sectorWidth, osf, imgDims);
    gnufft_plan *p = NULL;
    const gnufft_status st = gnufft_plan_load(
        &d, kSpaceTraj.data, dataIndices.data, sectorDataCount.data,
        reinterpret_cast<const uint32_t *>(sectorProcessingOrder.data),
        sectorProcessingOrder.data ? sectorProcessingOrder.count() : 0u,
        sectorCenters.data, dens_of(densCompData),
        d.n_coils ? sensData.data : NULL, deapoData.data, &p);
    op = finish(op, st, p, sensData);
    void *handed[] = {kSpaceTraj.data,   dataIndices.data,
                      sectorDataCount.data, sectorProcessingOrder.data,
                      sectorCenters.data, densCompData.data, deapoData.data};
    for (void *h : handed)
      if (h)
        op->owned.push_back(h);
    return op;
  }

  GpuNUFFTOperator *loadPrecomputedGpuNUFFTOperator(
      Array<DType> &kSpaceTraj, Array<IndType> &dataIndices,
      Array<IndType> &sectorDataCount, Array<IndType2> &sectorProcessingOrder,
      Array<IndType> &sectorCenters, Array<DType2> &sensData,
      Array<DType> &deapoData, const IndType &kernelWidth,
      const IndType &sectorWidth, const DType &osf, Dimensions &imgDims)
  {
    Array<DType> noDens;
    return loadPrecomputedGpuNUFFTOperator(
        kSpaceTraj, dataIndices, sectorDataCount, sectorProcessingOrder,
        sectorCenters, noDens, sensData, deapoData, kernelWidth, sectorWidth,
        osf, imgDims);
  }

  void setUseTextures(bool t) { useTextures = t; }
  void setBalanceWorkload(bool b) { balanceWorkload = b; }
  /* CUDA device of the operators created from now on (default 0). */
  void setDevice(int dev) { device = dev; }

 private:
  OperatorType type() const
  {
    return useTextures ? (balanceWorkload ? BALANCED_TEXTURE : TEXTURE)
                       : (balanceWorkload ? BALANCED : DEFAULT);
  }

  GpuNUFFTOperator *make(IndType kw, IndType sw, DType osf,
                         Dimensions img) const
  {
    switch (type())
    {
    case BALANCED:
      return new BalancedGpuNUFFTOperator(kw, sw, osf, img, matlabSharedMem);
    case TEXTURE:
      return new TextureGpuNUFFTOperator(TEXTURE, kw, sw, osf, img,
                                         matlabSharedMem);
    case BALANCED_TEXTURE:
      return new BalancedTextureGpuNUFFTOperator(kw, sw, osf, img,
                                                 matlabSharedMem);
    default:
      return new GpuNUFFTOperator(DEFAULT, kw, sw, osf, img, matlabSharedMem);
    }
  }

  gnufft_desc desc(IndType n_samples, IndType kw, IndType sw, DType osf,
                   Dimensions &img, Array<DType2> &sens) const
  {
    gnufft_desc d;
    std::memset(&d, 0, sizeof(d));
    d.img_dims[0] = img.width;
    d.img_dims[1] = img.height;
    d.img_dims[2] = img.depth;
    d.n_samples = n_samples;
    d.n_coils = (sens.data && sens.count() > 1)
                    ? DEFAULT_VALUE(sens.dim.channels)
                    : 0;
    d.kernel_width = kw;
    d.sector_width = sw;
    d.osf = osf;
    d.operator_type = (int32_t)type();
    d.flags = 0;
    d.device = device;
    return d;
  }

  static const float *dens_of(Array<DType> &dens)
  {
    return (dens.data && dens.count() > 1) ? dens.data : NULL;
  }

  static GpuNUFFTOperator *finish(GpuNUFFTOperator *op, gnufft_status st,
                                  gnufft_plan *p, Array<DType2> &sens)
  {
    if (st != GNUFFT_SUCCESS)
    {
      delete op;
      detail::check(st);
    }
    try
    {
      op->attach(p);
    }
    catch (...)
    {
      gnufft_plan_destroy(p);
      op->plan = NULL;
      delete op;
      throw;
    }
    if (sens.data && sens.count() > 1)
      op->sens = sens;
    return op;
  }

  bool useTextures;
  bool useGpu;
  bool balanceWorkload;
  bool matlabSharedMem;
  int device;
};

}  // namespace gpuNUFFT

#endif  // GPUNUFFT_OPERATOR_FACTORY_H_INCLUDED
