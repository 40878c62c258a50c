// C++ caller of the gpuNUFFT operator API, written the way the upstream's
// own gtest suites call it (CUDA/test/gpu/...: GpuNUFFTOperatorFactory,
// createGpuNUFFTOperator, performGpuNUFFTAdj / performForwardGpuNUFFT with
// host Array and device GpuArray, loadPrecomputedGpuNUFFTOperator), built
// against include/ and linked with libgpunufft_b200.so (plus the CUDA
// runtime for the device buffers this caller allocates itself).
//
// Prints "<case> <values...>" lines that tests/test_gpu_cxx_shim.py checks
// against the upstream's outputs, and exits non-zero on a failed check of
// its own.  Without a CUDA device it only reports that (exit code 2).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <vector>

#include <cuda_runtime.h>

#include "gpuNUFFT_operator_factory.hpp"

namespace
{
int failures = 0;

void expect(bool ok, const char *what)
{
  if (!ok)
  {
    std::printf("FAIL %s\n", what);
    ++failures;
  }
}

int lin3(int x, int y, int z, int w) { return x + w * (y + z * w); }

// gpuNUFFT_forward_tests.cpp:167-256: 2-D 32^2, kw 5, osf 1.25, 3 samples,
// 4 coils, image of ones, all eight factory flag combinations.
void forward_2d_32_32_4()
{
  const int data_count = 3, n_coils = 4, w = 32;
  DType coords[6] = {-0.31719f, -0.38650f, 0.0f, 0.0f, 0.31719f, 0.38650f};
  // structure of arrays: x0 x1 x2 y0 y1 y2
  DType soa[6] = {coords[0], coords[2], coords[4],
                  coords[1], coords[3], coords[5]};
  gpuNUFFT::Array<DType2> img;
  img.dim.width = w;
  img.dim.height = w;
  img.dim.channels = n_coils;
  std::vector<DType2> im(img.count());
  for (auto &v : im)
    v = make_float2(1.0f, 1.0f);
  img.data = im.data();
  gpuNUFFT::Array<DType> kSpaceData;
  kSpaceData.data = soa;
  kSpaceData.dim.length = data_count;
  gpuNUFFT::Dimensions imgDims;
  imgDims.width = w;
  imgDims.height = w;
  for (int cnt = 0; cnt < 8; cnt++)
  {
    const bool useTextures = cnt & 1, useGpu = cnt & 2,
               loadBalancing = cnt & 4;
    gpuNUFFT::GpuNUFFTOperatorFactory factory(useTextures, useGpu,
                                              loadBalancing);
    gpuNUFFT::GpuNUFFTOperator *op =
        factory.createGpuNUFFTOperator(kSpaceData, 5, 8, 1.25f, imgDims);
    gpuNUFFT::Array<CufftType> k = op->performForwardGpuNUFFT(img);
    expect(k.dim.channels == (IndType)n_coils, "forward channel count");
    std::printf("forward_2d_32_32_4 %d %d", (int)op->getType(),
                (int)k.count());
    for (IndType j = 0; j < k.count(); ++j)
      std::printf(" %.9g %.9g", k.data[j].x, k.data[j].y);
    std::printf("\n");
    for (int c = 1; c < n_coils; ++c)
      expect(std::fabs(k.data[c * data_count].x - k.data[0].x) < 1e-5f,
             "coils of an image of ones agree");
    std::free(k.data);
    delete op;
  }
}

// gpuNUFFT_fft_tests.cpp:142-200: one sample at k = 0 on a 10^3 image,
// osf 1, kw 3, sw 5, adjoint to the FFT stage.
void fft_1sector()
{
  DType coords[3] = {0, 0, 0};
  DType2 data[1] = {make_float2(1, 1)};
  gpuNUFFT::Array<DType> kSpaceData;
  kSpaceData.data = coords;
  kSpaceData.dim.length = 1;
  gpuNUFFT::Dimensions imgDims(10, 10, 10);
  gpuNUFFT::GpuNUFFTOperatorFactory factory(false, true, true);
  gpuNUFFT::GpuNUFFTOperator *op =
      factory.createGpuNUFFTOperator(kSpaceData, 3, 5, 1.0f, imgDims);
  gpuNUFFT::Array<DType2> dataArray;
  dataArray.data = data;
  dataArray.dim.length = 1;
  gpuNUFFT::Array<CufftType> g =
      op->performGpuNUFFTAdj(dataArray, gpuNUFFT::FFT);
  expect(std::fabs(0.2172f - g.data[lin3(5, 5, 5, 10)].x) < 0.01f, ":197");
  expect(std::fabs(0.1975f - g.data[lin3(5, 4, 5, 10)].x) < 0.1f, ":198");
  expect(std::fabs(0.1975f - g.data[lin3(4, 5, 5, 10)].x) < 0.1f, ":199");
  expect(std::fabs(0.001619f - g.data[lin3(0, 1, 5, 10)].x) < 0.1f, ":200");
  std::printf("fft_1sector %.9g %.9g %.9g %.9g\n", g.data[555].x,
              g.data[lin3(5, 4, 5, 10)].x, g.data[lin3(4, 5, 5, 10)].x,
              g.data[lin3(0, 1, 5, 10)].x);
  std::free(g.data);
  delete op;
}

// gpuNUFFT_deapo_tests.cpp:342-429: 30 coils, constant maps and density,
// coil-combined adjoint has one channel.
void deapo_2d_b1()
{
  const int n_coils = 30, w = 32;
  DType coords[2] = {0, 0};
  DType dens[1] = {1};
  std::vector<DType2> data(n_coils, make_float2(1.0f, 0.5f));
  std::vector<DType2> b1((size_t)w * w * n_coils, make_float2(1.0f, 0.2f));
  gpuNUFFT::Array<DType> kSpaceData;
  kSpaceData.data = coords;
  kSpaceData.dim.length = 1;
  gpuNUFFT::Array<DType> densData;
  densData.data = dens;
  densData.dim.length = 1;
  gpuNUFFT::Dimensions imgDims;
  imgDims.width = w;
  imgDims.height = w;
  gpuNUFFT::Array<DType2> b1Data;
  b1Data.data = b1.data();
  b1Data.dim = imgDims;
  b1Data.dim.channels = n_coils;
  gpuNUFFT::GpuNUFFTOperatorFactory factory(false, true, true);
  gpuNUFFT::GpuNUFFTOperator *op = factory.createGpuNUFFTOperator(
      kSpaceData, densData, b1Data, 3, 8, 2.0f, imgDims);
  gpuNUFFT::Array<DType2> dataArray;
  dataArray.data = data.data();
  dataArray.dim.length = 1;
  dataArray.dim.channels = n_coils;
  gpuNUFFT::Array<CufftType> g =
      op->performGpuNUFFTAdj(dataArray, gpuNUFFT::DEAPODIZATION);
  expect(g.dim.channels == 1, "coil-combined adjoint has one channel");
  std::printf("deapo_2d_b1 %.9g %.9g\n", g.data[0].x, g.data[0].y);
  std::free(g.data);
  delete op;
}

// Device arrays (GpuArray overloads) equal the host-array calls, and an
// operator rebuilt from its exported tables (loadPrecomputed, arrays handed
// over and released with the operator) equals the original.
void device_and_precomputed()
{
  const int M = 2000, w = 24, C = 3;
  std::vector<DType> traj(3 * M);
  unsigned s = 12345u;
  for (auto &v : traj)
  {
    s = s * 1103515245u + 12345u;
    v = (DType)((s >> 8) & 0xFFFF) / 65536.0f - 0.5f;
  }
  gpuNUFFT::Array<DType> kSpaceData;
  kSpaceData.data = traj.data();
  kSpaceData.dim.length = M;
  gpuNUFFT::Dimensions imgDims(w, w, w);
  gpuNUFFT::GpuNUFFTOperatorFactory factory(true, true, true);
  gpuNUFFT::GpuNUFFTOperator *op =
      factory.createGpuNUFFTOperator(kSpaceData, 3, 8, 2.0f, imgDims);
  expect(op->getType() == gpuNUFFT::BALANCED_TEXTURE, "factory default type");
  std::vector<DType2> k((size_t)C * M);
  for (auto &v : k)
  {
    s = s * 1103515245u + 12345u;
    v.x = (DType)((s >> 8) & 0xFFFF) / 65536.0f - 0.5f;
    s = s * 1103515245u + 12345u;
    v.y = (DType)((s >> 8) & 0xFFFF) / 65536.0f - 0.5f;
  }
  gpuNUFFT::Array<DType2> kArr;
  kArr.data = k.data();
  kArr.dim.length = M;
  kArr.dim.channels = C;
  gpuNUFFT::Array<CufftType> host = op->performGpuNUFFTAdj(kArr);

  const size_t N = (size_t)w * w * w;
  DType2 *k_d = nullptr, *img_d = nullptr;
  if (cudaMalloc(&k_d, sizeof(DType2) * C * M) != cudaSuccess ||
      cudaMalloc(&img_d, sizeof(DType2) * C * N) != cudaSuccess)
    throw std::runtime_error("cudaMalloc failed");
  cudaMemcpy(k_d, k.data(), sizeof(DType2) * C * M, cudaMemcpyHostToDevice);
  gpuNUFFT::GpuArray<DType2> kg;
  kg.data = k_d;
  kg.dim = kArr.dim;
  gpuNUFFT::GpuArray<CufftType> ig;
  ig.data = img_d;
  ig.dim = imgDims;
  ig.dim.channels = C;
  op->performGpuNUFFTAdj(kg, ig, gpuNUFFT::DEAPODIZATION);
  std::vector<DType2> dev(C * N);
  cudaMemcpy(dev.data(), img_d, sizeof(DType2) * C * N,
             cudaMemcpyDeviceToHost);
  double num = 0, den = 0;
  for (size_t i = 0; i < C * N; ++i)
  {
    const double dx = dev[i].x - host.data[i].x, dy = dev[i].y - host.data[i].y;
    num += dx * dx + dy * dy;
    den += (double)host.data[i].x * host.data[i].x +
           (double)host.data[i].y * host.data[i].y;
  }
  expect(std::sqrt(num / den) < 1e-6, "device adjoint equals host adjoint");

  // forward on device from the host adjoint image
  cudaMemcpy(img_d, host.data, sizeof(DType2) * C * N, cudaMemcpyHostToDevice);
  gpuNUFFT::GpuArray<DType2> xg;
  xg.data = img_d;
  xg.dim = ig.dim;
  gpuNUFFT::GpuArray<CufftType> yg;
  yg.data = k_d;
  yg.dim = kArr.dim;
  op->performForwardGpuNUFFT(xg, yg);
  std::vector<DType2> ydev((size_t)C * M);
  cudaMemcpy(ydev.data(), k_d, sizeof(DType2) * C * M, cudaMemcpyDeviceToHost);
  gpuNUFFT::Array<DType2> xArr;
  xArr.data = host.data;
  xArr.dim = ig.dim;
  gpuNUFFT::Array<CufftType> yhost = op->performForwardGpuNUFFT(xArr);
  num = den = 0;
  for (size_t i = 0; i < (size_t)C * M; ++i)
  {
    const double dx = ydev[i].x - yhost.data[i].x,
                 dy = ydev[i].y - yhost.data[i].y;
    num += dx * dx + dy * dy;
    den += (double)yhost.data[i].x * yhost.data[i].x +
           (double)yhost.data[i].y * yhost.data[i].y;
  }
  expect(std::sqrt(num / den) < 1e-6, "device forward equals host forward");

  // precomputed operator from the exported tables (malloc'ed copies that
  // the new operator takes over)
  auto dup = [](const void *p, size_t bytes) {
    void *q = std::malloc(bytes ? bytes : 1);
    std::memcpy(q, p, bytes);
    return q;
  };
  gpuNUFFT::Array<DType> t = op->getKSpaceTraj();
  gpuNUFFT::Array<IndType> di = op->getDataIndices();
  gpuNUFFT::Array<IndType> sdc = op->getSectorDataCount();
  gpuNUFFT::Array<IndType> ctr = op->getSectorCenters();
  gpuNUFFT::Array<IndType2> order =
      dynamic_cast<gpuNUFFT::BalancedOperator *>(op)
          ->getSectorProcessingOrder();
  expect(order.count() > 0, "balanced operator has a processing order");
  std::vector<DType> deapo(N);
  gnufft_export_tables(op->getPlan(), nullptr, nullptr, nullptr, nullptr,
                       nullptr, nullptr, deapo.data(), nullptr);
  gpuNUFFT::Array<DType> t2;  // count() samples, one array per axis
  t2.data = (DType *)dup(t.data, sizeof(DType) * t.count() * 3);
  t2.dim = t.dim;
  gpuNUFFT::Array<IndType> di2;
  di2.data = (IndType *)dup(di.data, sizeof(IndType) * di.count());
  di2.dim = di.dim;
  gpuNUFFT::Array<IndType> sdc2;
  sdc2.data = (IndType *)dup(sdc.data, sizeof(IndType) * sdc.count());
  sdc2.dim = sdc.dim;
  gpuNUFFT::Array<IndType2> ord2;
  ord2.data = (IndType2 *)dup(order.data, sizeof(IndType2) * order.count());
  ord2.dim = order.dim;
  gpuNUFFT::Array<IndType> ctr2;
  ctr2.data = (IndType *)dup(ctr.data, sizeof(IndType) * ctr.count());
  ctr2.dim = ctr.dim;
  gpuNUFFT::Array<DType> de2;
  de2.data = (DType *)dup(deapo.data(), sizeof(DType) * N);
  de2.dim = imgDims;
  gpuNUFFT::Array<DType2> noSens;
  gpuNUFFT::GpuNUFFTOperator *op2 = factory.loadPrecomputedGpuNUFFTOperator(
      t2, di2, sdc2, ord2, ctr2, noSens, de2, 3, 8, 2.0f, imgDims);
  gpuNUFFT::Array<CufftType> again = op2->performGpuNUFFTAdj(kArr);
  bool same = true;
  for (size_t i = 0; i < C * N; ++i)
    same = same && again.data[i].x == host.data[i].x &&
           again.data[i].y == host.data[i].y;
  expect(same, "precomputed operator equals the original");
  std::printf("device_and_precomputed ok\n");
  std::free(again.data);
  std::free(yhost.data);
  std::free(host.data);
  cudaFree(k_d);
  cudaFree(img_d);
  delete op2;  // releases t2, di2, sdc2, ord2, ctr2, de2
  delete op;
}

// Errors are exceptions (the upstream factory throws invalid_argument).
void errors()
{
  DType coords[2] = {0, 0};
  gpuNUFFT::Array<DType> kSpaceData;
  kSpaceData.data = coords;
  kSpaceData.dim.length = 1;
  gpuNUFFT::Dimensions imgDims(16, 16);
  gpuNUFFT::GpuNUFFTOperatorFactory factory(false, true, true);
  bool thrown = false;
  try
  {
    delete factory.createGpuNUFFTOperator(kSpaceData, 0, 8, 2.0f, imgDims);
  }
  catch (const std::invalid_argument &)
  {
    thrown = true;
  }
  expect(thrown, "kernel width 0 is rejected with invalid_argument");
  gpuNUFFT::GpuNUFFTOperator *op =
      factory.createGpuNUFFTOperator(kSpaceData, 3, 8, 2.0f, imgDims);
  thrown = false;
  try
  {
    op->setOsf(1.5f);
  }
  catch (const std::logic_error &)
  {
    thrown = true;
  }
  expect(thrown, "geometry setters throw");
  delete op;
  std::printf("errors ok\n");
}
}  // namespace

int main()
{
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0)
  {
    std::printf("no CUDA device\n");
    return 2;
  }
  try
  {
    forward_2d_32_32_4();
    fft_1sector();
    deapo_2d_b1();
    device_and_precomputed();
    errors();
  }
  catch (const std::exception &e)
  {
    std::printf("FAIL exception: %s\n", e.what());
    return 1;
  }
  std::printf("failures %d\n", failures);
  return failures ? 1 : 0;
}
