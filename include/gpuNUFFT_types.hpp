/*
 * gpuNUFFT C++ API types for the gpunufft_b200 drop-in (header-only shim
 * over the C ABI in gpunufft_b200.h).
 *
 * Same names, members and semantics as the upstream's gpuNUFFT_types.hpp
 * (andyschwarzl/gpuNUFFT, CUDA/inc/gpuNUFFT_types.hpp:25-214) and the
 * scalar types of its single-precision config.hpp (DType = float, DType2 =
 * float2, CufftType = cufftComplex, IndType = unsigned int, IndType2 =
 * uint2), so that C++ code written against the upstream headers compiles
 * unchanged against this directory.  The structs are plain data; no CUDA
 * library is needed to use them (only the CUDA vector types).
 */
#ifndef GPUNUFFT_TYPES_H_INCLUDED
#define GPUNUFFT_TYPES_H_INCLUDED

#include <cstddef>
#include <cstdlib>
#include <utility>

#include <vector_types.h>

typedef float DType;
typedef float2 DType2;
typedef float3 DType3;
typedef float2 CufftType;  // layout of cufftComplex
typedef unsigned int SizeType;
typedef unsigned int IndType;
typedef uint2 IndType2;
typedef uint3 IndType3;

/* upstream gpuNUFFT_types.hpp:16 */
#define DEFAULT_VALUE(a) ((a == 0) ? 1 : a)
/* samples per work item of the balanced operators (gpuNUFFT_types.hpp:23) */
#define MAXIMUM_PAYLOAD 256

namespace gpuNUFFT
{

/* (index, sector) pair ordered by the sector (gpuNUFFT_types.hpp:33-49). */
struct IndPair : std::pair<IndType, IndType>
{
  IndPair(IndType first, IndType second)
    : std::pair<IndType, IndType>(first, second)
  {
  }
  bool operator<(const IndPair &o) const { return second < o.second; }
  bool operator>(const IndPair &o) const { return second > o.second; }
};

/* Array extents (gpuNUFFT_types.hpp:69-140): zero extents count as one. */
struct Dimensions
{
  Dimensions()
    : width(0), height(0), depth(0), channels(1), frames(1), length(0)
  {
  }
  Dimensions(IndType w, IndType h, IndType d)
    : width(w), height(h), depth(d), channels(1), frames(1), length(0)
  {
  }
  Dimensions(IndType w, IndType h)
    : width(w), height(h), depth(0), channels(1), frames(1), length(0)
  {
  }

  IndType width;
  IndType height;
  IndType depth;
  IndType channels;
  IndType frames;
  IndType length;  // 1-D arrays

  IndType count()
  {
    return DEFAULT_VALUE(length) * DEFAULT_VALUE(width) *
           DEFAULT_VALUE(height) * DEFAULT_VALUE(depth) *
           DEFAULT_VALUE(channels) * DEFAULT_VALUE(frames);
  }

  /* extents scaled (and truncated) by alpha, e.g. image -> grid */
  Dimensions operator*(const DType alpha)
  {
    Dimensions r;
    r.width = (IndType)(width * alpha);
    r.height = (IndType)(height * alpha);
    r.depth = (IndType)(depth * alpha);
    r.length = (IndType)(length * alpha);
    return r;
  }

  /* non-zero extents grown by alpha */
  Dimensions operator+(const IndType alpha)
  {
    Dimensions r;
    if (width > 0)
      r.width = width + alpha;
    if (height > 0)
      r.height = height + alpha;
    if (depth > 0)
      r.depth = depth + alpha;
    if (length > 0)
      r.length = length + alpha;
    return r;
  }
};

/* Non-owning host array with its extents (gpuNUFFT_types.hpp:142-157). */
template <typename T> struct Array
{
  Array() : data(NULL) {}
  T *data;
  Dimensions dim;
  IndType count() { return dim.count(); }
};

/* The same over device memory (gpuNUFFT_types.hpp:159-164). */
template <typename T> struct GpuArray : Array<T>
{
};

/* gpuNUFFT_types.hpp:166-181 */
enum InterpolationType
{
  CONST_LOOKUP,
  TEXTURE_LOOKUP,
  TEXTURE2D_LOOKUP,
  TEXTURE3D_LOOKUP
};

/* Last stage of a call (gpuNUFFT_types.hpp:183-193). */
enum GpuNUFFTOutput
{
  CONVOLUTION,
  FFT,
  DEAPODIZATION,
  DENSITY_ESTIMATION,
};

/* gpuNUFFT_types.hpp:195-200 */
enum FFTShiftDir
{
  FORWARD,
  INVERSE
};

/* gpuNUFFT_types.hpp:202-214 */
enum OperatorType
{
  DEFAULT,
  TEXTURE,
  BALANCED,
  BALANCED_TEXTURE
};

}  // namespace gpuNUFFT

#endif  // GPUNUFFT_TYPES_H_INCLUDED
