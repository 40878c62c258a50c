/*
 * Build-compatibility header used ONLY to compile the upstream gpuNUFFT
 * sources (where they lie, unmodified) into the test oracle under
 * oracle/_ref/.  It is force-included (-include) ahead of every upstream
 * translation unit.  Nothing in the product includes it.
 *
 * CUDA 12 removed legacy texture references (texture<>, tex1Dfetch on a
 * texture reference, cudaBindTexture, ...).  The upstream DEFAULT and
 * BALANCED operators never touch them, but every upstream .cu file includes
 * cuda_utils.cuh, which declares them.  This header supplies inert
 * stand-ins so those translation units compile; the TEXTURE and
 * BALANCED_TEXTURE operators built from them are NOT functional and the
 * oracle harness never constructs them (it always passes
 * useTextures=false to the upstream factory).
 *
 * The stand-in texture objects get internal linkage (the macro below turns
 * the upstream `texture<...> name;` definitions into `static ...`), so the
 * two upstream translation units that both include cuda_utils.cuh link.
 */
#ifndef GNUFFT_REF_COMPAT_H
#define GNUFFT_REF_COMPAT_H

#include <cuda_runtime.h>
#include <cufft.h>
#include <math.h>

namespace gnufft_ref_compat
{
template <class T, int dim = 1,
          enum cudaTextureReadMode mode = cudaReadModeElementType>
struct legacy_texture
{
  int normalized;
  enum cudaTextureFilterMode filterMode;
  enum cudaTextureAddressMode addressMode[3];
  struct cudaChannelFormatDesc channelDesc;
};

template <class T> __host__ __device__ inline T poison()
{
  T v;
  float *f = reinterpret_cast<float *>(&v);
  for (unsigned i = 0; i < sizeof(T) / sizeof(float); ++i)
    f[i] = nanf("");
  return v;
}
}  // namespace gnufft_ref_compat

// Upstream declares `texture<float, 1, cudaReadModeElementType> texKERNEL;`
#define texture static ::gnufft_ref_compat::legacy_texture

// Device-side fetches from the stand-in textures: never executed by the
// oracle (texture operators are never constructed); they yield NaN so any
// accidental use is loud.  Macros, because the stand-in objects are host
// variables and may not be named in device code.
#define tex1Dfetch(t, i) (::gnufft_ref_compat::poison<float2>())
#define tex1D(t, x) (::gnufft_ref_compat::poison<float>())
#define tex2D(t, x, y) (::gnufft_ref_compat::poison<float>())
#define tex3D(t, x, y, z) (::gnufft_ref_compat::poison<float>())

template <class T, int d, enum cudaTextureReadMode m>
inline cudaError_t cudaBindTexture(size_t *,
                                   gnufft_ref_compat::legacy_texture<T, d, m> &,
                                   const void *, size_t)
{
  return cudaErrorNotSupported;
}
template <class T, int d, enum cudaTextureReadMode m>
inline cudaError_t
cudaBindTextureToArray(gnufft_ref_compat::legacy_texture<T, d, m> &,
                       cudaArray_const_t)
{
  return cudaErrorNotSupported;
}
template <class T, int d, enum cudaTextureReadMode m>
inline cudaError_t
cudaUnbindTexture(gnufft_ref_compat::legacy_texture<T, d, m> &)
{
  return cudaSuccess;
}

#endif
