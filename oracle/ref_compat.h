/*
 * Build-compatibility header used ONLY to compile the upstream gpuNUFFT
 * sources (where they lie, unmodified) into the test oracle under
 * oracle/_ref/.  It is force-included (-include) ahead of every upstream
 * translation unit.  Nothing in the product includes it.
 *
 * CUDA 12 removed legacy texture references (texture<>, tex1Dfetch / tex2D
 * on a texture reference, cudaBindTexture, cudaBindTextureToArray,
 * cudaUnbindTexture).  The upstream declares five of them in cuda_utils.cuh
 * (texKERNEL, texKERNEL2D, texKERNEL3D, texDATA, texGDATA) and its TEXTURE
 * and BALANCED_TEXTURE operators read the kernel lookup table through
 * texKERNEL2D (linear filtering, normalised coordinates, clamp:
 * std_gpuNUFFT_kernels.cu:49-60) and the k-space / grid through texDATA /
 * texGDATA (linear memory, point fetches: :24-34).  This header re-creates
 * that behaviour with texture OBJECTS, which the hardware filters exactly
 * like the legacy references it replaces:
 *
 *  - `texture<T, dim, mode> name;` becomes a host-side state object (the
 *    macro below), and each of the five names gets a `__constant__`
 *    cudaTextureObject_t handle `name##_compat_obj` in the translation unit;
 *  - cudaBindTexture / cudaBindTextureToArray create a texture object for
 *    the bound memory with the reference's current attributes and store it
 *    in the handle; assigning filterMode / normalized / addressMode (the
 *    upstream does so right after binding, relying on the legacy rule that
 *    attributes are read at launch) re-creates the object;
 *  - tex1Dfetch / tex1D / tex2D / tex3D on a reference fetch through its
 *    handle (float2 for the two linear-memory references, float for the
 *    lookup-table arrays, the only types the upstream declares).
 *
 * The handles are file-static: the upstream binds and launches from the
 * same translation unit (atomic_gpuNUFFT.cu includes std_gpuNUFFT_kernels.cu
 * and both kernel files), and the other unit that includes cuda_utils.cuh
 * (precomp_kernels.cu) never touches textures.
 */
#ifndef GNUFFT_REF_COMPAT_H
#define GNUFFT_REF_COMPAT_H

#include <cuda_runtime.h>
#include <cufft.h>
#include <math.h>
#include <string.h>

namespace gnufft_ref_compat
{
struct tex_base;

/* An attribute the upstream assigns after binding: the assignment
 * re-creates the bound texture object. */
template <class V> struct attr
{
  V v;
  tex_base *owner;
  attr &operator=(V x);
  operator V() const { return v; }
};

struct tex_base
{
  attr<int> normalized;
  attr<cudaTextureFilterMode> filterMode;
  attr<cudaTextureAddressMode> addressMode[3];
  cudaChannelFormatDesc channelDesc;
  /* bound resource */
  bool bound;
  cudaResourceDesc res;
  const void *symbol; /* host shadow of the __constant__ handle */
  cudaTextureObject_t obj;

  explicit tex_base(cudaChannelFormatDesc d)
  {
    normalized.v = 0;
    filterMode.v = cudaFilterModePoint;
    for (int i = 0; i < 3; ++i)
    {
      addressMode[i].v = cudaAddressModeClamp;
      addressMode[i].owner = this;
    }
    normalized.owner = this;
    filterMode.owner = this;
    channelDesc = d;
    bound = false;
    memset(&res, 0, sizeof(res));
    symbol = 0;
    obj = 0;
  }

  void release()
  {
    if (obj)
      cudaDestroyTextureObject(obj);
    obj = 0;
  }

  cudaError_t rebuild()
  {
    if (!bound)
      return cudaSuccess;
    release();
    cudaTextureDesc td;
    memset(&td, 0, sizeof(td));
    for (int i = 0; i < 3; ++i)
      td.addressMode[i] = addressMode[i].v;
    td.filterMode = filterMode.v;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = normalized.v;
    cudaError_t e = cudaCreateTextureObject(&obj, &res, &td, 0);
    if (e != cudaSuccess)
      return e;
    return cudaMemcpyToSymbol(symbol, &obj, sizeof(obj));
  }
};

template <class V> attr<V> &attr<V>::operator=(V x)
{
  v = x;
  if (owner)
    owner->rebuild();
  return *this;
}

template <class T, int dim = 1,
          enum cudaTextureReadMode mode = cudaReadModeElementType>
struct legacy_texture : tex_base
{
  legacy_texture() : tex_base(cudaCreateChannelDesc<T>()) {}
};

inline cudaError_t bind_linear(tex_base &t, const void *symbol,
                               const void *ptr, size_t bytes)
{
  t.release();
  memset(&t.res, 0, sizeof(t.res));
  t.res.resType = cudaResourceTypeLinear;
  t.res.res.linear.devPtr = const_cast<void *>(ptr);
  t.res.res.linear.desc = t.channelDesc;
  t.res.res.linear.sizeInBytes = bytes;
  t.symbol = symbol;
  t.bound = true;
  return t.rebuild();
}

inline cudaError_t bind_array(tex_base &t, const void *symbol,
                              cudaArray_const_t a)
{
  t.release();
  memset(&t.res, 0, sizeof(t.res));
  t.res.resType = cudaResourceTypeArray;
  t.res.res.array.array = const_cast<cudaArray_t>(a);
  t.symbol = symbol;
  t.bound = true;
  return t.rebuild();
}

inline cudaError_t unbind(tex_base &t, const void *symbol)
{
  t.release();
  t.bound = false;
  cudaTextureObject_t zero = 0;
  return cudaMemcpyToSymbol(symbol, &zero, sizeof(zero));
}
}  // namespace gnufft_ref_compat

/* handles of the five upstream texture references (cuda_utils.cuh:10-15) */
static __constant__ cudaTextureObject_t texKERNEL_compat_obj;
static __constant__ cudaTextureObject_t texKERNEL2D_compat_obj;
static __constant__ cudaTextureObject_t texKERNEL3D_compat_obj;
static __constant__ cudaTextureObject_t texDATA_compat_obj;
static __constant__ cudaTextureObject_t texGDATA_compat_obj;

// Upstream declares `texture<float, 1, cudaReadModeElementType> texKERNEL;`
#define texture static ::gnufft_ref_compat::legacy_texture

#define cudaBindTexture(offset, t, ptr, bytes)                               \
  ::gnufft_ref_compat::bind_linear(t, &t##_compat_obj, ptr, bytes)
#define cudaBindTextureToArray(t, a)                                         \
  ::gnufft_ref_compat::bind_array(t, &t##_compat_obj, a)
#define cudaUnbindTexture(t) ::gnufft_ref_compat::unbind(t, &t##_compat_obj)

#define tex1Dfetch(t, i) tex1Dfetch<float2>(t##_compat_obj, (int)(i))
#define tex1D(t, x) tex1D<float>(t##_compat_obj, (float)(x))
#define tex2D(t, x, y) tex2D<float>(t##_compat_obj, (float)(x), (float)(y))
#define tex3D(t, x, y, z)                                                    \
  tex3D<float>(t##_compat_obj, (float)(x), (float)(y), (float)(z))

#endif
