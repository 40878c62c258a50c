#!/usr/bin/env bash
# Builds the upstream gpuNUFFT library from its own, unmodified sources
# (read where they lie under the upstream tree) into oracle/_ref/ as a test
# oracle.  Output: oracle/_ref/libgnufft_ref.so (upstream host code + the
# upstream DEFAULT/BALANCED CUDA kernels for sm_100a + oracle/ref_harness.cpp).
#
# Not the upstream build system: the upstream CMake targets sm_50..sm_75 and
# generates config.hpp / cufft_config.hpp from *.cmake templates.  This
# recipe writes those two configuration headers itself (float precision,
# DEBUG=false, the values the upstream Release build uses) and force-includes
# oracle/ref_compat.h into the upstream .cu files so they compile under
# CUDA 12 (legacy texture references were removed; see that header).
#
# Usage: oracle/build_ref.sh [UPSTREAM_ROOT]
#   UPSTREAM_ROOT defaults to $GNUFFT_UPSTREAM_ROOT, else to a checkout named
#   "reference" next to this repository.
set -euo pipefail
HERE="$(cd "$(dirname "$0")" && pwd)"
DEFAULT_UP="${GNUFFT_UPSTREAM_ROOT:-$(cd "$HERE/../.." && pwd)/reference}"
UP="${1:-$DEFAULT_UP}/CUDA"
OUT="$HERE/_ref"
if [ ! -d "$UP/src" ]; then
  echo "upstream sources not found at $UP" >&2
  exit 2
fi
CUDA_HOME="${CUDA_HOME:-/usr/local/cuda}"
NVCC="$CUDA_HOME/bin/nvcc"
mkdir -p "$OUT/include" "$OUT/obj"

cat > "$OUT/include/config.hpp" <<'H'
/* written by oracle/build_ref.sh: upstream single-precision configuration */
#ifndef CONFIG_H
#define CONFIG_H
#include "cufft.h"
#define MATLAB_DEBUG false
#define DEBUG false
typedef float DType;
typedef float2 DType2;
typedef float3 DType3;
typedef cufftComplex CufftType;
typedef unsigned int SizeType;
typedef unsigned int IndType;
typedef uint2 IndType2;
typedef uint3 IndType3;
#endif
H
cat > "$OUT/include/cufft_config.hpp" <<'H'
/* written by oracle/build_ref.sh: single-precision C2C */
#ifndef CUFFT_CONFIG_H
#define CUFFT_CONFIG_H
#include "config.hpp"
#include "cufft.h"
static cufftType_t CufftTransformType = CUFFT_C2C;
static cufftResult (*pt2CufftExec)(cufftHandle, cufftComplex *, cufftComplex *,
                                   int) = &cufftExecC2C;
#endif
H

INC=(-I"$OUT/include" -I"$UP/inc" -I"$CUDA_HOME/include")
GEN=(-gencode arch=compute_100a,code=sm_100a)
CXXFLAGS=(-O2 -fPIC -std=c++14 -w)

objs=()
for cu in "$UP/src/gpu/atomic/atomic_gpuNUFFT.cu" "$UP/src/gpu/precomp_kernels.cu"; do
  o="$OUT/obj/$(basename "$cu" .cu).o"
  "$NVCC" "${GEN[@]}" -O2 -std=c++14 -w -Xcompiler -fPIC -include "$HERE/ref_compat.h" \
    "${INC[@]}" -I"$UP/src/gpu" -c "$cu" -o "$o"
  objs+=("$o")
done
for cpp in "$UP/src/gpuNUFFT_utils.cpp" "$UP/src/gpuNUFFT_operator_factory.cpp" \
           "$UP/src/gpuNUFFT_operator.cpp" "$UP/src/balanced_gpuNUFFT_operator.cpp" \
           "$UP/src/texture_gpuNUFFT_operator.cpp" "$UP/src/balanced_texture_gpuNUFFT_operator.cpp" \
           "$UP/src/cpu/gpuNUFFT_cpu.cpp" "$HERE/ref_harness.cpp"; do
  o="$OUT/obj/$(basename "$cpp" .cpp).o"
  g++ "${CXXFLAGS[@]}" "${INC[@]}" -c "$cpp" -o "$o"
  objs+=("$o")
done
"$NVCC" "${GEN[@]}" -shared -Xcompiler -fPIC "${objs[@]}" -o "$OUT/libgnufft_ref.so" \
  -L"$CUDA_HOME/lib64" -lcufft -lcudart -Xlinker -rpath -Xlinker "$CUDA_HOME/lib64"
echo "built $OUT/libgnufft_ref.so"
