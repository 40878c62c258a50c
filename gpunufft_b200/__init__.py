"""gpunufft_b200: the gpuNUFFT operator path, hand-written for B200 (sm_100a).

``NUFFTOp`` mirrors the upstream Python binding; ``Plan`` exposes the full
C ABI (output stages, precomputed tables, device buffers, timing).
"""
from ._capi import (BALANCED, BALANCED_TEXTURE, CONVOLUTION, DEAPODIZATION,
                    DEFAULT, DENSITY_ESTIMATION, FFT, TEXTURE, GnufftError,
                    lib)
from .operator import NUFFTOp, Plan

__all__ = ["NUFFTOp", "Plan", "GnufftError", "lib", "DEFAULT", "TEXTURE",
           "BALANCED", "BALANCED_TEXTURE", "CONVOLUTION", "FFT",
           "DEAPODIZATION", "DENSITY_ESTIMATION"]


def version() -> str:
    return lib().gnufft_version().decode()
