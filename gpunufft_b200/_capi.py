"""ctypes binding of the C ABI in ``include/gpunufft_b200.h``.

The library ``libgpunufft_b200.so`` is built in-tree by
``gpunufft_b200/build.py``.  Importing this module fails loudly when it is
missing: there is no CPU fallback for the operator path.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgpunufft_b200.so")

SUCCESS = 0
ERROR_INVALID_ARGUMENT = 1
ERROR_OUT_OF_MEMORY = 2
ERROR_CUDA = 3
ERROR_CUFFT = 4
ERROR_NOT_SUPPORTED = 5
ERROR_INTERNAL = 6

DEFAULT, TEXTURE, BALANCED, BALANCED_TEXTURE = 0, 1, 2, 3
CONVOLUTION, FFT, DEAPODIZATION, DENSITY_ESTIMATION = 0, 1, 2, 3
FLAG_REFERENCE_ORDER = 0x1
FLAG_PLAIN = 0x2
FLAG_CUFFT = 0x4
# GNUFFT_NOALLOC_SCRATCH_BYTES: staging area of the no-allocation adjoint
NOALLOC_SCRATCH_BYTES = 16 << 20


def fwd_tile_flag(coils: int) -> int:
    """GNUFFT_FLAG_FWD_TILE_COILS(coils); 0 selects automatically."""
    if not coils:
        return 0
    if coils not in (1, 2, 4, 8, 16, 32):
        raise ValueError("tile coils must be 1, 2, 4, 8, 16 or 32")
    return (coils.bit_length()) << 8

# Every entry point declared in include/gpunufft_b200.h.
EXPORTED = (
    "gnufft_plan_create", "gnufft_plan_load", "gnufft_plan_destroy",
    "gnufft_plan_get_info", "gnufft_export_tables", "gnufft_set_sens",
    "gnufft_adjoint_host", "gnufft_adjoint_device", "gnufft_forward_host",
    "gnufft_forward_device", "gnufft_set_timing", "gnufft_get_stage_times",
    "gnufft_last_error", "gnufft_status_string", "gnufft_version",
    "gnufft_adjoint_convolution_noalloc",
    "gnufft_traj_grad_device", "gnufft_set_sens_device",
    "gnufft_set_copy_wait", "gnufft_plan_check",
    "gnufft_set_memory_limit", "gnufft_call_scratch_bytes",
    "gnufft_batch_create", "gnufft_batch_forward", "gnufft_batch_adjoint",
    "gnufft_batch_get_info", "gnufft_batch_destroy",
)


class Desc(ctypes.Structure):
    _fields_ = [("img_dims", ctypes.c_uint32 * 3),
                ("n_samples", ctypes.c_uint32),
                ("n_coils", ctypes.c_uint32),
                ("kernel_width", ctypes.c_uint32),
                ("sector_width", ctypes.c_uint32),
                ("osf", ctypes.c_float),
                ("operator_type", ctypes.c_int32),
                ("flags", ctypes.c_uint32),
                ("device", ctypes.c_int32)]


class PlanInfo(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_uint32),
                ("img_dims", ctypes.c_uint32 * 3),
                ("grid_dims", ctypes.c_uint32 * 3),
                ("sector_dims", ctypes.c_uint32 * 3),
                ("n_sectors", ctypes.c_uint32),
                ("n_samples", ctypes.c_uint32),
                ("n_coils", ctypes.c_uint32),
                ("kernel_lut_len", ctypes.c_uint32),
                ("n_processing_order", ctypes.c_uint32),
                ("has_dens", ctypes.c_uint32),
                ("device_bytes", ctypes.c_uint64)]


class StageTimes(ctypes.Structure):
    _fields_ = [("prepare_ms", ctypes.c_float),
                ("gridding_ms", ctypes.c_float),
                ("fft_ms", ctypes.c_float),
                ("finish_ms", ctypes.c_float),
                ("launches", ctypes.c_uint32)]


class BatchInfo(ctypes.Structure):
    _fields_ = [("n_instances", ctypes.c_uint32),
                ("units", ctypes.c_uint32 * 5),
                ("kernels_forward", ctypes.c_uint32),
                ("kernels_adjoint", ctypes.c_uint32),
                ("fft_calls", ctypes.c_uint32),
                ("device_bytes", ctypes.c_uint64)]


class GnufftError(RuntimeError):
    """A C-ABI call returned a non-success status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{message} (status {status})")
        self.status = status


_lib = None
_P = ctypes.c_void_p
_U = ctypes.c_uint32
_I = ctypes.c_int32


def lib() -> ctypes.CDLL:
    """Load the native library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} not found: build it with `python -m "
            "gpunufft_b200.build` (the operator has no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    st = ctypes.c_int
    L.gnufft_plan_create.restype = st
    L.gnufft_plan_create.argtypes = [ctypes.POINTER(Desc), _P, _P, _P,
                                     ctypes.POINTER(_P)]
    L.gnufft_plan_load.restype = st
    L.gnufft_plan_load.argtypes = [ctypes.POINTER(Desc), _P, _P, _P, _P, _U,
                                   _P, _P, _P, _P, ctypes.POINTER(_P)]
    L.gnufft_plan_destroy.restype = st
    L.gnufft_plan_destroy.argtypes = [_P]
    L.gnufft_plan_get_info.restype = st
    L.gnufft_plan_get_info.argtypes = [_P, ctypes.POINTER(PlanInfo)]
    L.gnufft_export_tables.restype = st
    L.gnufft_export_tables.argtypes = [_P] + [_P] * 8
    L.gnufft_set_sens.restype = st
    L.gnufft_set_sens.argtypes = [_P, _P, _U]
    L.gnufft_set_sens_device.restype = st
    L.gnufft_set_sens_device.argtypes = [_P, _P, _U, _P]
    for name in ("gnufft_adjoint_host", "gnufft_forward_host"):
        f = getattr(L, name)
        f.restype = st
        f.argtypes = [_P, _P, _P, _U, _I]
    for name in ("gnufft_adjoint_device", "gnufft_forward_device"):
        f = getattr(L, name)
        f.restype = st
        f.argtypes = [_P, _P, _P, _U, _I, _P]
    L.gnufft_adjoint_convolution_noalloc.restype = st
    L.gnufft_adjoint_convolution_noalloc.argtypes = [_P, _P, _P, _U, _P]
    L.gnufft_traj_grad_device.restype = st
    L.gnufft_traj_grad_device.argtypes = [_P, _P, _P, _U, _P, _P]
    L.gnufft_set_timing.restype = st
    L.gnufft_set_memory_limit.restype = ctypes.c_int
    L.gnufft_set_memory_limit.argtypes = [_P, ctypes.c_uint64]
    L.gnufft_call_scratch_bytes.restype = ctypes.c_int
    L.gnufft_call_scratch_bytes.argtypes = [_P, _U,
                                            ctypes.POINTER(ctypes.c_uint64)]
    L.gnufft_set_copy_wait.restype = ctypes.c_int
    L.gnufft_set_copy_wait.argtypes = [_P, ctypes.c_int64]
    L.gnufft_plan_check.restype = ctypes.c_int
    L.gnufft_plan_check.argtypes = [_P]
    L.gnufft_set_timing.argtypes = [_P, ctypes.c_int]
    L.gnufft_get_stage_times.restype = st
    L.gnufft_get_stage_times.argtypes = [_P, ctypes.POINTER(StageTimes)]
    L.gnufft_batch_create.restype = st
    L.gnufft_batch_create.argtypes = [_P, _P, _U, ctypes.POINTER(_P)]
    for name in ("gnufft_batch_forward", "gnufft_batch_adjoint"):
        f = getattr(L, name)
        f.restype = st
        f.argtypes = [_P, _P, _P, _P]
    L.gnufft_batch_get_info.restype = st
    L.gnufft_batch_get_info.argtypes = [_P, ctypes.POINTER(BatchInfo)]
    L.gnufft_batch_destroy.restype = st
    L.gnufft_batch_destroy.argtypes = [_P]
    L.gnufft_last_error.restype = ctypes.c_char_p
    L.gnufft_last_error.argtypes = []
    L.gnufft_status_string.restype = ctypes.c_char_p
    L.gnufft_status_string.argtypes = [ctypes.c_int]
    L.gnufft_version.restype = ctypes.c_char_p
    L.gnufft_version.argtypes = []
    _lib = L
    return L


def check(status: int) -> None:
    if status != SUCCESS:
        msg = lib().gnufft_last_error().decode(errors="replace")
        raise GnufftError(status, msg or
                          lib().gnufft_status_string(status).decode())
