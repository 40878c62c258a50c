"""ctypes access to the upstream gpuNUFFT library built from its own sources.

TEST INFRASTRUCTURE ONLY (the oracle): imported by tests/, by
``__graft_entry__.smoke()`` and by the CPU-baseline leg of ``bench.py``.
The product (``gpunufft_b200``) never imports this module.

``oracle/build_ref.sh`` compiles the upstream sources into
``oracle/_ref/libgnufft_ref.so`` together with ``oracle/ref_harness.cpp``.
When that library is absent (e.g. the upstream tree was not available when
the repository was built) :func:`available` returns False and the callers
skip the checks that need it.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libgnufft_ref.so")

_lib: Optional[ctypes.CDLL] = None

_P = ctypes.c_void_p
_U = ctypes.c_uint32
_F = ctypes.c_float
_I = ctypes.c_int
_L = ctypes.c_long


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(
                f"{LIB_PATH} missing: run oracle/build_ref.sh")
        L = ctypes.CDLL(LIB_PATH)
        L.refh_last_error.restype = ctypes.c_char_p
        L.refh_kernel_lut.restype = _L
        L.refh_kernel_lut.argtypes = [_F, _U, _I, _P, _L]
        L.refh_sector_dims.restype = _U
        L.refh_sector_dims.argtypes = [_U, _U, _U, _F, _U, _P]
        L.refh_sector_tables.restype = _L
        L.refh_sector_tables.argtypes = [_P, _U, _U, _U, _U, _F, _U, _U, _I,
                                         _P, _P, _P, _P, _P, _P, _L, _P, _P]
        L.refh_cpu_gridding.restype = None
        L.refh_cpu_gridding.argtypes = [_P, _P, _P, _P, _P, _I, _P, _I, _I,
                                        _I, _I]
        L.refg_create.restype = _P
        L.refg_create.argtypes = [_P, _U, _U, _U, _U, _P, _P, _U, _U, _U, _F,
                                  _I, _I]
        L.refg_adjoint.restype = _I
        L.refg_adjoint.argtypes = [_P, _P, _P, _I]
        L.refg_forward.restype = _I
        L.refg_forward.argtypes = [_P, _P, _P, _I]
        L.refg_destroy.restype = None
        L.refg_destroy.argtypes = [_P]
        _lib = L
    return _lib


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def kernel_lut(osf: float, kw: int, lin: bool = False) -> np.ndarray:
    """Upstream LUT (gpuNUFFT_utils.cpp:47-60 sizes, :74-107 values)."""
    L = lib()
    n = L.refh_kernel_lut(osf, kw, int(lin), None, 0)
    out = np.zeros(n, np.float32)
    L.refh_kernel_lut(osf, kw, int(lin), out.ctypes.data, n)
    return out


def sector_dims(img_dims, osf: float, sw: int):
    w, h = img_dims[0], img_dims[1]
    d = img_dims[2] if len(img_dims) > 2 else 0
    out = np.zeros(3, np.uint32)
    total = lib().refh_sector_dims(w, h, d, osf, sw, out.ctypes.data)
    return out, int(total)


def sector_tables(traj: np.ndarray, img_dims, osf: float, kw: int, sw: int,
                  balance: bool = True, dens: Optional[np.ndarray] = None):
    """Upstream factory tables with useGpu=false.

    ``traj`` is SoA float32 of shape (dim, M).  Returns a dict with
    ``assigned`` (per-sample sector, original order), ``data_indices``,
    ``sector_data_count``, ``centers``, ``order`` (W, 2), ``traj_sorted``
    and ``dens_sorted``.
    """
    traj = np.ascontiguousarray(traj, np.float32)
    dim, M = traj.shape
    w, h = img_dims[0], img_dims[1]
    d = img_dims[2] if dim == 3 else 0
    _, S = sector_dims((w, h, d), osf, sw)
    assigned = np.zeros(M, np.uint32)
    di = np.zeros(M, np.uint32)
    cnt = np.zeros(S + 1, np.uint32)
    ctr = np.zeros(dim * S, np.uint32)
    cap = S + M // 256 + 2
    order = np.zeros(2 * cap, np.uint32)
    ts = np.zeros(dim * M, np.float32)
    dens_c = None if dens is None else np.ascontiguousarray(dens, np.float32)
    ds = None if dens is None else np.zeros(M, np.float32)
    n = lib().refh_sector_tables(
        traj.ctypes.data, M, w, h, d, osf, kw, sw, int(balance),
        _ptr(dens_c), assigned.ctypes.data, di.ctypes.data, cnt.ctypes.data,
        ctr.ctypes.data, order.ctypes.data, cap, ts.ctypes.data, _ptr(ds))
    if n < 0:
        raise RuntimeError(lib().refh_last_error().decode())
    return dict(assigned=assigned, data_indices=di, sector_data_count=cnt,
                centers=ctr, order=order[: 2 * n].reshape(n, 2),
                traj_sorted=ts.reshape(dim, M), dens_sorted=ds)


def cpu_gridding(data_sorted: np.ndarray, crds_sorted_aos: np.ndarray,
                 lut: np.ndarray, sector_data_count: np.ndarray,
                 centers: np.ndarray, sw: int, kw: int, width: int,
                 gdata: Optional[np.ndarray] = None) -> np.ndarray:
    """The upstream CPU gridding routine gpuNUFFT_cpu (cpu/gpuNUFFT_cpu.cpp).

    3D isotropic only; ``data_sorted`` complex64 (M,), ``crds_sorted_aos``
    float32 (M, 3).  Returns the complex64 grid (width**3,) accumulated in
    ``gdata`` (zero-initialised when not given)."""
    data = np.ascontiguousarray(data_sorted, np.complex64)
    crds = np.ascontiguousarray(crds_sorted_aos, np.float32)
    lutc = np.ascontiguousarray(lut, np.float32)
    sec = np.ascontiguousarray(sector_data_count, np.int32)
    ctr = np.ascontiguousarray(centers, np.int32)
    if gdata is None:
        gdata = np.zeros(width ** 3, np.complex64)
    lib().refh_cpu_gridding(data.ctypes.data, crds.ctypes.data,
                            gdata.ctypes.data, lutc.ctypes.data,
                            sec.ctypes.data, len(sec) - 1, ctr.ctypes.data,
                            sw, kw, len(lutc), width)
    return gdata


class RefGpuOperator:
    """The upstream operator on the GPU, host-array calls.  ``textures``
    selects the TEXTURE / BALANCED_TEXTURE operators (the factory's
    useTextures), which read the kernel table through hardware-filtered
    texture fetches (texture objects standing in for the legacy references,
    oracle/ref_compat.h)."""

    def __init__(self, traj, img_dims, n_coils, kw=3, sw=8, osf=2.0,
                 dens=None, sens=None, balance=True, textures=False):
        self.traj = np.ascontiguousarray(traj, np.float32)
        self.dim, self.M = self.traj.shape
        self.img_dims = tuple(int(v) for v in img_dims)
        w, h = self.img_dims[0], self.img_dims[1]
        d = self.img_dims[2] if self.dim == 3 else 0
        self.C = int(n_coils)
        dens_c = None if dens is None else np.ascontiguousarray(dens,
                                                               np.float32)
        sens_c = None if sens is None else np.ascontiguousarray(
            sens, np.complex64)
        self.has_sens = sens is not None
        self.h = lib().refg_create(self.traj.ctypes.data, self.M, w, h, d,
                                   _ptr(dens_c), _ptr(sens_c), self.C, kw, sw,
                                   osf, int(balance), int(textures))
        if not self.h:
            raise RuntimeError(lib().refh_last_error().decode())
        self.n_img = int(np.prod([v for v in self.img_dims if v]))

    def adjoint(self, kspace, stage=2, out_len=None):
        k = np.ascontiguousarray(kspace, np.complex64).ravel()
        ch = 1 if (self.has_sens and stage >= 1) else self.C
        n = out_len if out_len is not None else self.n_img * ch
        out = np.zeros(n, np.complex64)
        if lib().refg_adjoint(self.h, k.ctypes.data, out.ctypes.data, stage):
            raise RuntimeError("upstream adjoint failed")
        return out

    def forward(self, image, stage=2):
        x = np.ascontiguousarray(image, np.complex64).ravel()
        out = np.zeros(self.C * self.M, np.complex64)
        if lib().refg_forward(self.h, x.ctypes.data, out.ctypes.data, stage):
            raise RuntimeError("upstream forward failed")
        return out.reshape(self.C, self.M)

    def close(self):
        if self.h:
            lib().refg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
