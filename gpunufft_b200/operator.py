"""Python face of the operator path.

:class:`Plan` wraps one C-ABI plan (the counterpart of one upstream
``GpuNUFFTOperator``).  :class:`NUFFTOp` mirrors the upstream pybind11
binding ``gpuNUFFT.NUFFTOp`` (CUDA/src/gpu/python/
gpuNUFFT_operator_python_factory.cpp:70-182): same constructor arguments,
same ``op`` / ``adj_op`` methods, same array conventions, so existing callers
can switch by changing the import.

NumPy inputs run through the host-buffer entry points (copies inside the
call, like the upstream).  CUDA ``torch.Tensor`` inputs run through the
device entry points on the current torch stream and return CUDA tensors.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _capi as C

try:  # torch is optional for the NumPy path
    import torch
except Exception:  # pragma: no cover
    torch = None


def _is_cuda_tensor(x) -> bool:
    return torch is not None and isinstance(x, torch.Tensor) and x.is_cuda


def _raw(a, dtype) -> np.ndarray:
    """The array's elements in memory order, as the upstream binding reads
    the raw buffer (C- or Fortran-contiguous inputs alike)."""
    a = np.asarray(a)
    if a.dtype != dtype:
        a = a.astype(dtype)
    return np.ascontiguousarray(np.ravel(a, order="K"))


class Plan:
    """One trajectory's operator (tables, maps, FFT plans resident).

    ``traj``: float32 (dim, M) coordinates in [-0.5, 0.5).  ``img_dims``:
    (width, height[, depth]).  ``sens``: complex64 (C, [depth,] height,
    width) or None.  ``operator_type``: one of DEFAULT / TEXTURE / BALANCED /
    BALANCED_TEXTURE (upstream OperatorType).
    """

    def __init__(self, traj, img_dims: Sequence[int], kernel_width: int = 3,
                 sector_width: int = 8, osf: float = 2.0, dens=None,
                 sens=None, operator_type: int = C.BALANCED,
                 reference_order: bool = False, plain: bool = False,
                 device: int = 0, tile_coils: int = 0,
                 use_cufft: bool = False, _load: Optional[dict] = None):
        self._h = ctypes.c_void_p()
        dims = [int(v) for v in img_dims]
        if len(dims) == 2:
            dims.append(0)
        self.dim = 2 if dims[2] == 0 else 3
        if _load is None:
            t = _raw(traj, np.float32)
            if t.size % self.dim:
                raise ValueError("trajectory size is not a multiple of dim")
            M = t.size // self.dim
        else:
            M = int(_load["data_indices"].size)
        self.M = M
        self.img_dims = tuple(dims)
        self.img_shape = ((dims[1], dims[0]) if self.dim == 2 else
                          (dims[2], dims[1], dims[0]))
        self.n_img = int(np.prod(self.img_shape))
        sens_arr = None
        n_sens = 0
        if sens is not None and np.asarray(sens).size > 0:
            sens_arr = _raw(sens, np.complex64)
            if sens_arr.size % self.n_img:
                raise ValueError("sensitivity maps do not match the image")
            n_sens = sens_arr.size // self.n_img
        d = C.Desc()
        d.img_dims[:] = dims
        d.n_samples = M
        d.n_coils = n_sens
        d.kernel_width = int(kernel_width)
        d.sector_width = int(sector_width)
        d.osf = float(osf)
        d.operator_type = int(operator_type)
        d.flags = ((C.FLAG_REFERENCE_ORDER if reference_order else 0) |
                   (C.FLAG_PLAIN if plain else 0) |
                   (C.FLAG_CUFFT if use_cufft else 0) |
                   C.fwd_tile_flag(tile_coils))
        d.device = int(device)
        self.device = int(device)
        self.n_sens = n_sens
        self.kernel_width = int(kernel_width)
        self.sector_width = int(sector_width)
        self.osf = float(osf)
        self.operator_type = int(operator_type)
        self.tile_coils = int(tile_coils)
        L = C.lib()
        dens_arr = None if dens is None else _raw(dens, np.float32)
        if dens_arr is not None and dens_arr.size != M:
            raise ValueError("density compensation must have one value per "
                             "sample")
        if _load is None:
            C.check(L.gnufft_plan_create(
                ctypes.byref(d), t.ctypes.data,
                None if dens_arr is None else dens_arr.ctypes.data,
                None if sens_arr is None else sens_arr.ctypes.data,
                ctypes.byref(self._h)))
        else:
            # converted copies stay referenced until the call returns
            def arr(key, dtype):
                v = _load.get(key)
                return None if v is None else np.ascontiguousarray(v, dtype)
            traj_s = arr("traj_sorted", np.float32)
            di = arr("data_indices", np.uint32)
            sdc = arr("sector_data_count", np.uint32)
            order = arr("processing_order", np.uint32)
            ctr = arr("sector_centers", np.uint32)
            dens_s = arr("dens_sorted", np.float32)
            deapo = arr("deapo", np.float32)
            n_order = 0 if order is None else order.size // 2
            ptr = lambda a: None if a is None else a.ctypes.data  # noqa: E731
            C.check(L.gnufft_plan_load(
                ctypes.byref(d), ptr(traj_s), ptr(di), ptr(sdc), ptr(order),
                n_order, ptr(ctr), ptr(dens_s),
                None if sens_arr is None else sens_arr.ctypes.data,
                ptr(deapo), ctypes.byref(self._h)))
        self.info = self._info()
        self.grid_shape = (
            tuple(int(v) for v in self.info.grid_dims[:2][::-1])
            if self.dim == 2 else
            tuple(int(v) for v in self.info.grid_dims[:3][::-1]))
        self.n_grid = int(np.prod(self.grid_shape))

    # ------------------------------------------------------------------
    @classmethod
    def load(cls, tables: dict, img_dims, kernel_width=3, sector_width=8,
             osf=2.0, sens=None, operator_type=C.BALANCED, device=0):
        """Plan from precomputed tables (upstream
        loadPrecomputedGpuNUFFTOperator)."""
        return cls(None, img_dims, kernel_width, sector_width, osf, None, sens,
                   operator_type, device=device, _load=tables)

    def _info(self) -> C.PlanInfo:
        info = C.PlanInfo()
        C.check(C.lib().gnufft_plan_get_info(self._h, ctypes.byref(info)))
        return info

    def tables(self) -> dict:
        """Sector tables, sorted trajectory, deapodization and LUT."""
        i = self.info
        out = dict(
            traj_sorted=np.zeros(self.dim * self.M, np.float32),
            data_indices=np.zeros(self.M, np.uint32),
            sector_data_count=np.zeros(i.n_sectors + 1, np.uint32),
            processing_order=np.zeros(2 * i.n_processing_order, np.uint32),
            sector_centers=np.zeros(self.dim * i.n_sectors, np.uint32),
            dens_sorted=np.zeros(self.M, np.float32) if i.has_dens else None,
            deapo=np.zeros(self.n_img, np.float32),
            kernel_lut=np.zeros(i.kernel_lut_len, np.float32))
        p = lambda a: None if a is None else a.ctypes.data  # noqa: E731
        C.check(C.lib().gnufft_export_tables(
            self._h, p(out["traj_sorted"]), p(out["data_indices"]),
            p(out["sector_data_count"]), p(out["processing_order"]),
            p(out["sector_centers"]), p(out["dens_sorted"]), p(out["deapo"]),
            p(out["kernel_lut"])))
        out["traj_sorted"] = out["traj_sorted"].reshape(self.dim, self.M)
        out["processing_order"] = out["processing_order"].reshape(-1, 2)
        return out

    # the precomputed-operator contract of the upstream MATLAB path
    # (gpuNUFFT.m:101 / loadPrecomputedGpuNUFFTOperator): these arrays plus
    # the geometry rebuild the operator without re-binning
    PLAN_ARRAYS = ("traj_sorted", "data_indices", "sector_data_count",
                   "processing_order", "sector_centers", "dens_sorted",
                   "deapo")

    def save(self, path) -> None:
        """Write the plan's precomputed tables and geometry to ``path``
        (NumPy .npz); ``Plan.from_file`` rebuilds the operator from it."""
        t = self.tables()
        arrays = {k: t[k] for k in self.PLAN_ARRAYS if t[k] is not None}
        np.savez(path, img_dims=np.asarray(self.img_dims, np.uint32),
                 kernel_width=np.uint32(self.kernel_width),
                 sector_width=np.uint32(self.sector_width),
                 osf=np.float32(self.osf),
                 operator_type=np.int32(self.operator_type), **arrays)

    @classmethod
    def from_file(cls, path, sens=None, device: int = 0) -> "Plan":
        """Plan from a file written by ``save`` (tables validated)."""
        with np.load(path) as f:
            tables = {k: (f[k] if k in f.files else None)
                      for k in cls.PLAN_ARRAYS}
            dims = [int(v) for v in f["img_dims"]]
            if dims[2] == 0:
                dims = dims[:2]
            return cls.load(tables, dims, int(f["kernel_width"]),
                            int(f["sector_width"]), float(f["osf"]), sens,
                            int(f["operator_type"]), device=device)

    def set_sens(self, sens) -> None:
        """Replace the maps (host arrays; CUDA tensors are copied on the
        device, ordered on the current torch stream)."""
        if _is_cuda_tensor(sens):
            t = sens.reshape(-1).to(torch.complex64).contiguous()
            n = t.numel() // self.n_img
            if n * self.n_img != t.numel():
                raise ValueError("sensitivity maps do not match the image")
            stream = torch.cuda.current_stream(t.device).cuda_stream
            C.check(C.lib().gnufft_set_sens_device(
                self._h, t.data_ptr(), n, ctypes.c_void_p(stream)))
            self.n_sens = n
            return
        if sens is None:
            C.check(C.lib().gnufft_set_sens(self._h, None, 0))
            self.n_sens = 0
            return
        s = _raw(sens, np.complex64)
        n = s.size // self.n_img
        C.check(C.lib().gnufft_set_sens(self._h, s.ctypes.data, n))
        self.n_sens = n

    def set_memory_limit(self, nbytes: int) -> None:
        """Cap a call's device scratch (0: the free device memory); calls
        whose all-coil scratch exceeds it run in coil passes."""
        C.check(C.lib().gnufft_set_memory_limit(self._h, int(nbytes)))

    def call_scratch_bytes(self, n_coils: int) -> int:
        """Device scratch the plan holds after a call with n_coils coils."""
        v = ctypes.c_uint64()
        C.check(C.lib().gnufft_call_scratch_bytes(self._h, int(n_coils),
                                                  ctypes.byref(v)))
        return int(v.value)

    def set_timing(self, enable: bool = True) -> None:
        C.check(C.lib().gnufft_set_timing(self._h, int(enable)))

    def stage_times(self) -> dict:
        t = C.StageTimes()
        C.check(C.lib().gnufft_get_stage_times(self._h, ctypes.byref(t)))
        return dict(prepare_ms=t.prepare_ms, gridding_ms=t.gridding_ms,
                    fft_ms=t.fft_ms, finish_ms=t.finish_ms,
                    launches=t.launches)

    # ------------------------------------------------------------------
    def _adj_count(self, n_coils, output):
        if output in (C.CONVOLUTION, C.DENSITY_ESTIMATION):
            return n_coils * self.n_grid, (n_coils,) + self.grid_shape
        if output == C.DEAPODIZATION and self.n_sens:
            return self.n_img, self.img_shape
        return n_coils * self.n_img, (n_coils,) + self.img_shape

    def adjoint(self, kspace, output: int = C.DEAPODIZATION,
                n_coils: Optional[int] = None):
        """Adjoint NUFFT of k-space (C, M) (original sample order)."""
        if _is_cuda_tensor(kspace):
            k = kspace.reshape(-1).to(torch.complex64).contiguous()
            nc = n_coils or k.numel() // self.M
            if k.numel() != nc * self.M:
                raise ValueError("k-space size does not match the plan")
            cnt, shape = self._adj_count(nc, output)
            out = torch.empty(cnt, dtype=torch.complex64, device=k.device)
            stream = torch.cuda.current_stream(k.device).cuda_stream
            C.check(C.lib().gnufft_adjoint_device(
                self._h, k.data_ptr(), out.data_ptr(), nc, int(output),
                ctypes.c_void_p(stream)))
            return out.reshape(shape)
        k = _raw(kspace, np.complex64)
        nc = n_coils or k.size // self.M
        if k.size != nc * self.M:
            raise ValueError("k-space size does not match the plan")
        cnt, shape = self._adj_count(nc, output)
        out = np.empty(cnt, np.complex64)
        C.check(C.lib().gnufft_adjoint_host(self._h, k.ctypes.data,
                                            out.ctypes.data, nc, int(output)))
        return out.reshape(shape)

    def forward(self, image, output: int = C.DEAPODIZATION,
                n_coils: Optional[int] = None):
        """Forward NUFFT; returns k-space (C, M) in original sample order."""
        nc_default = self.n_sens if self.n_sens else None
        if _is_cuda_tensor(image):
            x = image.reshape(-1).to(torch.complex64).contiguous()
            nc = n_coils or nc_default or x.numel() // self.n_img
            need = self.n_img if self.n_sens else nc * self.n_img
            if x.numel() != need:
                raise ValueError("image size does not match the plan")
            out = torch.empty(nc * self.M, dtype=torch.complex64,
                              device=x.device)
            stream = torch.cuda.current_stream(x.device).cuda_stream
            C.check(C.lib().gnufft_forward_device(
                self._h, x.data_ptr(), out.data_ptr(), nc, int(output),
                ctypes.c_void_p(stream)))
            return out.reshape(nc, self.M)
        x = _raw(image, np.complex64)
        nc = n_coils or nc_default or x.size // self.n_img
        need = self.n_img if self.n_sens else nc * self.n_img
        if x.size != need:
            raise ValueError("image size does not match the plan")
        out = np.empty(nc * self.M, np.complex64)
        C.check(C.lib().gnufft_forward_host(self._h, x.ctypes.data,
                                            out.ctypes.data, nc, int(output)))
        return out.reshape(nc, self.M)

    def traj_grad(self, image, kspace_weights,
                  n_coils: Optional[int] = None):
        """grad[a][j] = sum_c Re(conj(u[c][j]) * d forward(image)[c][j] /
        d k_a[j]) for CUDA tensors (float32 (dim, M), original order)."""
        if not (_is_cuda_tensor(image) and _is_cuda_tensor(kspace_weights)):
            raise TypeError("traj_grad takes CUDA tensors")
        x = image.reshape(-1).to(torch.complex64).contiguous()
        u = kspace_weights.reshape(-1).to(torch.complex64).contiguous()
        nc = n_coils or u.numel() // self.M
        if u.numel() != nc * self.M:
            raise ValueError("k-space weights do not match the plan")
        need = self.n_img if self.n_sens else nc * self.n_img
        if x.numel() != need:
            raise ValueError("image size does not match the plan")
        out = torch.empty((self.dim, self.M), dtype=torch.float32,
                          device=u.device)
        stream = torch.cuda.current_stream(u.device).cuda_stream
        C.check(C.lib().gnufft_traj_grad_device(
            self._h, x.data_ptr(), u.data_ptr(), nc, out.data_ptr(),
            ctypes.c_void_p(stream)))
        return out

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            C.lib().gnufft_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NUFFTOp:
    """Drop-in for the upstream ``gpuNUFFT.NUFFTOp``.

    ``NUFFTOp(kspace_loc, image_size, num_coils, sense_maps, density_comp,
    kernel_width=3, sector_width=8, osr=2, balance_workload=True)``:
    ``kspace_loc`` (dim, M) float32 in [-0.5, 0.5); ``image_size``
    [width, height(, depth)]; ``sense_maps`` complex64 maps or None / an
    empty array; ``density_comp`` (M,) float32 or None.  The upstream factory
    default interpolates the kernel with texture lookups; ``use_textures``
    keeps that default and can be switched off (DEFAULT / BALANCED
    arithmetic).  ``osr`` may be fractional here (the upstream binding takes
    an int).
    """

    def __init__(self, kspace_loc, image_size, num_coils, sense_maps=None,
                 density_comp=None, kernel_width=3, sector_width=8, osr=2,
                 balance_workload=True, use_textures=True, **plan_kwargs):
        dims = [int(v) for v in np.asarray(image_size).ravel()]
        self.dimension = len(dims)
        self.n_coils = int(num_coils)
        if use_textures:
            op_type = C.BALANCED_TEXTURE if balance_workload else C.TEXTURE
        else:
            op_type = C.BALANCED if balance_workload else C.DEFAULT
        has_sens = sense_maps is not None and np.asarray(sense_maps).size > 0
        self.has_sense_data = has_sens
        self.plan = Plan(kspace_loc, dims, kernel_width, sector_width,
                         float(osr), density_comp,
                         sense_maps if has_sens else None, op_type,
                         **plan_kwargs)
        self.trajectory_length = self.plan.M

    def op(self, image, interpolate_data: bool = False):
        """Forward operator -> (n_coils, M) complex64."""
        out = C.DENSITY_ESTIMATION if interpolate_data else C.DEAPODIZATION
        return self.plan.forward(image, out, self.n_coils)

    def adj_op(self, kspace_data, grid_data: bool = False):
        """Adjoint operator -> (n_coils, depth, H, W), or (depth, H, W) with
        sensitivity maps; 2-D results have depth 1."""
        out = C.DENSITY_ESTIMATION if grid_data else C.DEAPODIZATION
        res = self.plan.adjoint(kspace_data, out, self.n_coils)
        shape = self.plan.grid_shape if grid_data else self.plan.img_shape
        if self.dimension == 2:
            shape = (1,) + tuple(shape)
        if self.has_sense_data and not grid_data:
            return res.reshape(shape)
        return res.reshape((self.n_coils,) + tuple(shape))
