"""CPU restatement of the gpuNUFFT operator path (the test oracle).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` as the checker.  The product
(``gpunufft_b200``) never imports it.

Every function restates the upstream algorithm in NumPy and cites the
upstream file:line it follows (paths relative to the upstream ``CUDA/``
directory).  Arithmetic that decides integer results (sector ids, footprint
bounds, LUT indices) is carried out in float32 / float64 exactly as the
upstream C++/CUDA does, so integer outputs are bit-exact.  Accumulations
use float64 (the upstream uses float32 atomics in an unspecified order),
and the FFT runs in float64.

Layouts follow the upstream API: trajectory SoA ``(dim, M)`` float32;
k-space ``(C, M)`` complex64 in original sample order; images and grids
``(C, [Z,] Y, X)`` with x fastest.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple

import numpy as np

f32 = np.float32
MAXIMUM_PAYLOAD = 256  # gpuNUFFT_types.hpp:23
MAXIMUM_ALIASING_ERROR = f32(0.001)  # gpuNUFFT_utils.hpp:47
MAXIMUM_ALIASING_ERROR_LIN_INT = f32(0.0001)  # gpuNUFFT_utils.hpp:50

CONVOLUTION, FFT, DEAPODIZATION, DENSITY_ESTIMATION = 0, 1, 2, 3

# The upstream LUT is computed on the host with the C library's float
# functions; call the same expf / sqrtf so the table is bit-identical (expf
# is not always correctly rounded).  The compiler turns powf(x, 2) into x*x.
_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
for _fn in ("expf", "sqrtf"):
    getattr(_libm, _fn).restype = ctypes.c_float
    getattr(_libm, _fn).argtypes = [ctypes.c_float]
_libm.powf.restype = ctypes.c_float
_libm.powf.argtypes = [ctypes.c_float, ctypes.c_float]


def _expf(x):
    return f32(_libm.expf(float(x)))


def _sqrtf(x):
    return f32(_libm.sqrtf(float(x)))


def _powf(x, y):
    return f32(_libm.powf(float(x), float(y)))


# --------------------------------------------------------------------------
# rounding helpers
# --------------------------------------------------------------------------
def c_round(x: np.ndarray) -> np.ndarray:
    """C ``round``: half away from zero, in the dtype of ``x``."""
    a = np.abs(x)
    f = np.floor(a)
    r = f + (a - f >= 0.5).astype(a.dtype)
    return np.copysign(r, x)


# --------------------------------------------------------------------------
# Kaiser-Bessel lookup table
# --------------------------------------------------------------------------
def i0_f32(x):
    """Modified Bessel I0, polynomial approximation of Abramowitz & Stegun
    9.8.1-9.8.2, evaluated in float32 as gpuNUFFT_utils.cpp:3-34."""
    x = f32(x)
    ax = f32(abs(x))
    if ax < f32(3.75):
        y = f32(x / f32(3.75))
        y = f32(y * y)
        return f32(f32(1.0) + y * (f32(3.5156229) + y * (f32(3.0899424) + y * (
            f32(1.2067492) + y * (f32(0.2659732) + y * (f32(0.360768e-1) + y *
                                                         f32(0.45813e-2)))))))
    y = f32(f32(3.75) / ax)
    poly = (f32(0.39894228) + y * (f32(0.1328592e-1) + y * (f32(0.225319e-2) + y * (
        f32(-0.157565e-2) + y * (f32(0.916281e-2) + y * (f32(-0.2057706e-1) + y * (
            f32(0.2635537e-1) + y * (f32(-0.1647633e-1) + y * f32(0.392377e-2)))))))))
    return f32(f32(_expf(ax) / _sqrtf(ax)) * f32(poly))


def beta(kw: int, osf: float) -> np.float32:
    """gpuNUFFT_utils.hpp:60-63 (float32)."""
    osf = f32(osf)
    t = f32(f32(kw) / osf * (osf - f32(0.5)))
    return f32(f32(math.pi) * _sqrtf(f32(t * t - f32(0.8))))


def kernel_value(r, kw: int, osf: float) -> np.float32:
    """gpuNUFFT_utils.hpp:72-75: I0(beta*sqrt(1-r^2)) / I0(beta)."""
    b = beta(kw, osf)
    r = f32(r)
    return f32(i0_f32(f32(b * _sqrtf(f32(f32(1.0) - r * r)))) /
               i0_f32(b))


def lut_size(osf: float, kw: int, lin: bool = False) -> int:
    """gpuNUFFT_utils.cpp:47-60."""
    osf = f32(osf)
    if lin:
        kosf = int(math.floor(math.sqrt(
            0.37 / float(f32(osf * osf) * MAXIMUM_ALIASING_ERROR_LIN_INT))))
    else:
        kosf = int(math.floor(float(f32(0.91) /
                                    f32(osf * MAXIMUM_ALIASING_ERROR))))
    return int(kosf * float(f32(kw)) * 0.5)


def kernel_lut(osf: float, kw: int, lin: bool = False) -> np.ndarray:
    """gpuNUFFT_utils.cpp:74-107 (load1DKernel): table over r^2 in [0,1]."""
    n = lut_size(osf, kw, lin)
    k = np.zeros(n, np.float32)
    for i in range(1, n - 1):
        if kw == 1:
            k[i] = 1.0
        else:
            r = math.sqrt(i / float(n - 1))
            k[i] = kernel_value(f32(r), kw, osf)
    k[0] = 1.0
    k[n - 1] = 0.0
    return k


# --------------------------------------------------------------------------
# problem geometry (GpuNUFFTInfo, gpuNUFFT_operator.cpp:53-146)
# --------------------------------------------------------------------------
@dataclass
class Geometry:
    img: Tuple[int, int, int]      # (X, Y, Z); Z == 0 for 2D
    grid: Tuple[int, int, int]     # (GX, GY, GZ); GZ == 0 for 2D
    kw: int
    sw: int
    osf: float
    lut_len: int
    kernel_radius: np.float32
    radius_sq: np.float32
    radius_sq_inv: np.float32
    dist_multiplier: np.float32
    pad: int
    offset: int
    aniso: Tuple[np.float32, np.float32, np.float32]
    sectors: Tuple[int, int, int]  # per axis (Z count 1 for 2D)

    @property
    def dim(self) -> int:
        return 2 if self.img[2] == 0 else 3

    @property
    def n_sectors(self) -> int:
        return int(np.prod([s for s in self.sectors]))

    @property
    def grid_count(self) -> int:
        return self.grid[0] * self.grid[1] * max(self.grid[2], 1)

    @property
    def img_count(self) -> int:
        return self.img[0] * self.img[1] * max(self.img[2], 1)

    @property
    def grid_shape(self) -> Tuple[int, ...]:
        return (self.grid[1], self.grid[0]) if self.dim == 2 else (
            self.grid[2], self.grid[1], self.grid[0])

    @property
    def img_shape(self) -> Tuple[int, ...]:
        return (self.img[1], self.img[0]) if self.dim == 2 else (
            self.img[2], self.img[1], self.img[0])


def grid_extent(n: int, osf: float) -> int:
    """gpuNUFFT_types.hpp:109-117: (IndType)(n * osf) in float."""
    return int(f32(f32(n) * f32(osf)))


def make_geometry(img_dims: Sequence[int], osf: float, kw: int, sw: int,
                  lin_lut: bool = False) -> Geometry:
    X, Y = int(img_dims[0]), int(img_dims[1])
    Z = int(img_dims[2]) if len(img_dims) > 2 else 0
    GX, GY, GZ = grid_extent(X, osf), grid_extent(Y, osf), grid_extent(Z, osf)
    L = lut_size(osf, kw, lin_lut)
    gmax = max(GX, GY, GZ)
    kernel_radius = kw / 2.0
    radius = kernel_radius / gmax
    rsq = radius * radius
    rinv = 1.0 / rsq
    dm = f32((L - 1) * rinv)
    pad = sw + 2 * int(math.floor(f32(kw) / f32(2.0)))
    offset = int(math.floor(f32(pad) / f32(2.0)))
    aniso = (f32(f32(GX) / f32(gmax)), f32(f32(GY) / f32(gmax)),
             f32(f32(GZ) / f32(gmax)))

    def nsec(g):  # gpuNUFFT_operator_factory.cpp:22-26
        return int(math.ceil(float(f32(g)) / sw)) if g else 0

    sectors = (nsec(GX), nsec(GY), max(nsec(GZ), 1))
    return Geometry((X, Y, Z), (GX, GY, GZ), kw, sw, float(f32(osf)), L,
                    f32(kernel_radius), f32(rsq), f32(rinv), dm, pad, offset,
                    aniso, sectors)


# --------------------------------------------------------------------------
# sector binning (factory)
# --------------------------------------------------------------------------
def sector_of_axis(c: np.ndarray, G: int, sw: int) -> np.ndarray:
    """precomp_utils.hpp:34-48: floor(round(c*G + 0.5*G) / sw) clamped.
    c*G is a float32 product; +0.5*G, round and the division are double."""
    prod = (c.astype(np.float32) * f32(G)).astype(np.float64)
    s = np.floor(c_round(prod + 0.5 * float(f32(G))) / float(f32(sw)))
    top = math.ceil(float(f32(G)) / float(f32(sw))) - 1
    s = np.where(s >= top + 1, top, s)
    s = np.where(s < 0, 0, s)
    return s.astype(np.int64)


def assign_sectors(traj: np.ndarray, g: Geometry) -> np.ndarray:
    """gpuNUFFT_operator_factory.cpp:128-181 + precomp_utils.hpp:142-153."""
    sx = sector_of_axis(traj[0], g.grid[0], g.sw)
    sy = sector_of_axis(traj[1], g.grid[1], g.sw)
    lin = sx + g.sectors[0] * sy
    if g.dim == 3:
        sz = sector_of_axis(traj[2], g.grid[2], g.sw)
        lin = lin + g.sectors[0] * g.sectors[1] * sz
    return lin.astype(np.uint32)


def sector_data_count(assigned: np.ndarray, n_sectors: int) -> np.ndarray:
    """gpuNUFFT_operator_factory.cpp:183-205: exclusive offsets (S+1)."""
    counts = np.bincount(assigned.astype(np.int64), minlength=n_sectors)
    return np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)


def sector_centers(g: Geometry) -> np.ndarray:
    """gpuNUFFT_operator_factory.cpp:207-270: s*sw + floor(sw/2), x fastest,
    interleaved per sector ([x,y] or [x,y,z])."""
    half = int(math.floor(f32(g.sw) / f32(2.0)))
    sx, sy, sz = g.sectors
    if g.dim == 2:
        yy, xx = np.meshgrid(np.arange(sy), np.arange(sx), indexing="ij")
        c = np.stack([xx * g.sw + half, yy * g.sw + half], -1)
    else:
        zz, yy, xx = np.meshgrid(np.arange(sz), np.arange(sy), np.arange(sx),
                                 indexing="ij")
        c = np.stack([xx * g.sw + half, yy * g.sw + half, zz * g.sw + half],
                     -1)
    return c.reshape(-1).astype(np.uint32)


def processing_order(sdc: np.ndarray) -> np.ndarray:
    """gpuNUFFT_operator_factory.cpp:74-126: non-empty sectors by count
    descending, each split into ceil(n/256) chunks (sector, 256*k).  The
    upstream sorts with an unstable std::sort, so only the multiset of
    chunks (and the descending count order) is defined; this restatement
    breaks count ties by sector id."""
    counts = np.diff(sdc.astype(np.int64))
    order = sorted([(-int(n), s) for s, n in enumerate(counts) if n > 0])
    out = []
    for negn, s in order:
        n = -negn
        out.append((s, 0))
        rem, k = n, 1
        while rem - MAXIMUM_PAYLOAD > 0:
            rem -= MAXIMUM_PAYLOAD
            out.append((s, k * MAXIMUM_PAYLOAD))
            k += 1
    return np.array(out, np.uint32).reshape(-1, 2)


@dataclass
class Tables:
    assigned: np.ndarray        # per-sample sector (original order)
    data_indices: np.ndarray    # sorted position -> original index
    sector_data_count: np.ndarray
    centers: np.ndarray
    order: np.ndarray
    traj_sorted: np.ndarray
    dens_sorted: Optional[np.ndarray]
    sector_sorted: np.ndarray   # sector of each sorted sample


def build_tables(traj: np.ndarray, g: Geometry,
                 dens: Optional[np.ndarray] = None,
                 data_indices: Optional[np.ndarray] = None) -> Tables:
    """gpuNUFFT_operator_factory.cpp:450-553 without the deapodization step.
    The within-sector order is a stable one unless ``data_indices`` (e.g.
    the upstream's own unstable-sort order) is given."""
    traj = np.ascontiguousarray(traj, np.float32)
    a = assign_sectors(traj, g)
    if data_indices is None:
        di = np.argsort(a, kind="stable").astype(np.uint32)
    else:
        di = np.asarray(data_indices, np.uint32)
    sdc = sector_data_count(a, g.n_sectors)
    return Tables(a, di, sdc, sector_centers(g), processing_order(sdc),
                  traj[:, di], None if dens is None else
                  np.asarray(dens, np.float32)[di], a[di])


# --------------------------------------------------------------------------
# per-sample footprint and weights (atomic_gpuNUFFT_kernels.cu:302-451)
# --------------------------------------------------------------------------
def _footprint_axis(c: np.ndarray, G: int, center: np.ndarray, g: Geometry,
                    aniso: np.float32, lut: np.ndarray, texture: bool):
    """One axis of the upstream footprint for every sample.

    pos = mapKSpaceToGrid (gpuNUFFT_utils.hpp:194-199; the GPU contracts
    c*G + 0.5*G into one fma), bounds by set_minmax (:89-104) in the sample's
    own sector tile, cell k-space position by mapGridToKSpace (:202-209).
    Returns (global unwrapped cell [M,K], weight [M,K] float32, valid [M,K]).
    """
    Gf = f32(G)
    pos = (c.astype(np.float64) * float(Gf) + float(f32(0.5) * Gf)).astype(
        np.float32)
    pos = f32(pos - center.astype(np.float32)) + f32(g.offset)
    pos = pos.astype(np.float32)
    pmax = g.pad - 1
    kr = g.kernel_radius
    imin = np.ceil((pos - kr).astype(np.float32)).astype(np.int64)
    imax = np.floor((pos + kr).astype(np.float32)).astype(np.int64)
    imin = np.where(imin < 0, 0, imin)
    imax = np.where(imax < 0, 0, imax)
    imax = np.where(imax >= pmax, pmax, imax)
    imin = np.where(imin >= pmax, int(pmax - 2 * float(kr)), imin)
    K = g.kw + 2
    i = imin[:, None] + np.arange(K)[None, :]
    valid = i <= imax[:, None]
    gcell = i + center[:, None].astype(np.int64) - g.offset
    kx = (gcell.astype(np.float32) / Gf - f32(0.5)).astype(np.float32)
    d = ((kx - c[:, None].astype(np.float32)) * aniso).astype(np.float32)
    d2 = (d * d).astype(np.float32)
    if texture:
        w = lerp_lut(lut, (d2 * g.radius_sq_inv).astype(np.float32))
    else:
        valid &= d2 < g.radius_sq
        idx = c_round((d2 * g.dist_multiplier).astype(np.float32))
        idx = np.clip(idx, 0, len(lut) - 1).astype(np.int64)
        w = lut[idx]
    return gcell, w.astype(np.float32), valid


def lerp_lut(lut: np.ndarray, u: np.ndarray, frac_bits: int = 8) -> np.ndarray:
    """Normalised-coordinate linear filtering with clamp addressing as the
    texture unit does it (texel coordinate u*W-0.5, weight quantised to
    ``frac_bits`` fractional bits); used by the TEXTURE operators
    (cuda_utils.cuh:27-37 with load2DKernel, gpuNUFFT_utils.cpp:109-124,
    whose 2D table is the outer product of the 1D table)."""
    W = len(lut)
    x = u.astype(np.float32) * f32(W) - f32(0.5)
    i0 = np.floor(x)
    a = (x - i0).astype(np.float32)
    q = float(1 << frac_bits)
    a = np.round(a * q) / q
    i0 = i0.astype(np.int64)
    lo = lut[np.clip(i0, 0, W - 1)]
    hi = lut[np.clip(i0 + 1, 0, W - 1)]
    return ((1.0 - a) * lo + a * hi).astype(np.float32)


def footprints(tab: Tables, g: Geometry, lut: np.ndarray,
               texture: bool = False):
    """Per-axis footprints of every sorted sample in its own sector frame."""
    ctr = tab.centers.reshape(-1, g.dim).astype(np.int64)
    sec = tab.sector_sorted.astype(np.int64)
    out = []
    for ax in range(g.dim):
        out.append(_footprint_axis(tab.traj_sorted[ax], g.grid[ax],
                                   ctr[sec, ax], g, g.aniso[ax], lut, texture))
    return out


def _wrap(cell: np.ndarray, G: int) -> np.ndarray:
    """calculateOppositeIndex (gpuNUFFT_utils.hpp:268-278): one wrap."""
    return np.where(cell >= G, cell - G, np.where(cell < 0, cell + G, cell))


def _stencil(fp, g: Geometry):
    """Flattened (M, K^dim) grid index and float32 weight (z*y*x order of
    atomic_gpuNUFFT_kernels.cu:361-363) with validity mask."""
    if g.dim == 2:
        (cx, wx, vx), (cy, wy, vy) = fp
        idx = _wrap(cy, g.grid[1])[:, :, None] * g.grid[0] + _wrap(
            cx, g.grid[0])[:, None, :]
        w = (wy[:, :, None] * wx[:, None, :]).astype(np.float32)
        v = vy[:, :, None] & vx[:, None, :]
    else:
        (cx, wx, vx), (cy, wy, vy), (cz, wz, vz) = fp
        gx, gy, gz = g.grid
        idx = (_wrap(cz, gz)[:, :, None, None] * gy +
               _wrap(cy, gy)[:, None, :, None]) * gx + _wrap(cx, gx)[:, None,
                                                                     None, :]
        w = ((wz[:, :, None, None] * wy[:, None, :, None]).astype(np.float32)
             * wx[:, None, None, :]).astype(np.float32)
        v = vz[:, :, None, None] & vy[:, None, :, None] & vx[:, None, None, :]
    M = idx.shape[0]
    return idx.reshape(M, -1), w.reshape(M, -1), v.reshape(M, -1)


# --------------------------------------------------------------------------
# gridding kernels
# --------------------------------------------------------------------------
def adjoint_convolution(data_sorted: np.ndarray, tab: Tables, g: Geometry,
                        lut: np.ndarray, texture: bool = False) -> np.ndarray:
    """Adjoint spread (atomic_gpuNUFFT_kernels.cu:302-451, 469-617) of sorted
    samples ``(C, M)`` onto the oversampled grid ``(C, G)`` (flattened,
    x fastest), with the single wrap-around of the flush."""
    data_sorted = np.atleast_2d(data_sorted)
    idx, w, v = _stencil(footprints(tab, g, lut, texture), g)
    C = data_sorted.shape[0]
    out = np.zeros((C, g.grid_count), np.complex128)
    ii = idx[v]
    for c in range(C):
        # weight * value in float32 (as the kernels multiply), summed in f64
        d = data_sorted[c].astype(np.complex64)
        contrib = (w * d.real[:, None]).astype(np.float32) + 1j * (
            w * d.imag[:, None]).astype(np.float32)
        np.add.at(out[c], ii, contrib[v])
    return out


def forward_interpolation(grid: np.ndarray, tab: Tables, g: Geometry,
                          lut: np.ndarray, texture: bool = False) -> np.ndarray:
    """Forward interpolation (atomic_gpuNUFFT_kernels.cu:966-1131,
    1234-1400): out[c, t] = sum over the footprint of w * grid[c, cell]."""
    grid = np.atleast_2d(grid).reshape(-1, g.grid_count)
    idx, w, v = _stencil(footprints(tab, g, lut, texture), g)
    wv = np.where(v, w, 0).astype(np.float64)
    return np.einsum("mk,cmk->cm", wv, grid[:, idx])


# --------------------------------------------------------------------------
# image-space stages (std_gpuNUFFT_kernels.cu)
# --------------------------------------------------------------------------
def fftshift(x: np.ndarray, g: Geometry, inverse: bool = True) -> np.ndarray:
    """std_gpuNUFFT_kernels.cu:374-462, 569-654: out[x] = in[(x+off) % G]
    with off = floor(G/2) (INVERSE) or ceil(G/2) (FORWARD), all axes."""
    axes = tuple(range(-g.dim, 0))
    shape = g.grid_shape
    offs = []
    for n in shape:
        offs.append(n // 2 if inverse else (n + 1) // 2)
    return np.roll(x, [-o for o in offs], axis=axes)


def crop_offsets(g: Geometry) -> Tuple[int, ...]:
    """std_gpuNUFFT_kernels.cu:546-556: (IndType)(N*(osf-1)/2) in float,
    ordered like the array axes ((z,) y, x)."""
    def o(n):
        return int(f32(f32(n) * f32(f32(g.osf) - f32(1.0)) / f32(2)))
    if g.dim == 2:
        return (o(g.img[1]), o(g.img[0]))
    return (o(g.img[2]), o(g.img[1]), o(g.img[0]))


def crop(grid: np.ndarray, g: Geometry) -> np.ndarray:
    off = crop_offsets(g)
    sl = tuple(slice(o, o + n) for o, n in zip(off, g.img_shape))
    return grid[(Ellipsis,) + sl]


def pad(img: np.ndarray, g: Geometry) -> np.ndarray:
    out = np.zeros(img.shape[:-g.dim] + g.grid_shape, img.dtype)
    off = crop_offsets(g)
    sl = tuple(slice(o, o + n) for o, n in zip(off, g.img_shape))
    out[(Ellipsis,) + sl] = img
    return out


def _ifftn(x, g):
    axes = tuple(range(-g.dim, 0))
    return np.fft.ifftn(x, axes=axes) * np.prod([x.shape[a] for a in axes])


def _fftn(x, g):
    return np.fft.fftn(x, axes=tuple(range(-g.dim, 0)))


def deapodization(g: Geometry, lut: np.ndarray,
                  texture: bool = False) -> np.ndarray:
    """gpuNUFFT_operator_factory.cpp:359-448: adjoint (up to FFT: crop and
    1/sqrt(Ng)) of one unit sample at k=0 with sector width 8, then
    1/|h*sqrt(Ng)|."""
    g8 = make_geometry(g.img[:2] if g.dim == 2 else g.img, g.osf, g.kw, 8,
                       lin_lut=texture)
    traj = np.zeros((g.dim, 1), np.float32)
    tab = build_tables(traj, g8)
    grid = adjoint_convolution(np.ones((1, 1), np.complex64), tab, g8, lut,
                               texture)[0].reshape(g8.grid_shape)
    h = fftshift(_ifftn(fftshift(grid, g8, True), g8), g8, True)
    h = crop(h, g8) / math.sqrt(g8.grid_count)
    val = h * math.sqrt(g8.grid_count)
    return (1.0 / np.abs(val)).astype(np.float32)


# --------------------------------------------------------------------------
# the operator (gpuNUFFT_operator.cpp:615-861 adjoint, :1092-1268 forward)
# --------------------------------------------------------------------------
class OracleOperator:
    """Restatement of GpuNUFFTOperator (DEFAULT / BALANCED: same arithmetic;
    TEXTURE / BALANCED_TEXTURE with ``texture=True``)."""

    def __init__(self, traj: np.ndarray, img_dims: Sequence[int], kw=3, sw=8,
                 osf=2.0, dens: Optional[np.ndarray] = None,
                 sens: Optional[np.ndarray] = None, texture: bool = False,
                 data_indices: Optional[np.ndarray] = None):
        self.traj = np.ascontiguousarray(traj, np.float32)
        self.g = make_geometry(img_dims, osf, kw, sw, lin_lut=texture)
        self.texture = texture
        self.lut = kernel_lut(osf, kw, lin=texture)
        self.tab = build_tables(self.traj, self.g, dens, data_indices)
        self.deapo = deapodization(self.g, self.lut, texture)
        self.dens = None if dens is None else np.asarray(dens, np.float32)
        self.sens = None if sens is None else np.asarray(
            sens, np.complex64).reshape((-1,) + self.g.img_shape)
        self.M = self.traj.shape[1]

    # adjoint -------------------------------------------------------------
    def adjoint(self, kspace: np.ndarray, stage: int = DEAPODIZATION):
        g = self.g
        k = np.asarray(kspace, np.complex64).reshape(-1, self.M)
        ks = k[:, self.tab.data_indices].astype(np.complex64)
        if self.dens is not None:  # std_gpuNUFFT_kernels.cu:220-242
            ks = (ks * np.sqrt(self.tab.dens_sorted)).astype(np.complex64)
        grid = adjoint_convolution(ks, self.tab, g, self.lut, self.texture)
        grid = grid.reshape((-1,) + g.grid_shape)
        if stage in (CONVOLUTION, DENSITY_ESTIMATION):
            return grid
        img = fftshift(_ifftn(fftshift(grid, g, True), g), g, True)
        img = crop(img, g) / math.sqrt(g.grid_count)
        if stage == FFT:
            return img
        img = img * self.deapo
        if self.sens is not None:
            img = np.sum(np.conj(self.sens) * img, axis=0)
        return img

    # forward -------------------------------------------------------------
    def forward(self, image: np.ndarray, stage: int = DEAPODIZATION):
        g = self.g
        x = np.asarray(image, np.complex128).reshape((-1,) + g.img_shape)
        if self.sens is not None:
            x = self.sens * x[0]
        x = x * self.deapo
        if stage == DENSITY_ESTIMATION:
            # interpolation straight from the (image-sized) array
            # (gpuNUFFT_operator.cpp:1178-1187); meaningful at osf = 1
            out = forward_interpolation(x.reshape(x.shape[0], -1), self.tab,
                                        g, self.lut, self.texture)
            res = np.zeros_like(out)
            res[:, self.tab.data_indices] = out
            return res
        grid = fftshift(_fftn(fftshift(pad(x, g), g, True), g), g, False)
        out = forward_interpolation(grid.reshape(grid.shape[0], -1), self.tab,
                                    g, self.lut, self.texture)
        out = out / math.sqrt(g.grid_count)
        if self.dens is not None:
            out = out * np.sqrt(self.tab.dens_sorted)
        res = np.zeros_like(out)
        res[:, self.tab.data_indices] = out
        return res


# --------------------------------------------------------------------------
# exact references for error statements
# --------------------------------------------------------------------------
def nudft_adjoint(traj: np.ndarray, kspace: np.ndarray,
                  img_shape: Sequence[int]) -> np.ndarray:
    """FP64 direct adjoint NUDFT: x[n] = sum_m k[m] exp(+2 pi i k_m . n),
    n centred (n - N//2), x fastest in ``img_shape`` ((z,) y, x)."""
    dim = traj.shape[0]
    grids = np.meshgrid(*[np.arange(n) - n // 2 for n in img_shape],
                        indexing="ij")
    pts = np.stack([gg.ravel() for gg in grids[::-1]], 0)  # (dim: x, y, z)
    ph = 2j * np.pi * (traj.astype(np.float64).T @ pts[:dim])
    k = np.atleast_2d(kspace).astype(np.complex128)
    return (k @ np.exp(ph)).reshape((k.shape[0],) + tuple(img_shape))


def nudft_forward(traj: np.ndarray, image: np.ndarray) -> np.ndarray:
    """FP64 direct forward NUDFT (adjoint of :func:`nudft_adjoint`)."""
    img = np.asarray(image, np.complex128)
    dim = traj.shape[0]
    shape = img.shape[-dim:]
    grids = np.meshgrid(*[np.arange(n) - n // 2 for n in shape],
                        indexing="ij")
    pts = np.stack([gg.ravel() for gg in grids[::-1]], 0)
    ph = -2j * np.pi * (traj.astype(np.float64).T @ pts[:dim])
    flat = img.reshape(-1, int(np.prod(shape)))
    return flat @ np.exp(ph).T


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# --------------------------------------------------------------------------
# CG-SENSE (matlab/demo/utils/cg_sense_2d.m:40-108, multicoil form)
# --------------------------------------------------------------------------
def cg_sense(op: "OracleOperator", kspace: np.ndarray, maxit: int = 10,
             alpha: float = 0.0, mask: Optional[np.ndarray] = None):
    """The upstream demo's own CG loop with ``op`` carrying the maps:
    rhs = A^H (y sqrt(mask)); M(x) = A^H A x + alpha x; x0 = 0; ``maxit``
    iterations.  Vectors in complex128, operator applications in the
    restated single-precision operator."""
    y = np.asarray(kspace, np.complex64)
    if mask is not None:
        y = (y * np.sqrt(np.asarray(mask, np.float32))).astype(np.complex64)
    rhs = op.adjoint(y).astype(np.complex128)

    def apply_m(v):
        out = op.adjoint(op.forward(v.astype(np.complex64))).astype(
            np.complex128)
        return out + alpha * v if alpha else out

    x = np.zeros_like(rhs)
    r = rhs.copy()
    p = r.copy()
    rr = np.vdot(r, r).real
    for _ in range(maxit):
        ap = apply_m(p)
        a = rr / np.vdot(p, ap)
        x = x + a * p
        r = r - a * ap
        rr_new = np.vdot(r, r).real
        p = r + (rr_new / rr) * p
        rr = rr_new
    return x
