"""Seeded synthetic inputs shared by the tests (trajectories, data, maps)."""
import math

import numpy as np

GOLDEN_ANGLE = math.pi * (3.0 - math.sqrt(5.0)) / 1.0  # 2D golden angle


def radial_2d(n_spokes, n_read, rng=None):
    """Golden-angle radial spokes through the centre, coords in [-0.5,0.5)."""
    ang = np.arange(n_spokes) * (math.pi / ((1 + math.sqrt(5)) / 2))
    r = (np.arange(n_read) - n_read / 2) / n_read
    kx = np.outer(np.cos(ang), r).ravel()
    ky = np.outer(np.sin(ang), r).ravel()
    return np.stack([kx, ky]).astype(np.float32)


def kooshball_3d(n_spokes, n_read):
    """3D radial spokes with 2D golden-means directions (Chan et al. 2009)."""
    phi1, phi2 = 0.4656, 0.6823
    m = np.arange(n_spokes)
    z = (m * phi1) % 1.0 * 2 - 1
    az = 2 * math.pi * ((m * phi2) % 1.0)
    s = np.sqrt(np.maximum(0.0, 1 - z * z))
    d = np.stack([s * np.cos(az), s * np.sin(az), z], 1)
    r = (np.arange(n_read) - n_read / 2) / n_read
    k = d[:, None, :] * r[None, :, None]
    return np.ascontiguousarray(k.reshape(-1, 3).T).astype(np.float32)


def cplx(rng, *shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(
        np.complex64)


def gaussian_maps(n_coils, img_shape, rng):
    """Smooth complex coil maps normalised to unit root-sum-of-squares."""
    dim = len(img_shape)
    grids = np.meshgrid(*[np.linspace(-0.5, 0.5, n) for n in img_shape],
                        indexing="ij")
    maps = []
    for c in range(n_coils):
        if dim == 2:
            a = 2 * math.pi * c / n_coils
            cen = 0.6 * np.array([math.sin(a), math.cos(a)])
        else:
            v = rng.standard_normal(3)
            cen = 0.6 * v / np.linalg.norm(v)
        r2 = sum((g - cc) ** 2 for g, cc in zip(grids, cen))
        ramp = sum(rng.uniform(-2, 2) * g for g in grids)
        maps.append(np.exp(-r2 / 0.3) * np.exp(1j * ramp))
    maps = np.array(maps)
    rss = np.sqrt(np.sum(np.abs(maps) ** 2, 0))
    return (maps / rss).astype(np.complex64)


def rel_l2(a, b):
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def spiral_2d(n_interleaves, n_samples, rng):
    """Variable-density 2-D spiral (radius ~ u^1.6), ``n_interleaves``
    rotated arms, ``n_samples`` points in total, coords in [-0.5, 0.5)."""
    per = max(1, n_samples // n_interleaves)
    u = np.arange(per) / per
    turns = rng.uniform(6, 14)
    r = 0.499 * u ** 1.6
    arms = []
    for arm in range(n_interleaves):
        th = 2 * np.pi * (turns * u + arm / n_interleaves)
        arms.append(np.stack([r * np.cos(th), r * np.sin(th)]))
    return np.ascontiguousarray(np.concatenate(arms, 1), np.float32)
