"""Writes the golden fixtures of this directory from the upstream library
built from its own sources (oracle/build_ref.sh -> oracle/_ref).

  python tests/golden/make_golden.py            # upstream_cpu.npz (no GPU)
  python tests/golden/make_golden.py --gpu DIR  # upstream_gpu.npz into DIR
                                                # (needs a CUDA device)

upstream_cpu.npz: kernel lookup tables (load1DKernel), factory sector
tables (assignSectors / sortVector / computeSectorDataCount /
computeProcessingOrder / computeSectorCenters, useGpu=false) and the CPU
gridding routine gpuNUFFT_cpu for seeded trajectories.
upstream_gpu.npz: the upstream GPU operator (BALANCED, textures off) on
seeded small inputs: coil-combined adjoint and forward.
upstream_gpu_known.npz: the upstream GPU operator, all four operator types
(DEFAULT, BALANCED, TEXTURE, BALANCED_TEXTURE; the texture operators run
on the texture unit through oracle/ref_compat.h), on the inputs of the
upstream's own gtest known-answer cases (KNOWN_CASES): its outputs at the
entries the gtests check plus a strided sample of the rest.

  python tests/golden/make_golden.py --gpu-known DIR
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import nufft_oracle as O  # noqa: E402
from oracle import ref as R  # noqa: E402
from tests.helpers import cplx, gaussian_maps, kooshball_3d, radial_2d  # noqa

TABLE_CASES = [
    # name, dims, osf, kw, sw, trajectory factory
    ("2d64_radial", (64, 64), 2.0, 3, 8, lambda r: radial_2d(32, 128)),
    ("3d20x20x10_uniform", (20, 20, 10), 1.5, 3, 5,
     lambda r: r.uniform(-0.5, 0.5, (3, 1500))),
    ("3d16_koosh", (16, 16, 16), 2.0, 4, 8, lambda r: kooshball_3d(60, 24)),
]
GPU_CASES = [
    # name, dims, coils, osf, kw, sw, trajectory factory
    ("2d64_radial_4coil", (64, 64), 4, 2.0, 3, 8,
     lambda r: radial_2d(40, 128)),
    ("3d16_koosh_3coil", (16, 16, 16), 3, 2.0, 3, 8,
     lambda r: kooshball_3d(120, 32)),
]


# The upstream gtest known-answer cases (test/gpu/...), restated as inputs:
# name -> (trajectory, img dims, coils, kw, sw, osf, dens, sens,
#          direction, output stage, input, checked entries, gtest values)
# gtest values: (entry, expected real part, epsilon) the upstream asserts;
# None where the upstream's own code no longer produces the asserted value
# (the fixture then pins the value it does produce).
def _lin3(x, y, z, w):
    return x + w * (y + z * w)


def _lin2(x, y, w):
    return x + w * y


def known_cases():
    z3 = np.zeros((3, 1), np.float32)
    z2 = np.zeros((2, 1), np.float32)
    c1 = np.array([[-0.31719], [-0.38650], [0.0]], np.float32)
    c4 = np.array([[-0.31719, 0.0, 0.31719], [-0.38650, 0.0, 0.38650]],
                  np.float32)
    c8 = np.array([[-0.31719, 0.0, 0.25], [-0.38650, 0.0, 0.25]], np.float32)
    f2 = np.array([[0, 0, 0, 0.5, 0.3], [0, 0, 0, 0, 0.3], [0, 0, 0, 0, 0]],
                  np.float32)
    s8 = np.stack([np.full((32, 32), (c + 1) * (1 + 1j), np.complex64)
                   for c in range(8)])
    b1 = np.full((30, 32, 32), 1 + 0.2j, np.complex64)
    one = lambda *v: np.array(v, np.complex64)  # noqa: E731
    return {
        # gpuNUFFT_fft_tests.cpp:142-200, epsilon 0.01 (x10 for the last 3)
        "fft_1sector": (z3, (10, 10, 10), 1, 3, 5, 1.0, None, None, "adj", 1,
                        one(1 + 1j),
                        [_lin3(5, 5, 5, 10), _lin3(5, 4, 5, 10),
                         _lin3(4, 5, 5, 10), _lin3(0, 1, 5, 10)],
                        [(0, 0.2172, 0.01), (1, 0.1975, 0.1),
                         (2, 0.1975, 0.1), (3, 0.001619, 0.1)]),
        # :217-271
        "fft_k5w64": (z3, (64, 64, 64), 1, 5, 8, 1.0, None, None, "adj", 1,
                      one(1), [_lin3(57, 33, 32, 64)], [(0, 0.0001, 0.1)]),
        # :290-381
        "fft_factor2": (f2, (16, 16, 16), 1, 3, 8, 1.0, None, None, "adj", 1,
                        one(0.5 + 0.5j, 0.5 + 0.5j, 1 + 1j, 1 + 1j, 1 + 1j),
                        [_lin3(8, 8, 5, 16), _lin3(2, 2, 5, 16),
                         _lin3(4, 3, 5, 16)],
                        [(0, 0.28397, 0.01), (1, 0.0039668, 0.01),
                         (2, 0.0159846, 0.01)]),
        # gpuNUFFT_deapo_tests.cpp:89-152 (asserts 0.00637)
        "deapo_1sector": (z3, (64, 64, 64), 1, 3, 8, 1.75, None, None, "adj",
                          2, one(1), [_lin3(10, 0, 16, 64)], None),
        # :161-243 (asserts 0.005513 and coil 1 == coil 0)
        "deapo_2coils": (z3, (32, 32, 32), 2, 3, 8, 2.0, None, None, "adj", 2,
                         one(1, 1),
                         [_lin3(i, j, 16, 32) + c * 32768
                          for c in (0, 1) for i, j in
                          ((0, 0), (10, 0), (0, 5), (4, 4), (15, 14))], None),
        # :255-332 (30 coils, textures on: every coil equal)
        "deapo_2d_30coil": (z2, (32, 32), 30, 3, 8, 2.0, None, None, "adj", 2,
                            np.full(30, 1 + 0.5j, np.complex64),
                            [_lin2(i, j, 32) + c * 1024
                             for c in (0, 15, 29) for i, j in
                             ((10, 0), (0, 5), (4, 4), (15, 14))], None),
        # :342-429 (asserts 1.03125 for the b1-combined pixel 0)
        "deapo_2d_b1": (z2, (32, 32), 30, 3, 8, 2.0, np.ones(1, np.float32),
                        b1, "adj", 2, np.full(30, 1 + 0.5j, np.complex64),
                        [0, 17, 527], None),
        # gpuNUFFT_forward_tests.cpp:12-83, epsilon 0.02
        "fwd_1sector": (c1, (32, 32, 32), 1, 5, 8, 1.25, None, None, "fwd", 2,
                        np.full((1, 32, 32, 32), 1 + 1j, np.complex64), [0],
                        [(0, 0.0001973, 0.02)]),
        # :85-165 (two channels, equal)
        "fwd_1sector_2ch": (c1, (32, 32, 32), 2, 5, 8, 1.25, None, None,
                            "fwd", 2,
                            np.full((2, 32, 32, 32), 1 + 1j, np.complex64),
                            [0, 1], [(0, 0.0001973, 0.02)]),
        # :167-256 (asserts 0.816 textures / 0.73328 otherwise)
        "fwd_2d_32_4": (c4, (32, 32), 4, 5, 8, 1.25, None, None, "fwd", 2,
                        np.full((4, 32, 32), 1 + 1j, np.complex64),
                        list(range(12)), None),
        # :258-383 (coil c = (c + 1) x coil 0)
        "fwd_2d_32_8_sens": (c8, (32, 32), 8, 5, 8, 1.25,
                             np.ones(3, np.float32), s8, "fwd", 2,
                             np.full((32, 32), 1 + 1j, np.complex64),
                             list(range(24)), None),
        # gpuNUFFT_2D_conv_tests.cpp:1093-1204, epsilon 0.01
        "conv2d_256x128_30": (z2, (256, 128), 30, 3, 8, 1.0, None, None,
                              "adj", 0, np.full(30, 1 + 0.5j, np.complex64),
                              [_lin2(128, 64, 256) + c * 32768
                               for c in (0, 29)] +
                              [_lin2(127, 64, 256) + c * 32768
                               for c in (0, 29)],
                              [(0, 1.0, 0.01), (1, 1.0, 0.01),
                               (2, 0.45, 0.01), (3, 0.45, 0.01)]),
    }


# upstream operator types in the order (textures, balanced)
KNOWN_MODES = [(False, False), (False, True), (True, False), (True, True)]


def cpu_fixtures():
    out = {}
    for osf, kw in [(2.0, 3), (1.5, 4), (1.25, 5), (2.0, 7), (1.0, 3)]:
        out[f"lut_{osf}_{kw}"] = R.kernel_lut(osf, kw)
    for i, (name, dims, osf, kw, sw, mk) in enumerate(TABLE_CASES):
        rng = np.random.default_rng(1000 + i)
        traj = np.ascontiguousarray(mk(rng), np.float32)
        t = R.sector_tables(traj, dims, osf, kw, sw, balance=True)
        out[f"{name}/traj"] = traj
        for k in ("assigned", "data_indices", "sector_data_count", "centers",
                  "order"):
            out[f"{name}/{k}"] = t[k]
    # gpuNUFFT_cpu (3-D isotropic; drops contributions beyond the grid
    # edge, so the trajectory stays inside |k| < 0.4): one coil on 16^3
    name, dims, osf, kw, sw, _ = TABLE_CASES[2]
    traj = np.ascontiguousarray(0.8 * kooshball_3d(60, 24), np.float32)
    out["cpu_gridding/traj"] = traj
    rng = np.random.default_rng(77)
    k = cplx(rng, 1, traj.shape[1])[0]
    g = O.make_geometry(dims, osf, kw, sw)
    tab = O.build_tables(traj, g)
    data = np.ascontiguousarray(k[tab.data_indices])
    grid = np.zeros(g.grid_count, np.complex64)
    R.cpu_gridding(data, np.ascontiguousarray(tab.traj_sorted.T),
                   O.kernel_lut(osf, kw), tab.sector_data_count, tab.centers,
                   sw, kw, g.grid[0], grid)
    out["cpu_gridding/kspace"] = k
    out["cpu_gridding/grid"] = grid
    np.savez_compressed(os.path.join(HERE, "upstream_cpu.npz"), **out)


def gpu_fixtures(dest):
    out = {}
    for i, (name, dims, C, osf, kw, sw, mk) in enumerate(GPU_CASES):
        rng = np.random.default_rng(2000 + i)
        traj = np.ascontiguousarray(mk(rng), np.float32)
        M = traj.shape[1]
        dens = rng.uniform(0.2, 1.0, M).astype(np.float32)
        maps = gaussian_maps(C, dims[::-1], rng)
        k = cplx(rng, C, M)
        x = cplx(rng, *dims[::-1])
        op = R.RefGpuOperator(traj, dims, C, kw, sw, osf, dens=dens,
                              sens=maps, balance=True)
        try:
            adj = op.adjoint(k, 2)
            fwd = op.forward(x)
        finally:
            op.close()
        for key, val in dict(traj=traj, dens=dens, maps=maps, kspace=k,
                             image=x, adjoint=adj, forward=fwd).items():
            out[f"{name}/{key}"] = val
    np.savez_compressed(os.path.join(dest, "upstream_gpu.npz"), **out)


def known_outputs(op, case):
    """Run one known-answer case on an operator with the harness / Plan
    calling convention (adjoint(k, stage) / forward(x, stage))."""
    traj, dims, C, kw, sw, osf, dens, sens, way, stage, x = case[:11]
    if way == "adj":
        return np.asarray(op.adjoint(x.reshape(C, -1), stage)).ravel()
    return np.asarray(op.forward(x, stage)).ravel()


def gpu_known_fixtures(dest):
    out = {}
    for name, case in known_cases().items():
        traj, dims, C, kw, sw, osf, dens, sens = case[:8]
        for tex, bal in KNOWN_MODES:
            op = R.RefGpuOperator(traj, dims, C, kw, sw, osf, dens=dens,
                                  sens=sens, balance=bal, textures=tex)
            try:
                way, stage = case[8], case[9]
                if way == "adj":
                    ch = 1 if (sens is not None and stage >= 1) else C
                    n = ch * int(np.prod([int(v * osf) if stage in (0, 3)
                                          else v for v in dims]))
                    y = op.adjoint(case[10].reshape(C, -1), stage, out_len=n)
                else:
                    y = op.forward(case[10], stage).ravel()
            finally:
                op.close()
            idx = np.unique(np.concatenate(
                [np.asarray(case[11], np.int64),
                 np.arange(0, y.size, max(1, y.size // 4096))]))
            key = f"{name}/{int(tex)}{int(bal)}"
            out[key + "/idx"] = idx
            out[key + "/val"] = y[idx]
    np.savez_compressed(os.path.join(dest, "upstream_gpu_known.npz"), **out)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpu", metavar="DIR", default=None)
    ap.add_argument("--gpu-known", metavar="DIR", default=None)
    a = ap.parse_args()
    if not R.available():
        sys.exit("oracle/_ref is not built (oracle/build_ref.sh)")
    if a.gpu:
        gpu_fixtures(a.gpu)
    elif a.gpu_known:
        gpu_known_fixtures(a.gpu_known)
    else:
        cpu_fixtures()
