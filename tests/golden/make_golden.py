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


def cpu_fixtures():
    out = {}
    for osf, kw in [(2.0, 3), (1.5, 4), (1.25, 5), (2.0, 7)]:
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


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpu", metavar="DIR", default=None)
    a = ap.parse_args()
    if not R.available():
        sys.exit("oracle/_ref is not built (oracle/build_ref.sh)")
    if a.gpu:
        gpu_fixtures(a.gpu)
    else:
        cpu_fixtures()
