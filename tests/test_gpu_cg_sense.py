"""CG-SENSE (matlab/demo/utils/cg_sense_2d.m:40-108) on the GPU operator
against the same loop on the oracle operator.

Tolerance: 1e-4 relative L2 after the stated iterations.  Each operator
application agrees with the oracle to ~1e-6; CG is a nonlinear function of
the operator and amplifies such differences by up to the condition number
of the normal equations over the iterations run.
"""
import numpy as np
import pytest

from oracle import nufft_oracle as O
from tests.helpers import gaussian_maps, kooshball_3d, radial_2d, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-4


def _phantom(shape):
    grids = np.meshgrid(*[np.linspace(-1, 1, n) for n in shape],
                        indexing="ij")
    r2 = sum(g * g for g in grids)
    img = (r2 < 0.6).astype(np.float64) + 0.5 * (
        sum((g - 0.2) ** 2 for g in grids) < 0.05)
    return (img * np.exp(1j * grids[-1])).astype(np.complex64)


def _ramp(traj):
    r = np.sqrt((traj.astype(np.float64) ** 2).sum(0))
    return np.maximum(r / r.max(), 1e-3).astype(np.float32)


@pytest.mark.parametrize("case", ["2d64_radial_4coil", "3d16_koosh_2coil"])
def test_cg_sense_matches_oracle_loop(case):
    import torch

    import gpunufft_b200 as G
    from gpunufft_b200.cg_sense import cg_sense
    rng = np.random.default_rng(7)
    if case.startswith("2d"):
        dims, C, traj, maxit = (64, 64), 4, radial_2d(96, 128), 10
    else:
        dims, C, traj, maxit = (16, 16, 16), 2, kooshball_3d(300, 32), 6
    shape = dims[::-1]
    maps = gaussian_maps(C, shape, rng)
    dens = _ramp(traj)
    x_true = _phantom(shape)
    ora = O.OracleOperator(traj, dims, 3, 8, 2.0, dens=dens, sens=maps)
    y = ora.forward(x_true).astype(np.complex64)
    y += (0.01 * np.abs(y).mean() * (rng.standard_normal(y.shape) + 1j *
          rng.standard_normal(y.shape))).astype(np.complex64)
    plan = G.Plan(traj, dims, 3, 8, 2.0, dens, maps, G.BALANCED)
    y_d = torch.from_numpy(y).cuda()
    x_gpu = cg_sense(plan, y_d, maxit=maxit, alpha=1e-3).cpu().numpy()
    x_ora = O.cg_sense(ora, y, maxit=maxit, alpha=1e-3)
    assert rel_l2(x_gpu, x_ora) < TOL, rel_l2(x_gpu, x_ora)


def test_cg_sense_reduces_the_residual_and_beats_the_adjoint():
    import torch

    import gpunufft_b200 as G
    from gpunufft_b200.cg_sense import cg_sense
    rng = np.random.default_rng(8)
    dims, C = (64, 64), 8
    traj = radial_2d(128, 128)
    shape = dims[::-1]
    maps = gaussian_maps(C, shape, rng)
    dens = _ramp(traj)
    x_true = torch.from_numpy(_phantom(shape)).cuda()
    plan = G.Plan(traj, dims, 3, 8, 2.0, dens, maps, G.BALANCED)
    y = plan.forward(x_true)
    res = []

    def cb(it, x):
        res.append(float(torch.linalg.vector_norm(plan.forward(x) - y)))
    x = cg_sense(plan, y, maxit=15, callback=cb)
    assert all(b <= a * 1.0001 for a, b in zip(res, res[1:])), res
    err_cg = float(torch.linalg.vector_norm(x - x_true) /
                   torch.linalg.vector_norm(x_true))
    # best scalar multiple of the plain adjoint
    xa = plan.adjoint(y)
    s = torch.vdot(xa.reshape(-1), x_true.reshape(-1)) / torch.vdot(
        xa.reshape(-1), xa.reshape(-1))
    err_adj = float(torch.linalg.vector_norm(s * xa - x_true) /
                    torch.linalg.vector_norm(x_true))
    assert err_cg < err_adj, (err_cg, err_adj)
