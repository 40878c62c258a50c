"""Differentiable operator: gradients in the data and in the trajectory.

References, at reduced size: the dense NUDFT matrix in FP64 torch (the model
the operator approximates: A[j, n] = sqrt(w_j) exp(-2 pi i k_j . r_n) /
sqrt(Ng) times the coil map, r_n centred) differentiated by torch autograd,
and FP64 central finite differences of the same dense loss.  The operator
is a Kaiser-Bessel approximation of that model, so the tolerances are set by
its accuracy.  At kernel width 7, osf 2 the kernel truncation error is
small and the nearest-entry lookup table of the upstream kernel (about
1,600 entries over the squared radius) dominates: ~2e-3 relative L2 against
the NUDFT.  Tolerances: 5e-3 for the data gradient, 2e-2 for the trajectory
gradient (the derivative of the kernel interpolation).
"""
import math

import numpy as np
import pytest

from tests.helpers import gaussian_maps, kooshball_3d, radial_2d, rel_l2

pytestmark = pytest.mark.gpu

TOL_X = 5e-3
TOL_K = 2e-2


def _dense_model(torch, traj, shape, maps, dens, grid_count):
    """y(x, k)[c, j] as a differentiable FP64 function."""
    dim = len(shape)
    axes = [torch.arange(n, dtype=torch.float64) - n // 2 for n in shape]
    mesh = torch.meshgrid(*axes, indexing="ij")
    # r: (dim, Npix) ordered x, y(, z) to match the trajectory rows
    r = torch.stack([m.reshape(-1) for m in mesh[::-1]], 0)
    sw = torch.sqrt(torch.as_tensor(dens, dtype=torch.float64))
    S = torch.as_tensor(maps).to(torch.complex128).reshape(maps.shape[0], -1)

    def model(x, k):
        ph = -2 * math.pi * (k.T @ r[:dim])          # (M, Npix)
        E = torch.polar(torch.ones_like(ph), ph)
        y = (S * x.reshape(1, -1)) @ E.T               # (C, M)
        return y * sw / math.sqrt(grid_count)
    return model


def _case(dim):
    rng = np.random.default_rng(21 + dim)
    if dim == 2:
        dims, shape, sw = (16, 16), (16, 16), 8
        traj = radial_2d(12, 16)
    else:
        # sector width 4 keeps the kw-7 sector tile within shared memory
        dims, shape, sw = (8, 8, 8), (8, 8, 8), 4
        traj = kooshball_3d(12, 8)
    traj = (traj * 0.9).astype(np.float32)
    M = traj.shape[1]
    maps = gaussian_maps(2, shape, rng)
    dens = rng.uniform(0.5, 1.0, M).astype(np.float32)
    return rng, dims, shape, traj, maps, dens, sw


@pytest.mark.parametrize("dim", [2, 3])
def test_forward_gradients_vs_dense_nudft_and_finite_differences(dim):
    import torch

    from gpunufft_b200.autograd import NUFFT
    rng, dims, shape, traj, maps, dens, sw = _case(dim)
    op = NUFFT(dims, kernel_width=7, sector_width=sw, osf=2.0, sens=maps,
               dens=dens)
    x0 = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape))
    y_obs = (rng.standard_normal((2, traj.shape[1])) +
             1j * rng.standard_normal((2, traj.shape[1])))
    # this library
    x = torch.tensor(x0, dtype=torch.complex64, device="cuda",
                     requires_grad=True)
    k = torch.tensor(traj, device="cuda", requires_grad=True)
    yo = torch.tensor(y_obs, dtype=torch.complex64, device="cuda")
    loss = (op(x, k) - yo).abs().pow(2).sum()
    loss.backward()
    # dense FP64 model
    Ng = int(np.prod([2 * n for n in shape]))
    model = _dense_model(torch, traj, shape, maps, dens, Ng)
    xd = torch.tensor(x0, dtype=torch.complex128, requires_grad=True)
    kd = torch.tensor(traj, dtype=torch.float64, requires_grad=True)
    yod = torch.tensor(y_obs, dtype=torch.complex128)
    ld = (model(xd, kd) - yod).abs().pow(2).sum()
    ld.backward()
    el = abs(float(loss.detach()) - float(ld)) / float(ld)
    ex = rel_l2(x.grad.cpu().numpy(), xd.grad.numpy())
    ek = rel_l2(k.grad.cpu().numpy(), kd.grad.numpy())
    assert el < TOL_X and ex < TOL_X and ek < TOL_K, (el, ex, ek)
    # FP64 central differences of the dense loss for a few coordinates
    h = 1e-6
    for a, j in [(0, 3), (1, 17), (dim - 1, traj.shape[1] - 5)]:
        kp = kd.detach().clone()
        km = kd.detach().clone()
        kp[a, j] += h
        km[a, j] -= h
        with torch.no_grad():
            fd = (float((model(xd, kp) - yod).abs().pow(2).sum()) -
                  float((model(xd, km) - yod).abs().pow(2).sum())) / (2 * h)
        assert abs(fd - float(kd.grad[a, j])) <= 1e-6 * max(1.0, abs(fd))
        scale = float(kd.grad.abs().max())
        assert abs(float(k.grad[a, j]) - fd) <= TOL_K * scale, (a, j)


@pytest.mark.parametrize("dim", [2, 3])
def test_adjoint_gradients_vs_dense_nudft(dim):
    import torch

    from gpunufft_b200.autograd import NUFFT
    rng, dims, shape, traj, maps, dens, sw = _case(dim)
    op = NUFFT(dims, kernel_width=7, sector_width=sw, osf=2.0, sens=maps,
               dens=dens)
    M = traj.shape[1]
    y0 = rng.standard_normal((2, M)) + 1j * rng.standard_normal((2, M))
    x_obs = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    y = torch.tensor(y0, dtype=torch.complex64, device="cuda",
                     requires_grad=True)
    k = torch.tensor(traj, device="cuda", requires_grad=True)
    xo = torch.tensor(x_obs, dtype=torch.complex64, device="cuda")
    loss = (op.adjoint(y, k) - xo).abs().pow(2).sum()
    loss.backward()
    Ng = int(np.prod([2 * n for n in shape]))
    model = _dense_model(torch, traj, shape, maps, dens, Ng)
    yd = torch.tensor(y0, dtype=torch.complex128, requires_grad=True)
    kd = torch.tensor(traj, dtype=torch.float64, requires_grad=True)
    xod = torch.tensor(x_obs, dtype=torch.complex128)
    # adjoint of the dense model: x = sum_c conj(S_c) * (E^H (sqrt(w) y_c))
    dim_ = len(shape)
    axes = [torch.arange(n, dtype=torch.float64) - n // 2 for n in shape]
    mesh = torch.meshgrid(*axes, indexing="ij")
    r = torch.stack([m.reshape(-1) for m in mesh[::-1]], 0)
    ph = 2 * math.pi * (kd.T @ r[:dim_])
    E = torch.polar(torch.ones_like(ph), ph)          # (M, Npix)
    S = torch.as_tensor(maps).to(torch.complex128).reshape(2, -1)
    sw = torch.sqrt(torch.as_tensor(dens, dtype=torch.float64))
    xdense = ((yd * sw) @ E / math.sqrt(Ng) * S.conj()).sum(0)
    ld = (xdense.reshape(shape) - xod).abs().pow(2).sum()
    ld.backward()
    ey = rel_l2(y.grad.cpu().numpy(), yd.grad.numpy())
    ek = rel_l2(k.grad.cpu().numpy(), kd.grad.numpy())
    assert ey < TOL_X and ek < TOL_K, (ey, ek)


def test_data_consistency_step_256_16coil():
    """The 2-D data-consistency loss at 256^2, 16 coils, 402 x 512 radial:
    gradients are finite and the data gradient equals A^H (2 (A x - y))
    (to rounding: autograd forms 2 (A x - y) through |.|^2)."""
    import torch

    from gpunufft_b200.autograd import NUFFT
    rng = np.random.default_rng(4)
    dims = (256, 256)
    traj = radial_2d(402, 512)
    maps = gaussian_maps(16, dims, rng)
    op = NUFFT(dims, 3, 8, 2.0, sens=maps)
    x_true = torch.tensor(rng.standard_normal(dims) +
                          1j * rng.standard_normal(dims),
                          dtype=torch.complex64, device="cuda")
    k = torch.tensor(traj, device="cuda", requires_grad=True)
    with torch.no_grad():
        y = op(x_true, k)
        y = y + 0.01 * y.abs().mean() * torch.randn_like(y)
    x = (0.5 * x_true).requires_grad_(True)
    loss = (op(x, k) - y).abs().pow(2).sum()
    loss.backward()
    assert torch.isfinite(k.grad).all()
    assert float(k.grad.abs().max()) > 0
    plan = op.plan_for(k)
    with torch.no_grad():
        ref = plan.adjoint(2 * (plan.forward(x) - y))
    assert rel_l2(x.grad.cpu().numpy(), ref.cpu().numpy()) < 1e-5


def test_plan_reuse_follows_the_trajectory():
    """The module rebuilds its plan only when the trajectory changes: the
    same tensor (or an equal one) reuses it, an in-place update or a new
    trajectory builds a new one, and results follow the trajectory."""
    import torch

    from gpunufft_b200.autograd import NUFFT
    traj = torch.from_numpy(radial_2d(16, 32)).cuda()
    op = NUFFT((16, 16))
    x = torch.randn(1, 16, 16, dtype=torch.complex64, device="cuda")
    y0 = op(x, traj)
    p0 = op._plan
    assert op(x, traj) is not None and op._plan is p0
    assert op(x, traj.clone()) is not None and op._plan is p0
    with torch.no_grad():
        traj[0, 3] += 0.01
    y1 = op(x, traj)
    assert op._plan is not p0
    assert rel_l2(y1.cpu().numpy(), y0.cpu().numpy()) > 1e-6
    p1 = op._plan
    fresh = NUFFT((16, 16))
    assert rel_l2(fresh(x, traj).cpu().numpy(), y1.cpu().numpy()) < 1e-6
    assert op(x, traj) is not None and op._plan is p1
