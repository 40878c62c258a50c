"""Differentiable operator: torch.autograd.Functions over the C ABI.

``forward`` y = A(k) x and ``adjoint`` x = A(k)^H y are differentiable in
their data argument (the backward of one is the other) and in the
trajectory k (the hand-written trajectory-gradient kernel,
``gnufft_traj_grad_device``).  Gradients follow torch's convention for
complex tensors (dL/dRe + i dL/dIm):

  forward:  dL/dx = A^H g,   dL/dk_a[j] = sum_c Re(conj(g[c,j]) dy[c,j]/dk_a[j])
  adjoint:  dL/dy = A v,     dL/dk_a[j] = sum_c Re(conj(y[c,j]) d(A v)[c,j]/dk_a[j])

where g = dL/dy and v = dL/dx.  A plan (sector tables, interpolation
matrix, cuFFT plans) is built from the trajectory's values; ``NUFFT``
rebuilds it only when the trajectory changes.
"""
from __future__ import annotations

from typing import Optional, Sequence

import numpy as np
import torch

from . import _capi as C
from .operator import Plan


class _Forward(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, traj, plan):
        ctx.plan = plan
        ctx.x_shape = x.shape
        ctx.save_for_backward(x)
        return plan.forward(x)

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, gy):
        (x,) = ctx.saved_tensors
        plan = ctx.plan
        gy = gy.contiguous()
        gx = gk = None
        if ctx.needs_input_grad[0]:
            gx = plan.adjoint(gy).reshape(ctx.x_shape)
        if ctx.needs_input_grad[1]:
            gk = plan.traj_grad(x, gy)
        return gx, gk, None


class _Adjoint(torch.autograd.Function):
    @staticmethod
    def forward(ctx, y, traj, plan):
        ctx.plan = plan
        ctx.y_shape = y.shape
        ctx.save_for_backward(y)
        return plan.adjoint(y)

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, gx):
        (y,) = ctx.saved_tensors
        plan = ctx.plan
        gx = gx.contiguous()
        gy = gk = None
        if ctx.needs_input_grad[0]:
            gy = plan.forward(gx).reshape(ctx.y_shape)
        if ctx.needs_input_grad[1]:
            gk = plan.traj_grad(gx, y)
        return gy, gk, None


def nufft_forward(x: torch.Tensor, traj: torch.Tensor, plan: Plan):
    """y = A(traj) x with a plan built from ``traj``'s values."""
    return _Forward.apply(x, traj, plan)


def nufft_adjoint(y: torch.Tensor, traj: torch.Tensor, plan: Plan):
    """x = A(traj)^H y with a plan built from ``traj``'s values."""
    return _Adjoint.apply(y, traj, plan)


class NUFFT(torch.nn.Module):
    """Differentiable gpuNUFFT operator for a (possibly learnable)
    trajectory (dim, M) float32 in [-0.5, 0.5).

    img_dims: (width, height[, depth]); sens: optional complex maps
    (coils, [depth,] height, width); dens: optional per-sample weights.
    """

    def __init__(self, img_dims: Sequence[int], kernel_width: int = 3,
                 sector_width: int = 8, osf: float = 2.0, sens=None,
                 dens=None, operator_type: int = C.BALANCED):
        super().__init__()
        self.img_dims = tuple(int(v) for v in img_dims)
        self.kernel_width = kernel_width
        self.sector_width = sector_width
        self.osf = osf
        self.operator_type = operator_type
        self.sens = None if sens is None else np.ascontiguousarray(
            torch.as_tensor(sens).detach().cpu().numpy(), np.complex64)
        self.dens = None if dens is None else np.ascontiguousarray(
            torch.as_tensor(dens).detach().cpu().numpy(), np.float32)
        self._plan: Optional[Plan] = None
        self._traj: Optional[torch.Tensor] = None  # copy the plan was built on
        self._key = None

    def plan_for(self, traj: torch.Tensor) -> Plan:
        """The plan of this trajectory, rebuilt only when it changed.  The
        same tensor unmodified since the last call (storage, version counter,
        shape, device) reuses the plan without looking at the values; any
        other tensor is compared with the plan's trajectory where it lives
        (on the GPU for CUDA tensors), and only a different trajectory is
        copied to the host to build a new plan."""
        t = traj.detach()
        key = (t.data_ptr(), t._version, tuple(t.shape), t.device)
        if self._plan is not None and key == self._key:
            return self._plan
        same = (self._plan is not None and self._traj is not None and
                self._traj.shape == t.shape and
                self._traj.device == t.device and
                bool(torch.equal(self._traj, t.to(self._traj.dtype))))
        if not same:
            if self._plan is not None:
                self._plan.close()
            dev = traj.device.index if traj.is_cuda else 0
            host = np.ascontiguousarray(t.cpu().numpy(), np.float32)
            self._plan = Plan(host, self.img_dims, self.kernel_width,
                              self.sector_width, self.osf, self.dens,
                              self.sens, self.operator_type, device=dev or 0)
            self._traj = t.to(torch.float32).clone()
        self._key = key
        return self._plan

    def forward(self, x: torch.Tensor, traj: torch.Tensor) -> torch.Tensor:
        return nufft_forward(x, traj, self.plan_for(traj))

    def adjoint(self, y: torch.Tensor, traj: torch.Tensor) -> torch.Tensor:
        return nufft_adjoint(y, traj, self.plan_for(traj))
