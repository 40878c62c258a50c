"""CG-SENSE reconstruction on top of the operator.

Restates the upstream demo solver ``matlab/demo/utils/cg_sense_2d.m:40-108``
(and ``cg_sense_3d.m``), the multicoil form: the operator carries the
sensitivity maps, so

    rhs = A^H (y * sqrt(mask)),   M(x) = A^H A x + alpha x,

and ``maxit`` plain conjugate-gradient iterations from x = 0 (the upstream
loop ignores ``tol``; so does this one unless ``tol`` is given).  Pruessmann
et al., MRM 46:638-651 (2001).

All vector arithmetic runs in torch on the current CUDA stream; the operator
applications go through the C ABI on the same stream, so a whole solve is
stream-ordered and needs no host synchronisation until the caller reads the
result.
"""
from __future__ import annotations

from typing import Callable, Optional

import torch

from .operator import Plan


def _dot(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    """<a, b> = sum(conj(a) * b) as a 0-d complex tensor on the device."""
    return torch.vdot(a.reshape(-1), b.reshape(-1))


def cg_sense(plan: Plan, kspace: torch.Tensor, maxit: int = 10,
             alpha: float = 0.0, mask: Optional[torch.Tensor] = None,
             tol: Optional[float] = None,
             callback: Optional[Callable[[int, torch.Tensor], None]] = None
             ) -> torch.Tensor:
    """Reconstruct one image from multicoil k-space.

    plan:   operator with sensitivity maps (and, as in the upstream demos,
            usually with density compensation)
    kspace: complex64 CUDA tensor (n_coils, n_samples), original order
    maxit:  CG iterations (each one forward + one adjoint)
    alpha:  Tikhonov weight
    mask:   optional per-sample weights, applied as sqrt(mask) to the data
    tol:    stop early when ||r|| <= tol * ||rhs|| (upstream: not used)
    """
    if not plan.n_sens:
        raise ValueError("CG-SENSE needs a plan with sensitivity maps")
    y = kspace
    if mask is not None:
        y = y * torch.sqrt(mask.to(y.device, torch.float32))
    rhs = plan.adjoint(y)

    def apply_m(v: torch.Tensor) -> torch.Tensor:
        out = plan.adjoint(plan.forward(v))
        if alpha:
            out = out + alpha * v
        return out

    x = torch.zeros_like(rhs)
    r = rhs.clone()
    p = r.clone()
    rr = _dot(r, r).real
    stop = None if tol is None else (tol ** 2) * rr
    for it in range(maxit):
        ap = apply_m(p)
        a = rr / _dot(p, ap)
        x = x + a * p
        r = r - a * ap
        rr_new = _dot(r, r).real
        b = rr_new / rr
        rr = rr_new
        p = r + b * p
        if callback is not None:
            callback(it, x)
        if stop is not None and bool(rr <= stop):
            break
    return x
