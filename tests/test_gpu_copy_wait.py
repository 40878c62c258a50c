"""Failure path of the bounded tile-copy waits, made to run out on purpose:
with the first wait of every block set to give up at once
(gnufft_set_copy_wait(plan, 0)), a host call reports GNUFFT_ERROR_CUDA for
itself, a device call reports it through gnufft_plan_check after the
caller synchronised its stream (once: the flag is cleared), and the
context stays usable: with the default bound restored the same plan
computes the right result.  The copies themselves complete normally; each
block waits for its copies in flight (full bound) before it returns."""
import ctypes

import numpy as np
import pytest

from oracle import nufft_oracle as O
from tests.helpers import cplx, gaussian_maps, kooshball_3d, rel_l2

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("C,maps", [(3, False), (32, True)])
def test_copy_wait_failure_is_reported_and_recoverable(C, maps):
    """(3, no maps): the column passes and the forward interpolation wait.
    (32, maps): the forward's first pass is the persistent row pass (jobs of
    one image row x 32 coils at this length) and the adjoint's last the
    persistent coil-sum pass, each with its own bounded waits."""
    torch = pytest.importorskip("torch")
    import gpunufft_b200 as G
    from gpunufft_b200 import _capi
    L = _capi.lib()
    rng = np.random.default_rng(4)
    dims = (16, 16, 16)  # grid 32^3: separable transforms, tensor copies
    traj = kooshball_3d(200, 32)
    sens = gaussian_maps(C, dims[::-1], rng) if maps else None
    p = G.Plan(traj, dims, 3, 8, 2.0, None, sens, G.BALANCED)
    ref = O.OracleOperator(traj, dims, 3, 8, 2.0, None, sens)
    x = cplx(rng, 16, 16, 16) if maps else cplx(rng, C, 16, 16, 16)
    k = cplx(rng, C, traj.shape[1])
    try:
        assert L.gnufft_set_copy_wait(p._h, 0) == _capi.SUCCESS
        with pytest.raises(RuntimeError, match="tile copy"):
            p.forward(x)
        with pytest.raises(RuntimeError, match="tile copy"):
            p.adjoint(k)
        # device call: reported after the stream is synchronised
        xd = torch.from_numpy(x).cuda()
        p.forward(xd)
        torch.cuda.synchronize()
        assert L.gnufft_plan_check(p._h) == _capi.ERROR_CUDA
        assert b"tile copy" in L.gnufft_last_error()
        assert L.gnufft_plan_check(p._h) == _capi.SUCCESS  # cleared
        # default bound again: correct results on the same plan
        assert L.gnufft_set_copy_wait(p._h, -1) == _capi.SUCCESS
        assert rel_l2(p.forward(x), ref.forward(x)) < 1e-5
        assert rel_l2(p.adjoint(k), ref.adjoint(k)) < 1e-5
        y = p.forward(xd)
        torch.cuda.synchronize()
        assert L.gnufft_plan_check(p._h) == _capi.SUCCESS
        assert rel_l2(y.cpu().numpy(), ref.forward(x)) < 1e-5
    finally:
        p.close()
