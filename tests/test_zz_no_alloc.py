"""The no-allocation adjoint entry point against the regular one.

``gnufft_adjoint_convolution_noalloc`` serves callers that may not allocate
device memory while they run (real-time loops and serving workers that
reserve memory up front, code inside another framework's fixed memory
budget, callers that cannot take the synchronisation of cudaMalloc /
cudaFree).  It stages its scratch in a fixed array inside the library.
This test calls it through the C ABI twice in a row -- the second call with
other data, so stale contents of the shared array would show -- and checks
both results against ``gnufft_adjoint_device`` with GNUFFT_CONVOLUTION.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from tests.helpers import cplx, kooshball_3d, radial_2d, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.mark.parametrize("dims,traj_fn,n_coils,dens", [
    ((24, 24, 24), lambda: kooshball_3d(300, 48), 20, True),
    ((64, 64), lambda: radial_2d(48, 128), 3, False),
])
def test_noalloc_matches_regular_adjoint_twice(dims, traj_fn, n_coils, dens):
    torch = pytest.importorskip("torch")
    import gpunufft_b200 as G
    from gpunufft_b200 import _capi

    rng = np.random.default_rng(5)
    traj = traj_fn()
    M = traj.shape[1]
    w = rng.uniform(0.2, 1.0, M).astype(np.float32) if dens else None
    plan = G.Plan(traj, dims, 3, 8, 2.0, w, None, G.BALANCED)
    L = _capi.lib()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        k = torch.from_numpy(cplx(rng, n_coils, M)).cuda()
        out = torch.empty((n_coils,) + plan.grid_shape,
                          dtype=torch.complex64, device="cuda")
        _capi.check(L.gnufft_adjoint_convolution_noalloc(
            plan._h, ctypes.c_void_p(k.data_ptr()),
            ctypes.c_void_p(out.data_ptr()), n_coils,
            ctypes.c_void_p(stream)))
        exp = plan.adjoint(k, G.CONVOLUTION)
        torch.cuda.synchronize()
        assert rel_l2(out.cpu().numpy(), exp.cpu().numpy()) < TOL, call


def test_noalloc_rejects_requests_beyond_its_staging_area():
    torch = pytest.importorskip("torch")
    import gpunufft_b200 as G
    from gpunufft_b200 import _capi

    traj = kooshball_3d(512, 64)  # 32768 samples x 64 coil lanes = 16 MiB
    plan = G.Plan(traj, (16, 16, 16), 3, 8, 2.0, None, None, G.BALANCED)
    n_coils = 65  # -> 96 coil lanes: 24 MiB needed
    k = torch.zeros((n_coils, traj.shape[1]), dtype=torch.complex64,
                    device="cuda")
    out = torch.empty((n_coils,) + plan.grid_shape, dtype=torch.complex64,
                      device="cuda")
    st = _capi.lib().gnufft_adjoint_convolution_noalloc(
        plan._h, ctypes.c_void_p(k.data_ptr()),
        ctypes.c_void_p(out.data_ptr()), n_coils, None)
    assert st == _capi.ERROR_INVALID_ARGUMENT
    assert b"staging area" in _capi.lib().gnufft_last_error()
