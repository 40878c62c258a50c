"""The no-allocation adjoint entry point against the regular one.

``gnufft_adjoint_convolution_noalloc`` serves callers that may not allocate
device memory while they run (real-time loops and serving workers that
reserve memory up front, code inside another framework's fixed memory
budget, callers that cannot take the synchronisation of cudaMalloc /
cudaFree).  It stages its scratch in a fixed array inside the library.
This test calls it through the C ABI twice in a row -- the second call with
other data, so stale contents of the shared array would show -- and checks
both results against ``gnufft_adjoint_device`` with GNUFFT_CONVOLUTION, and
that the device's free memory (cudaMemGetInfo) is the same before and after
a warm call.  A request that fills the staging area exactly is accepted; one
beyond it is rejected.  This file is collected last on purpose.
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
    ks = [torch.from_numpy(cplx(rng, n_coils, M)).cuda() for _ in range(2)]
    outs = [torch.empty((n_coils,) + plan.grid_shape, dtype=torch.complex64,
                        device="cuda") for _ in range(2)]
    exps = [plan.adjoint(k, G.CONVOLUTION) for k in ks]
    torch.cuda.synchronize()
    free = []
    for call in range(2):
        free.append(torch.cuda.mem_get_info()[0])
        _capi.check(L.gnufft_adjoint_convolution_noalloc(
            plan._h, ctypes.c_void_p(ks[call].data_ptr()),
            ctypes.c_void_p(outs[call].data_ptr()), n_coils,
            ctypes.c_void_p(stream)))
        torch.cuda.synchronize()
        assert rel_l2(outs[call].cpu().numpy(),
                      exps[call].cpu().numpy()) < TOL, call
    # the warm call allocated nothing on the device
    assert torch.cuda.mem_get_info()[0] == free[1]


def test_noalloc_accepts_a_request_that_fills_its_staging_area():
    torch = pytest.importorskip("torch")
    import gpunufft_b200 as G
    from gpunufft_b200 import _capi

    rng = np.random.default_rng(9)
    traj = kooshball_3d(512, 64)  # 32768 samples
    plan = G.Plan(traj, (16, 16, 16), 3, 8, 2.0, None, None, G.BALANCED)
    n_coils = 64  # 64 coil lanes x 32768 samples x 8 bytes = 16 MiB exactly
    assert traj.shape[1] * n_coils * 8 == _capi.NOALLOC_SCRATCH_BYTES
    k = torch.from_numpy(cplx(rng, n_coils, traj.shape[1])).cuda()
    out = torch.empty((n_coils,) + plan.grid_shape, dtype=torch.complex64,
                      device="cuda")
    _capi.check(_capi.lib().gnufft_adjoint_convolution_noalloc(
        plan._h, ctypes.c_void_p(k.data_ptr()),
        ctypes.c_void_p(out.data_ptr()), n_coils,
        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    exp = plan.adjoint(k, G.CONVOLUTION)
    torch.cuda.synchronize()
    assert rel_l2(out.cpu().numpy(), exp.cpu().numpy()) < TOL


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
