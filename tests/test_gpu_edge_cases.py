"""Edge cases of the trajectory against the oracle, on power-of-two grids
(the fused spread, the coil-pair forward and the tensor-copy transform
passes): no samples (rejected), a single sample, samples piled into one
sector (forward work items split, dense grid rows), samples exactly on the
-0.5 edge and just below +0.5 (wrap-around), and 12, 16 and 32 coils (one
16- or 32-coil group of the spread, transformed in place on its
accumulator; several tile groups of the forward).  Tolerance as the other
parity tests: 1e-5 relative L2 against the FP64-accumulating oracle."""
import numpy as np
import pytest

from oracle import nufft_oracle as O
from tests.helpers import cplx, gaussian_maps, kooshball_3d, radial_2d, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _check(traj, dims, n_coils, seed):
    import gpunufft_b200 as G
    rng = np.random.default_rng(seed)
    traj = np.asarray(traj, np.float32)
    M = traj.shape[1]
    p = G.Plan(traj, dims, 3, 8, 2.0, None, None, G.BALANCED)
    ref = O.OracleOperator(traj, dims, 3, 8, 2.0)
    k = cplx(rng, n_coils, M)
    got = p.adjoint(k)
    exp = ref.adjoint(k)
    assert rel_l2(got, exp) < TOL, ("adjoint", rel_l2(got, exp))
    x = cplx(rng, n_coils, *ref.g.img_shape)
    got = p.forward(x)
    exp = ref.forward(x)
    assert rel_l2(got, exp) < TOL, ("forward", rel_l2(got, exp))
    p.close()


@pytest.mark.parametrize("dims", [(32, 32), (16, 16, 16)])
def test_no_samples_rejected(dims):
    import gpunufft_b200 as G
    from gpunufft_b200 import _capi
    traj = np.zeros((len(dims), 0), np.float32)
    with pytest.raises(_capi.GnufftError) as e:
        G.Plan(traj, dims, 3, 8, 2.0, None, None, G.BALANCED)
    assert e.value.status == _capi.ERROR_INVALID_ARGUMENT


@pytest.mark.parametrize("dims", [(32, 32), (16, 16, 16)])
def test_single_sample(dims):
    traj = np.full((len(dims), 1), 0.1234, np.float32)
    _check(traj, dims, 3, 1)


def test_samples_piled_in_one_sector():
    rng = np.random.default_rng(2)
    dims = (16, 16, 16)
    # 2000 samples within one sector of the 32^3 grid: one forward item per
    # 512 samples of that sector, grid rows with thousands of entries
    traj = rng.uniform(0.01, 0.05, (3, 2000)).astype(np.float32)
    _check(traj, dims, 5, 3)


@pytest.mark.parametrize("dims", [(32, 32), (16, 16, 16)])
def test_samples_on_the_edges(dims):
    rng = np.random.default_rng(4)
    d = len(dims)
    interior = rng.uniform(-0.5, 0.5, (d, 600))
    edge = rng.uniform(-0.5, 0.5, (d, 300))
    edge[rng.integers(0, d, 300), np.arange(300)] = -0.5
    top = rng.uniform(-0.5, 0.5, (d, 300))
    top[rng.integers(0, d, 300), np.arange(300)] = np.nextafter(
        np.float32(0.5), np.float32(0))
    traj = np.concatenate([interior, edge, top], 1).astype(np.float32)
    _check(traj, dims, 3, 5)


def test_thirty_two_coils_3d():
    rng = np.random.default_rng(6)
    traj = rng.uniform(-0.5, 0.5, (3, 3000)).astype(np.float32)
    _check(traj, (16, 16, 16), 32, 7)


@pytest.mark.parametrize("dims", [(32, 32), (16, 16, 16)])
@pytest.mark.parametrize("n_coils", [12, 16])
def test_sixteen_coil_group(dims, n_coils):
    rng = np.random.default_rng(8)
    traj = rng.uniform(-0.5, 0.5, (len(dims), 3000)).astype(np.float32)
    _check(traj, dims, n_coils, 9)


@pytest.mark.parametrize("dims", [(16, 16, 16), (48, 40)])
def test_coil_passes_under_a_memory_limit(dims):
    """A plan whose memory limit admits only a few coils' scratch runs a
    call in coil passes (the upstream's concurrent coil count,
    gpuNUFFT_operator.cpp:327-368): the same results as one pass, for the
    coil-combined adjoint, the per-coil stages and the forward; a limit
    below one coil's scratch still runs, one coil per pass."""
    import gpunufft_b200 as G
    from oracle import nufft_oracle as O
    rng = np.random.default_rng(31)
    C = 12
    traj = (kooshball_3d(200, 32) if len(dims) == 3 else
            radial_2d(48, 96)).astype(np.float32)
    g = O.make_geometry(dims, 2.0, 3, 8)
    maps = gaussian_maps(C, g.img_shape, rng)
    k = cplx(rng, C, traj.shape[1])
    x = cplx(rng, *g.img_shape)
    one = G.Plan(traj, dims, 3, 8, 2.0, None, maps, G.BALANCED)
    split = G.Plan(traj, dims, 3, 8, 2.0, None, maps, G.BALANCED)
    try:
        assert split.call_scratch_bytes(5) < split.call_scratch_bytes(C)
        exp_adj = one.adjoint(k)
        exp_fwd = one.forward(x)
        exp_fft = one.adjoint(k, G.FFT)
        for limit in (split.call_scratch_bytes(5), 1):
            split.set_memory_limit(limit)
            assert rel_l2(split.adjoint(k), exp_adj) < 1e-6
            assert rel_l2(split.forward(x), exp_fwd) < 1e-6
            assert rel_l2(split.adjoint(k, G.FFT), exp_fft) < 1e-6
    finally:
        one.close()
        split.close()
