"""The separable pruned transforms (default when every grid axis is a power
of two in [16, 1024]) against the cuFFT path of the same plan geometry
(GNUFFT_FLAG_CUFFT), every output stage, with and without maps, 2-D and
3-D, isotropic and anisotropic.  On these even grids the cuFFT path's
forward folds the FORWARD shift into the prepare pass as (-1)^(x+y+z)
and reads sector tiles by tensor copies, so this also checks that path.
Both are FP32 transforms of the same data; tolerance 1e-5 relative L2
(observed differences are at rounding level)."""
import numpy as np
import pytest

from tests.helpers import cplx, gaussian_maps, kooshball_3d, radial_2d, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5

CASES = [
    # dims, traj factory, coils, osf, kw
    ((64, 64), lambda r: radial_2d(64, 128), 3, 2.0, 3),
    ((32, 16), lambda r: r.uniform(-0.5, 0.5, (2, 2000)), 2, 2.0, 4),
    ((128, 128), lambda r: radial_2d(96, 256), 20, 2.0, 3),
    ((256, 256), lambda r: radial_2d(64, 512), 2, 2.0, 3),
    ((512, 512), lambda r: radial_2d(32, 1024), 1, 2.0, 3),
    ((16, 16, 16), lambda r: kooshball_3d(200, 32), 4, 2.0, 3),
    ((16, 32, 8), lambda r: r.uniform(-0.5, 0.5, (3, 3000)), 3, 2.0, 3),
    ((32, 32, 32), lambda r: kooshball_3d(500, 64), 33, 2.0, 3),
    ((64, 64, 64), lambda r: kooshball_3d(800, 128), 2, 2.0, 5),
    # odd image widths on power-of-two grids (15 * 2.1334 -> 32): odd
    # crop offsets, and column passes over N_x = 15 columns (no tensor
    # copies: rows of odd length are not 16-byte strided)
    ((15, 30), lambda r: radial_2d(40, 64), 3, 2.1334, 3),
    ((15, 15, 15), lambda r: kooshball_3d(300, 32), 20, 2.1334, 3),
]


@pytest.mark.parametrize("maps", [False, True])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_pruned_matches_cufft(case, maps):
    import gpunufft_b200 as G
    dims, mk, C, osf, kw = CASES[case]
    rng = np.random.default_rng(case)
    traj = np.asarray(mk(rng), np.float32)
    M = traj.shape[1]
    dens = rng.uniform(0.2, 1.0, M).astype(np.float32)
    sens = gaussian_maps(C, dims[::-1], rng) if maps else None
    a = G.Plan(traj, dims, kw, 8, osf, dens, sens, G.BALANCED)
    b = G.Plan(traj, dims, kw, 8, osf, dens, sens, G.BALANCED,
               use_cufft=True)
    k = cplx(rng, C, M)
    for stage in (G.FFT, G.DEAPODIZATION):
        err = rel_l2(a.adjoint(k, stage), b.adjoint(k, stage))
        assert err < TOL, (stage, err)
    x = cplx(rng, *dims[::-1]) if maps else cplx(rng, C, *dims[::-1])
    err = rel_l2(a.forward(x), b.forward(x))
    assert err < TOL, err


def test_persistent_row_pass_equals_the_kernel_it_replaces():
    """Forward with maps, 32 coils on a 64-point x axis: the row pass runs
    as persistent jobs of one image row x 32 coils (TMA rows).  With 8
    coils it runs the per-line kernel.  Every other stage of the forward
    works per coil, so each coil's output must be bitwise the same."""
    import gpunufft_b200 as G
    rng = np.random.default_rng(11)
    dims = (32, 32, 32)
    traj = np.asarray(kooshball_3d(400, 64), np.float32)
    C = 32
    sens = gaussian_maps(C, dims[::-1], rng)
    x = cplx(rng, *dims[::-1])
    full = G.Plan(traj, dims, 3, 8, 2.0, None, sens, G.BALANCED)
    y = full.forward(x)
    full.close()
    for c0 in range(0, C, 8):
        part = G.Plan(traj, dims, 3, 8, 2.0, None, sens[c0:c0 + 8],
                      G.BALANCED)
        yp = part.forward(x)
        part.close()
        assert np.array_equal(yp.view(np.uint64), y[c0:c0 + 8].view(np.uint64))


@pytest.mark.parametrize("C,maps", [(8, False), (5, False), (6, True)])
def test_paired_forward_equals_plain_layout(C, maps):
    """The default 3-D forward writes the grid with coil pairs interleaved:
    its z pass copies one 4-D box per tile, transforms only the listed
    column tiles and runs two columns per thread, and the interpolation
    reads coil-pair tiles in the plan's lane order.  A plan with 8-coil
    forward tiles keeps the plain layout (one column per thread, every
    column tile, single-coil tiles).  Per coil the arithmetic is the same,
    so the outputs must be bitwise equal (odd C: the last pair's second
    coil is an out-of-range box)."""
    import gpunufft_b200 as G
    rng = np.random.default_rng(13 + C)
    dims = (32, 32, 32)
    traj = np.asarray(kooshball_3d(300, 64), np.float32)  # empty columns
    dens = rng.uniform(0.2, 1.0, traj.shape[1]).astype(np.float32)
    sens = gaussian_maps(C, dims[::-1], rng) if maps else None
    x = cplx(rng, *dims[::-1]) if maps else cplx(rng, C, *dims[::-1])
    paired = G.Plan(traj, dims, 3, 8, 2.0, dens, sens, G.BALANCED)
    plain = G.Plan(traj, dims, 3, 8, 2.0, dens, sens, G.BALANCED,
                   tile_coils=8)
    try:
        a, b = paired.forward(x), plain.forward(x)
    finally:
        paired.close()
        plain.close()
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))
