"""The 3-D adjoint spread of whole grid rows with the inverse x transform
fused, for many-coil calls (17-40 coils, 32-coil groups) on grids 256 cells
wide: against the oracle and against the cuFFT path (which spreads into the
full grid), with runs that cross the grid edge, exact cell ties and a dense
k-space centre; kernel widths 3-5, texture weights, osf 1.6.  Repeated
calls are bitwise identical (fixed summation order)."""
import numpy as np
import pytest

from oracle import nufft_oracle as O
from tests.helpers import cplx, kooshball_3d, rel_l2

pytestmark = pytest.mark.gpu


def _traj(rng, kind, M):
    if kind == "uniform":
        t = rng.uniform(-0.5, 0.5, (3, M)).astype(np.float32)
        t[:, :64] = np.round(t[:, :64] * 16) / 16  # exact cell ties
        t[0, 64:96] = -0.5  # runs that cross the grid edge
        t[0, 96:128] = 0.49
        return t
    return kooshball_3d(M // 64, 64)


@pytest.mark.parametrize("C", [17, 32, 40])
@pytest.mark.parametrize("kind", ["uniform", "koosh"])
def test_rows_spread_vs_oracle_and_cufft(C, kind):
    import gpunufft_b200 as G
    rng = np.random.default_rng(C)
    dims = (128, 16, 8)  # grid 256 x 32 x 16 (separable transforms)
    traj = _traj(rng, kind, 12000)
    M = traj.shape[1]
    dens = rng.uniform(0.2, 1.0, M).astype(np.float32)
    p = G.Plan(traj, dims, 3, 8, 2.0, dens, None, G.BALANCED)
    q = G.Plan(traj, dims, 3, 8, 2.0, dens, None, G.BALANCED, use_cufft=True)
    ref = O.OracleOperator(traj, dims, 3, 8, 2.0, dens=dens)
    try:
        k = cplx(rng, C, M)
        for stage in (G.FFT, G.DEAPODIZATION):
            got = np.asarray(p.adjoint(k, stage))
            assert rel_l2(got, ref.adjoint(k, stage)) < 1e-5, stage
            assert rel_l2(got, np.asarray(q.adjoint(k, stage))) < 1e-5
            again = np.asarray(p.adjoint(k, stage))
            assert np.array_equal(again, got)
    finally:
        p.close()
        q.close()


@pytest.mark.parametrize("kw,osf,texture", [(5, 2.0, False), (3, 2.0, True),
                                            (4, 1.6, False)])
def test_rows_spread_kernel_widths(kw, osf, texture):
    import gpunufft_b200 as G
    rng = np.random.default_rng(kw)
    dims = (128, 8, 8) if osf == 2.0 else (160, 10, 10)  # 256 x 16 x 16
    traj = _traj(rng, "uniform", 9000)
    C = 24
    op = G.BALANCED_TEXTURE if texture else G.BALANCED
    p = G.Plan(traj, dims, kw, 8, osf, None, None, op)
    ref = O.OracleOperator(traj, dims, kw, 8, osf, texture=texture)
    try:
        k = cplx(rng, C, traj.shape[1])
        got = np.asarray(p.adjoint(k))
        # texture weights come from the texture unit; the oracle models its
        # filtering (8-bit weights from the float coordinate) within 6e-5
        tol = 6e-5 if texture else 1e-5
        assert rel_l2(got, ref.adjoint(k)) < tol
    finally:
        p.close()
