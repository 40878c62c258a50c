"""Precomputed operators: export, save, load (upstream
loadPrecomputedGpuNUFFTOperator, gpuNUFFT_operator_factory.cpp:576-626, the
seven-array contract of the MATLAB path gpuNUFFT.m:101).

* a saved and reloaded plan gives bit-identical results (the adjoint sums
  every grid cell in a fixed order);
* tables produced by the upstream factory itself (its unstable-sort sample
  order) load and reproduce the oracle run on those tables within 1e-5;
* inconsistent tables are rejected with GNUFFT_ERROR_INVALID_ARGUMENT.
"""
import numpy as np
import pytest

from oracle import nufft_oracle as O
from oracle import ref as R
from tests.helpers import cplx, gaussian_maps, kooshball_3d, radial_2d, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5

CASES = [
    ((64, 64), lambda r: radial_2d(48, 128), 2.0, 3, 8),
    ((20, 20, 10), lambda r: r.uniform(-0.5, 0.5, (3, 4000)), 1.5, 3, 5),
    ((24, 24, 24), lambda r: kooshball_3d(300, 48), 2.0, 4, 8),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_save_load_round_trip(case, tmp_path):
    import gpunufft_b200 as G
    dims, mk, osf, kw, sw = CASES[case]
    rng = np.random.default_rng(40 + case)
    traj = np.asarray(mk(rng), np.float32)
    M = traj.shape[1]
    dens = rng.uniform(0.1, 1.0, M).astype(np.float32)
    maps = gaussian_maps(3, dims[::-1], rng)
    a = G.Plan(traj, dims, kw, sw, osf, dens, maps, G.BALANCED)
    path = tmp_path / "plan.npz"
    a.save(path)
    b = G.Plan.from_file(path, sens=maps)
    ta, tb = a.tables(), b.tables()
    for key in ("data_indices", "sector_data_count", "sector_centers",
                "traj_sorted", "dens_sorted", "deapo", "kernel_lut"):
        assert np.array_equal(ta[key], tb[key]), key
    k = cplx(rng, 3, M)
    ka = a.adjoint(k)
    assert np.array_equal(ka, b.adjoint(k))
    assert np.array_equal(ka, a.adjoint(k))        # repeatable
    x = cplx(rng, *dims[::-1])
    assert np.array_equal(a.forward(x), b.forward(x))


@pytest.mark.skipif(not R.available(), reason="upstream build absent")
@pytest.mark.parametrize("case", range(len(CASES)))
def test_load_upstream_factory_tables(case):
    """Tables from the upstream factory (useGpu=false) with its own sample
    order; deapodization from the oracle."""
    import gpunufft_b200 as G
    dims, mk, osf, kw, sw = CASES[case]
    rng = np.random.default_rng(60 + case)
    traj = np.asarray(mk(rng), np.float32)
    M = traj.shape[1]
    dens = rng.uniform(0.1, 1.0, M).astype(np.float32)
    up = R.sector_tables(traj, dims, osf, kw, sw, balance=True, dens=dens)
    g = O.make_geometry(dims, osf, kw, sw)
    deapo = O.deapodization(g, O.kernel_lut(osf, kw)).ravel()
    tables = dict(traj_sorted=up["traj_sorted"],
                  data_indices=up["data_indices"],
                  sector_data_count=up["sector_data_count"],
                  processing_order=up["order"],
                  sector_centers=up["centers"],
                  dens_sorted=up["dens_sorted"], deapo=deapo)
    p = G.Plan.load(tables, dims, kw, sw, osf)
    t = p.tables()
    assert np.array_equal(t["data_indices"], up["data_indices"])
    ref = O.OracleOperator(traj, dims, kw, sw, osf, dens=dens,
                           data_indices=up["data_indices"])
    k = cplx(rng, 2, M)
    for stage in (G.CONVOLUTION, G.DEAPODIZATION):
        err = rel_l2(p.adjoint(k, stage), ref.adjoint(k, stage))
        assert err < TOL, (stage, err)
    x = cplx(rng, 2, *dims[::-1])
    assert rel_l2(p.forward(x), ref.forward(x)) < TOL
    # the upstream order is also what REFERENCE_ORDER plan creation gives
    q = G.Plan(traj, dims, kw, sw, osf, dens, None, G.BALANCED,
               reference_order=True)
    assert np.array_equal(q.tables()["data_indices"], up["data_indices"])


def _good_tables(rng):
    import gpunufft_b200 as G
    dims = (32, 32)
    traj = radial_2d(32, 64)
    p = G.Plan(traj, dims, 3, 8, 2.0)
    t = p.tables()
    return dims, {k: t[k] for k in G.Plan.PLAN_ARRAYS}


@pytest.mark.parametrize("defect", ["not_permutation", "count_not_monotone",
                                    "count_short", "centers", "wrong_sector",
                                    "nan"])
def test_load_rejects_inconsistent_tables(defect):
    import gpunufft_b200 as G
    from gpunufft_b200 import _capi
    rng = np.random.default_rng(1)
    dims, t = _good_tables(rng)
    t = {k: (None if v is None else v.copy()) for k, v in t.items()}
    if defect == "not_permutation":
        t["data_indices"][1] = t["data_indices"][0]
    elif defect == "count_not_monotone":
        sdc = t["sector_data_count"]
        i = int(np.argmax(np.diff(sdc) > 0)) + 1
        sdc[i] = sdc[i - 1] - 1 if sdc[i - 1] > 0 else sdc[i + 1] + 1
    elif defect == "count_short":
        t["sector_data_count"][-1] -= 1
    elif defect == "centers":
        t["sector_centers"][0] += 1
    elif defect == "wrong_sector":
        # move the first sorted sample to the far corner of the k-space
        t["traj_sorted"][:, 0] = 0.49
    elif defect == "nan":
        t["traj_sorted"][0, 5] = np.nan
    with pytest.raises(_capi.GnufftError) as e:
        G.Plan.load(t, dims, 3, 8, 2.0)
    assert e.value.status == _capi.ERROR_INVALID_ARGUMENT
