"""The CUDA path against fixtures produced by the upstream library itself
(tests/golden/make_golden.py): sector tables bit-exact (the upstream sample
order with GNUFFT_FLAG_REFERENCE_ORDER), and the upstream GPU operator's
coil-combined adjoint and forward within 1e-5 relative L2.  Needs neither
the upstream tree nor its build."""
import os

import numpy as np
import pytest

from tests.golden.make_golden import GPU_CASES, TABLE_CASES
from tests.helpers import rel_l2

pytestmark = pytest.mark.gpu
HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("case", range(len(TABLE_CASES)))
def test_tables_match_upstream_factory(case):
    import gpunufft_b200 as G
    gold = np.load(os.path.join(HERE, "upstream_cpu.npz"))
    name, dims, osf, kw, sw, _ = TABLE_CASES[case]
    traj = gold[f"{name}/traj"]
    p = G.Plan(traj, dims, kw, sw, osf, reference_order=True)
    t = p.tables()
    assert np.array_equal(t["sector_data_count"],
                          gold[f"{name}/sector_data_count"])
    assert np.array_equal(t["sector_centers"], gold[f"{name}/centers"])
    assert np.array_equal(t["data_indices"], gold[f"{name}/data_indices"])
    assert np.array_equal(t["processing_order"], gold[f"{name}/order"])
    assert np.array_equal(t["kernel_lut"], gold[f"lut_{osf}_{kw}"]) \
        if f"lut_{osf}_{kw}" in gold.files else True


@pytest.mark.skipif(not os.path.exists(os.path.join(HERE, "upstream_gpu.npz")),
                    reason="upstream GPU fixtures not generated")
@pytest.mark.parametrize("case", range(len(GPU_CASES)))
def test_operator_matches_upstream_gpu_fixture(case):
    import gpunufft_b200 as G
    gold = np.load(os.path.join(HERE, "upstream_gpu.npz"))
    name, dims, C, osf, kw, sw, _ = GPU_CASES[case]
    f = {k.split("/", 1)[1]: gold[k] for k in gold.files
         if k.startswith(name + "/")}
    p = G.Plan(f["traj"], dims, kw, sw, osf, f["dens"], f["maps"],
               G.BALANCED)
    assert rel_l2(p.adjoint(f["kspace"]), f["adjoint"]) < 1e-5
    assert rel_l2(p.forward(f["image"]), f["forward"]) < 1e-5
