"""Uneven operators in one captured CUDA graph, and the autotuner.

Graph replays must give the same results as calling each operator directly
(the graph holds the same kernels); a second replay with new inputs must
too.  The autotuner must return a supported configuration whose results
agree with the default configuration within 1e-5 (sector width changes the
tile frame the upstream footprint arithmetic runs in, so results differ at
rounding level only).
"""
import numpy as np
import pytest

from tests.helpers import gaussian_maps, rel_l2

pytestmark = pytest.mark.gpu


def _build(n, seed, with_maps):
    import torch

    import gpunufft_b200 as G
    from gpunufft_b200.batch import spiral_instances
    rng = np.random.default_rng(seed)
    specs = spiral_instances(n, seed)
    plans, coils = [], []
    for s in specs:
        maps = (gaussian_maps(s["n_coils"], s["img_dims"][::-1], rng)
                if with_maps else None)
        plans.append(G.Plan(s["traj"], s["img_dims"], s["kernel_width"], 8,
                            s["osf"], None, maps, G.BALANCED))
        coils.append(s["n_coils"])
    return plans, coils, torch


def test_graph_replay_matches_direct_calls():
    from gpunufft_b200.batch import BatchedOperator
    plans, coils, torch = _build(10, 1, with_maps=True)
    bo = BatchedOperator(plans, coils, n_streams=4)
    for rep in range(2):
        imgs = [torch.randn(p.img_shape, dtype=torch.complex64,
                            device="cuda") for p in plans]
        ks = [torch.randn((c, p.M), dtype=torch.complex64, device="cuda")
              for p, c in zip(plans, coils)]
        fwd = [o.clone() for o in bo.forward(imgs)]
        adj = [o.clone() for o in bo.adjoint(ks)]
        torch.cuda.synchronize()
        for i, p in enumerate(plans):
            ef = rel_l2(fwd[i].cpu().numpy(), p.forward(imgs[i]).cpu().numpy())
            ea = rel_l2(adj[i].cpu().numpy(), p.adjoint(ks[i]).cpu().numpy())
            assert ef < 1e-6 and ea < 1e-6, (rep, i, ef, ea)


def test_graph_without_maps_per_coil_outputs():
    from gpunufft_b200.batch import BatchedOperator
    plans, coils, torch = _build(5, 2, with_maps=False)
    bo = BatchedOperator(plans, coils, n_streams=3)
    ks = [torch.randn((c, p.M), dtype=torch.complex64, device="cuda")
          for p, c in zip(plans, coils)]
    adj = [o.clone() for o in bo.adjoint(ks)]
    for i, p in enumerate(plans):
        assert adj[i].shape == (coils[i],) + p.img_shape
        assert rel_l2(adj[i].cpu().numpy(),
                      p.adjoint(ks[i]).cpu().numpy()) < 1e-6


def test_autotuner_choice_is_supported_and_consistent():
    import torch

    import gpunufft_b200 as G
    from gpunufft_b200.batch import autotune, spiral_instances
    s = spiral_instances(1, 5)[0]
    res = autotune(s["traj"], s["img_dims"], s["n_coils"],
                   s["kernel_width"], s["osf"], reps=2,
                   sector_widths=(4, 8, 12), tile_coils=(0, 4, 16))
    assert res.sector_width in (4, 8, 12)
    assert res.tile_coils in (0, 4, 16)
    assert len(res.table) >= 3 and res.ms > 0
    tuned = G.Plan(s["traj"], s["img_dims"], s["kernel_width"],
                   res.sector_width, s["osf"], tile_coils=res.tile_coils)
    ref = G.Plan(s["traj"], s["img_dims"], s["kernel_width"], 8, s["osf"])
    k = torch.randn((s["n_coils"], ref.M), dtype=torch.complex64,
                    device="cuda")
    x = torch.randn((s["n_coils"],) + ref.img_shape, dtype=torch.complex64,
                    device="cuda")
    assert rel_l2(tuned.adjoint(k).cpu().numpy(),
                  ref.adjoint(k).cpu().numpy()) < 1e-5
    assert rel_l2(tuned.forward(x).cpu().numpy(),
                  ref.forward(x).cpu().numpy()) < 1e-5


@pytest.mark.parametrize("tile_coils", [1, 2, 4, 8, 16, 32])
def test_forward_tile_shapes_agree(tile_coils):
    import torch

    import gpunufft_b200 as G
    from gpunufft_b200.batch import spiral_instances
    s = spiral_instances(1, 7)[0]
    ref = G.Plan(s["traj"], s["img_dims"], s["kernel_width"], 8, s["osf"])
    p = G.Plan(s["traj"], s["img_dims"], s["kernel_width"], 8, s["osf"],
               tile_coils=tile_coils)
    x = torch.randn((s["n_coils"],) + ref.img_shape, dtype=torch.complex64,
                    device="cuda")
    assert rel_l2(p.forward(x).cpu().numpy(),
                  ref.forward(x).cpu().numpy()) < 1e-6


@pytest.mark.parametrize("tile_coils", [1, 2, 4])
def test_forward_tile_shapes_agree_3d(tile_coils):
    """3-D: tiles of four coils run on the coil-pair grid, other tile widths
    on the plain grid; the interpolation arithmetic is the same."""
    import torch

    import gpunufft_b200 as G
    from tests.helpers import kooshball_3d
    traj = np.asarray(kooshball_3d(300, 64), np.float32)
    dims = (32, 32, 32)
    ref = G.Plan(traj, dims, 3, 8, 2.0)
    p = G.Plan(traj, dims, 3, 8, 2.0, tile_coils=tile_coils)
    x = torch.randn((5,) + ref.img_shape, dtype=torch.complex64,
                    device="cuda")
    assert rel_l2(p.forward(x).cpu().numpy(),
                  ref.forward(x).cpu().numpy()) < 1e-6
