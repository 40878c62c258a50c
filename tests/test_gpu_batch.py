"""Uneven operators run together, and the autotuner.

Persistent batches (one launch per stage for all instances, through
gnufft_batch_forward / gnufft_batch_adjoint) and stream graphs (the
instances' own launches captured on several streams) must give the results
of calling each operator directly: the stream graph holds the same kernels
(1e-6); the persistent batch runs every instance on the cuFFT transform
path with the shift folded into the gather, so results differ from the
operator's own path at rounding level (1e-5).  A second replay with new
inputs must agree too.  The autotuner must return a supported configuration
whose results agree with the default configuration within 1e-5 (sector
width changes the tile frame the upstream footprint arithmetic runs in, so
results differ at rounding level only).
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


TOL = {"persistent": 1e-5, "streams": 1e-6}


@pytest.mark.parametrize("mode", ["persistent", "streams"])
def test_graph_replay_matches_direct_calls(mode):
    from gpunufft_b200.batch import BatchedOperator
    plans, coils, torch = _build(10, 1, with_maps=True)
    bo = BatchedOperator(plans, coils, n_streams=4, mode=mode)
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
            assert ef < TOL[mode] and ea < TOL[mode], (rep, i, ef, ea)


@pytest.mark.parametrize("mode", ["persistent", "streams"])
def test_graph_without_maps_per_coil_outputs(mode):
    from gpunufft_b200.batch import BatchedOperator
    plans, coils, torch = _build(5, 2, with_maps=False)
    bo = BatchedOperator(plans, coils, n_streams=3, mode=mode)
    ks = [torch.randn((c, p.M), dtype=torch.complex64, device="cuda")
          for p, c in zip(plans, coils)]
    imgs = [torch.randn((c,) + p.img_shape, dtype=torch.complex64,
                        device="cuda") for p, c in zip(plans, coils)]
    adj = [o.clone() for o in bo.adjoint(ks)]
    fwd = [o.clone() for o in bo.forward(imgs)]
    for i, p in enumerate(plans):
        assert adj[i].shape == (coils[i],) + p.img_shape
        assert rel_l2(adj[i].cpu().numpy(),
                      p.adjoint(ks[i]).cpu().numpy()) < TOL[mode]
        assert rel_l2(fwd[i].cpu().numpy(),
                      p.forward(imgs[i]).cpu().numpy()) < TOL[mode]


def test_persistent_batch_frames_3d_density_texture():
    """Frames sharing one plan (each with its own data), a 3-D instance,
    density weights, kernel widths 3 and 5, odd and even grids, a TEXTURE
    operator: every instance against its own direct calls."""
    import torch

    import gpunufft_b200 as G
    from gpunufft_b200.batch import BatchedOperator, spiral_trajectory
    from tests.helpers import kooshball_3d
    rng = np.random.default_rng(11)
    t2 = spiral_trajectory(16, 20_000, rng)
    w2 = rng.uniform(0.3, 1.0, t2.shape[1]).astype(np.float32)
    frames = G.Plan(t2, (96, 96), 3, 8, 1.37, w2, None, G.BALANCED)
    maps = gaussian_maps(6, (120, 120), rng)
    wide = G.Plan(spiral_trajectory(24, 30_000, rng), (120, 120), 5, 12,
                  1.6, None, maps, G.BALANCED)
    tex = G.Plan(spiral_trajectory(12, 15_000, rng), (64, 64), 3, 8, 2.0,
                 None, None, G.BALANCED_TEXTURE)
    t3 = np.asarray(kooshball_3d(400, 64), np.float32)
    vol = G.Plan(t3, (32, 32, 32), 3, 8, 2.0, None, None, G.BALANCED)
    plans = [frames, wide, frames, tex, vol, frames]
    coils = [4, 6, 4, 3, 5, 4]
    bo = BatchedOperator(plans, coils)
    info = bo.info()
    assert info.n_instances == 6 and info.fft_calls == 6
    # prepare, then one interpolation launch for the 2-D and one for the
    # 3-D instances
    assert info.kernels_forward == 3 and info.kernels_adjoint == 3
    assert all(u > 0 for u in info.units) and info.device_bytes > 0
    imgs = [torch.randn(p.img_shape if p.n_sens else (c,) + p.img_shape,
                        dtype=torch.complex64, device="cuda")
            for p, c in zip(plans, coils)]
    ks = [torch.randn((c, p.M), dtype=torch.complex64, device="cuda")
          for p, c in zip(plans, coils)]
    fwd = [o.clone() for o in bo.forward(imgs)]
    adj = [o.clone() for o in bo.adjoint(ks)]
    torch.cuda.synchronize()
    for i, p in enumerate(plans):
        ef = rel_l2(fwd[i].cpu().numpy(), p.forward(imgs[i]).cpu().numpy())
        ea = rel_l2(adj[i].cpu().numpy(), p.adjoint(ks[i]).cpu().numpy())
        assert ef < 1e-5 and ea < 1e-5, (i, ef, ea)
    # frames of one plan: different data, different results
    assert rel_l2(fwd[0].cpu().numpy(), fwd[2].cpu().numpy()) > 0.1
    bo.close()


def test_batch_rejects_bad_arguments():
    import ctypes

    import gpunufft_b200 as G
    from gpunufft_b200 import _capi as C
    from gpunufft_b200.batch import spiral_trajectory
    rng = np.random.default_rng(3)
    maps = gaussian_maps(4, (64, 64), rng)
    p = G.Plan(spiral_trajectory(8, 5_000, rng), (64, 64), 3, 8, 2.0, None,
               maps, G.BALANCED)
    L = C.lib()
    h = ctypes.c_void_p()
    handles = (ctypes.c_void_p * 1)(p._h.value)
    bad = (ctypes.c_uint32 * 1)(3)  # the maps have 4 channels
    assert L.gnufft_batch_create(handles, bad, 1,
                                 ctypes.byref(h)) == C.ERROR_INVALID_ARGUMENT
    assert b"match the maps" in L.gnufft_last_error()
    ok = (ctypes.c_uint32 * 1)(4)
    assert L.gnufft_batch_create(handles, ok, 0,
                                 ctypes.byref(h)) == C.ERROR_INVALID_ARGUMENT
    C.check(L.gnufft_batch_create(handles, ok, 1, ctypes.byref(h)))
    null = (ctypes.c_void_p * 1)(None)
    assert L.gnufft_batch_forward(h, null, null,
                                  None) == C.ERROR_INVALID_ARGUMENT
    C.check(L.gnufft_batch_destroy(h))


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
