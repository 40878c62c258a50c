"""Continuous-batching CG-SENSE server: results alone and in the mix,
memory-based admission, resident operators per trajectory."""
import numpy as np
import pytest

from tests.helpers import cplx, gaussian_maps, kooshball_3d, radial_2d, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-6


def _requests():
    from gpunufft_b200.serving import Request
    rng = np.random.default_rng(9)
    specs = [  # (img dims, coils, trajectory, iterations)
        ((64, 64), 4, radial_2d(64, 128), 6),
        ((96, 96), 8, radial_2d(96, 192), 8),
        ((128, 128), 2, radial_2d(128, 256), 5),
        ((24, 24, 24), 6, kooshball_3d(400, 48), 4),
        ((64, 64), 3, radial_2d(64, 128), 7),   # same trajectory as #0
    ]
    reqs = []
    for i, (dims, C, traj, it) in enumerate(specs):
        shape = dims[::-1]
        reqs.append(Request(traj=traj, img_dims=dims,
                            kspace=cplx(rng, C, traj.shape[1]),
                            sens=gaussian_maps(C, shape, rng), n_iter=it,
                            arrival=0.002 * i, rid=i))
    return reqs


def _alone(req):
    import copy

    from gpunufft_b200.serving import Server
    s = Server(max_slots=1)
    try:
        r = copy.copy(req)
        r.arrival = 0.0
        (done,) = s.run([r])
        return done.result
    finally:
        s.close()


def test_results_alone_and_in_the_mix():
    from gpunufft_b200.serving import Server
    reqs = _requests()
    alone = {r.rid: _alone(r) for r in reqs}
    s = Server(max_slots=4)
    try:
        done = s.run(reqs)
        st = s.stats()
    finally:
        s.close()
    assert len(done) == len(reqs)
    assert st["max_concurrent"] >= 2          # requests overlapped
    assert st["plan_cache_hits"] + st["plan_cache_misses"] == len(reqs)
    for r in done:
        assert rel_l2(r.result, alone[r.rid]) < TOL, r.rid
    assert st["p99_ms"] >= st["p50_ms"] > 0
    # the admission accounting covers what requests and cached operators
    # actually held (operators' own figures plus allocated tensors)
    assert st["peak_admitted_gb"] >= st["peak_live_gb"] > 0


def test_results_match_the_direct_solver():
    import torch

    import gpunufft_b200 as G
    from gpunufft_b200.cg_sense import cg_sense
    req = _requests()[1]
    got = _alone(req)
    plan = G.Plan(req.traj, req.img_dims, 3, 8, 2.0, None, req.sens,
                  G.BALANCED)
    exp = cg_sense(plan, torch.from_numpy(req.kspace).cuda(),
                   maxit=req.n_iter).cpu().numpy()
    assert rel_l2(got, exp) < TOL


def test_memory_based_admission():
    from gpunufft_b200.serving import Server, request_bytes
    reqs = _requests()[:3]
    need = sorted(request_bytes(r) for r in reqs)
    # room for the two smallest at once, never for all three
    budget = need[0] + need[1] + need[0] // 2
    s = Server(max_slots=8, memory_budget=max(budget, need[2]))
    try:
        done = s.run(reqs)
        st = s.stats()
    finally:
        s.close()
    assert len(done) == 3
    assert st["max_concurrent"] <= 2
    assert st["peak_admitted_gb"] * 1e9 <= max(budget, need[2])
    big = _requests()[3]
    s2 = Server(memory_budget=request_bytes(big) - 1)
    with pytest.raises(ValueError):
        s2.submit(big)
    s2.close()


def test_operator_resident_per_trajectory():
    from gpunufft_b200.serving import Server
    reqs = [_requests()[0], _requests()[4]]
    reqs[1].arrival = 0.5                      # after #0 has finished
    s = Server(max_slots=4)
    try:
        s.run(reqs)
        st = s.stats()
    finally:
        s.close()
    assert st["plan_cache_misses"] == 1 and st["plan_cache_hits"] == 1


def test_operators_persist_on_disk(tmp_path):
    """A server with a plan directory writes one plan file per trajectory;
    a second server (fresh cache, same directory) loads them instead of
    sorting again, and gives the same results."""
    from gpunufft_b200.serving import Server
    reqs = _requests()[:4]  # four distinct trajectories, 2-D and 3-D
    first = Server(max_slots=2, plan_dir=str(tmp_path))
    try:
        done1 = {r.rid: r.result for r in first.run(reqs)}
        st1 = first.stats()
    finally:
        first.close()
    assert st1["plans_saved"] == 4 and st1["plans_loaded"] == 0
    assert len(list(tmp_path.glob("*.npz"))) == 4
    again = _requests()[:4]
    second = Server(max_slots=2, plan_dir=str(tmp_path))
    try:
        done2 = {r.rid: r.result for r in second.run(again)}
        st2 = second.stats()
    finally:
        second.close()
    assert st2["plans_loaded"] == 4 and st2["plans_saved"] == 0
    for rid, x in done1.items():
        assert rel_l2(done2[rid], x) < TOL, rid
