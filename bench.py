#!/usr/bin/env python
"""Benchmark of the gpuNUFFT operator path on B200.

Workload (default): 3D 128^3 image, osf 2, Kaiser-Bessel width 3, sector
width 8, 32 coils; kooshball trajectory of 8192 spokes x 256 readout points
(2,097,152 samples, 2D golden-means directions); complex64 N(0,1) k-space;
32 Gaussian-profile sensitivity maps with random phase ramps, unit
root-sum-of-squares.  One step = one forward (image -> 32-coil k-space) plus
one adjoint (32-coil k-space -> coil-combined image).  Synthetic, seeded
data of the published configuration's shape.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints ONE JSON line (rank 0).  For N > 1 (torchrun) every rank runs an
independent replica (the path has no cross-GPU exchange); value = all steps
/ the slowest rank's time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = ("fwd+adj/s 3D 128³×32coil batched vs plain; %HBM peak; "
          "served p99 @1e-5 err")
UNIT = "fwd+adj/s"

WORKLOADS = {
    # name: (img dims, n_coils, spokes, readout, osf, kw, sw)
    "3d128x32": ((128, 128, 128), 32, 8192, 256, 2.0, 3, 8),
    # smaller 3D cases of the same kernels, for profiler captures
    "3d96x32": ((96, 96, 96), 32, 4608, 192, 2.0, 3, 8),
    "3d64x8": ((64, 64, 64), 8, 2048, 128, 2.0, 3, 8),
    "3d64x32": ((64, 64, 64), 32, 2048, 128, 2.0, 3, 8),
    # 2D single-coil case (upstream CPU-runnable configuration)
    "2d128x1": ((128, 128), 1, 64, 256, 2.0, 3, 8),
}


def kooshball(n_spokes, n_read):
    phi1, phi2 = 0.4656, 0.6823
    m = np.arange(n_spokes)
    z = (m * phi1) % 1.0 * 2 - 1
    az = 2 * math.pi * ((m * phi2) % 1.0)
    s = np.sqrt(np.maximum(0.0, 1 - z * z))
    d = np.stack([s * np.cos(az), s * np.sin(az), z], 1)
    r = (np.arange(n_read) - n_read / 2) / n_read
    k = d[:, None, :] * r[None, :, None]
    return np.ascontiguousarray(k.reshape(-1, 3).T).astype(np.float32)


def radial2d(n_spokes, n_read):
    ang = np.arange(n_spokes) * (math.pi / ((1 + math.sqrt(5)) / 2))
    r = (np.arange(n_read) - n_read / 2) / n_read
    return np.stack([np.outer(np.cos(ang), r).ravel(),
                     np.outer(np.sin(ang), r).ravel()]).astype(np.float32)


def make_inputs(name, seed=0):
    dims, C, ns, nr, osf, kw, sw = WORKLOADS[name]
    rng = np.random.default_rng(seed)
    traj = kooshball(ns, nr) if len(dims) == 3 else radial2d(ns, nr)
    M = traj.shape[1]
    shape = tuple(dims[::-1])
    grids = np.meshgrid(*[np.linspace(-0.5, 0.5, n, dtype=np.float32)
                          for n in shape], indexing="ij")
    maps = np.empty((C,) + shape, np.complex64)
    rss = np.zeros(shape, np.float32)
    for c in range(C):
        v = rng.standard_normal(len(shape))
        cen = 0.6 * v / np.linalg.norm(v)
        r2 = sum((g - cc) ** 2 for g, cc in zip(grids, cen))
        ramp = sum(np.float32(rng.uniform(-2, 2)) * g for g in grids)
        maps[c] = np.exp(-r2 / 0.3) * np.exp(1j * ramp)
        rss += np.abs(maps[c]) ** 2
    maps /= np.sqrt(rss)
    k = (rng.standard_normal((C, M), dtype=np.float32) +
         1j * rng.standard_normal((C, M), dtype=np.float32)).astype(
             np.complex64)
    x = (rng.standard_normal(shape, dtype=np.float32) +
         1j * rng.standard_normal(shape, dtype=np.float32)).astype(
             np.complex64)
    return dict(traj=traj, maps=maps, k=k, x=x, dims=dims, C=C, M=M, osf=osf,
                kw=kw, sw=sw)


# --------------------------------------------------------------------------
# clocks during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,"
         "clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device),
                 "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
            return self
        # the timed region starts once the sampler reports (at most 5 s)
        t_end = time.monotonic() + 5.0
        while (not self.lines and self.proc.poll() is None
               and time.monotonic() < t_end):
            time.sleep(0.01)
        self.lines.clear()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        for ln in self.lines:
            f = [v.strip() for v in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [],
                    "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# --------------------------------------------------------------------------
# CPU reference (upstream gpuNUFFT_cpu, built from the upstream sources)
# --------------------------------------------------------------------------
def cpu_reference(inp, threads, coils_per_step=None):
    """Time the upstream CPU gridding routine (adjoint convolution of one
    coil; the upstream has no CPU forward, FFT or deapodization) on
    ``threads`` host threads, one coil per thread.  Returns (seconds for
    one coil pass per thread-slot, coils done)."""
    from oracle import nufft_oracle as O
    from oracle import ref
    if not ref.available():
        raise RuntimeError("oracle/_ref not built")
    dims, osf, kw, sw = inp["dims"], inp["osf"], inp["kw"], inp["sw"]
    if len(dims) == 2:  # exact 3D embedding of the 2D problem (z = 0)
        traj = np.concatenate([inp["traj"],
                               np.zeros((1, inp["M"]), np.float32)])
        gdims = (dims[0], dims[1], dims[0])
    else:
        traj, gdims = inp["traj"], dims
    g = O.make_geometry(gdims, osf, kw, sw)
    t = O.build_tables(traj, g)
    lut = O.kernel_lut(osf, kw)
    crds = np.ascontiguousarray(t.traj_sorted.T)
    data = [np.ascontiguousarray(inp["k"][c % inp["C"]][t.data_indices])
            for c in range(threads)]
    grids = [np.zeros(g.grid_count, np.complex64) for _ in range(threads)]

    def one(i):
        grids[i][:] = 0
        ref.cpu_gridding(data[i], crds, lut, t.sector_data_count, t.centers,
                         sw, kw, g.grid[0], grids[i])

    def step(n=threads):
        ths = [threading.Thread(target=one, args=(i,)) for i in
               range(n)]
        t0 = time.perf_counter()
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        return time.perf_counter() - t0
    return step


def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference_arm(args, rank):
    if rank != 0:
        return
    inp = make_inputs(args.workload)
    C = inp["C"]
    threads = min(cpu_threads(), C)
    step = cpu_reference(inp, threads)
    for _ in range(args.warmup):
        step()
    ts = [step() for _ in range(args.steps)]
    per_pass = statistics.mean(ts)  # `threads` coils gridded per step
    # one fwd+adj on C coils = 2*C gridding passes (forward counted like the
    # adjoint; FFT, deapodization and coil combine not counted)
    value = threads / (per_pass * 2 * C)
    sample = (f"upstream gpuNUFFT_cpu adjoint gridding of {threads} coil(s) "
              f"per step ({inp['M']} samples each) on {threads} thread(s); "
              f"fwd+adj/s = coils per second / (2 x {C} coils); FFT and "
              f"deapodization not counted")
    line = {"impl": "reference", "metric": METRIC, "value": value,
            "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_pass * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_label(args.workload)},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads,
                             "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def reference_gpu(inp, steps):
    """fwd+adj/s of the upstream GPU operator (BALANCED, textures off) on
    this workload, host arrays in and out like its API; None fields when the
    upstream build is absent."""
    from oracle import ref
    note = ("upstream BALANCED operator built from its sources for sm_100a "
            "(textures off); host arrays per call as its API takes them; "
            "CUDA events on the default stream (value) and wall clock")
    if not ref.available():
        return {"value": None, "unit": UNIT, "note": note + ": not built"}
    op = ref.RefGpuOperator(inp["traj"], inp["dims"], inp["C"], inp["kw"],
                            inp["sw"], inp["osf"], sens=inp["maps"],
                            balance=True)
    try:
        ms, wall_ms = timed_steps(lambda: (op.forward(inp["x"]),
                                           op.adjoint(inp["k"])), steps)
    finally:
        op.close()
    return {"value": 1e3 / ms, "unit": UNIT, "steps": steps,
            "ms_per_step": ms, "wall_value": 1e3 / wall_ms,
            "wall_ms_per_step": wall_ms, "note": note}


def timed_steps(fn, steps, warmup=1):
    """(device ms per step, wall ms per step) of fn after `warmup` calls:
    CUDA events on the current (legacy default) stream, which every call
    here is ordered on or synchronises with, and the host clock."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) * 1e3 / steps
    return e0.elapsed_time(e1) / steps, wall


def plan_creation_ms(make, reps=3):
    """Median wall ms of creating (and synchronising) a plan; the plan is
    destroyed after each creation."""
    import torch
    ts = []
    for _ in range(reps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        p = make()
        torch.cuda.synchronize()
        ts.append((time.perf_counter() - t0) * 1e3)
        p.close()
    return statistics.median(ts)


def workload_label(name):
    dims, C, ns, nr, osf, kw, sw = WORKLOADS[name]
    d = "x".join(str(v) for v in dims)
    return (f"{len(dims)}D {d} image, {C} coils, osf {osf}, kw {kw}, sw {sw}, "
            f"{'kooshball' if len(dims) == 3 else 'golden-angle radial'} "
            f"{ns}x{nr} ({ns * nr} samples), forward + adjoint with coil "
            f"maps")


# --------------------------------------------------------------------------
# GPU arm
# --------------------------------------------------------------------------
def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(name, kernel):
    """(DRAM bytes read + written per launch of ``kernel`` on workload
    ``name``, where the figure comes from) from the committed ncu summary;
    (None, None) without one."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        e = d[name][kernel]
        src = e.get("scaled_from")
        how = (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of the "
               f"{src} capture, scaled by the units processed" if src else
               "ncu dram__bytes_read.sum + dram__bytes_write.sum")
        return e["dram_bytes_per_launch"], how
    except Exception:
        return None, None


def reduce_over_ranks(value, dist, device, op="max"):
    """The max (or min) of a per-rank float over all ranks (identity when
    there is no process group).  Every rank takes part, in the same order."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max"
                    else dist.ReduceOp.MIN)
    return float(t.item())


def replica_throughput(steps, world, ms_max):
    """Whole-job steps per second: every replica runs ``steps``; the job
    takes as long as the slowest rank."""
    return world * steps / (ms_max / 1e3)


def run_gpu_arm(args, rank, world, dist):
    import torch
    import gpunufft_b200 as G

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    inp = make_inputs(args.workload, seed=rank)
    C, M, dims = inp["C"], inp["M"], inp["dims"]
    plan = G.Plan(inp["traj"], dims, inp["kw"], inp["sw"], inp["osf"], None,
                  inp["maps"], G.BALANCED, device=dev)
    x_d = torch.from_numpy(inp["x"]).to(dev)
    k_d = torch.from_numpy(inp["k"]).to(dev)

    def step():
        plan.forward(x_d)
        plan.adjoint(k_d)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    barrier()
    # the timed steps replay one step captured as a CUDA graph (the same
    # launches as the calls above, every kernel every step), so that the
    # device time does not depend on how fast the host enqueues launches
    graph = torch.cuda.CUDAGraph()
    s_cap = torch.cuda.Stream(device=dev)
    s_cap.wait_stream(torch.cuda.current_stream())
    with torch.cuda.graph(graph, stream=s_cap):
        step()
    torch.cuda.current_stream().wait_stream(s_cap)
    graph.replay()
    barrier()
    stream = torch.cuda.current_stream()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(dev) as clk:
        barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            graph.replay()
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = reduce_over_ranks(ev0.elapsed_time(ev1), dist, dev)
    ms_per_step = ms / args.steps
    value = replica_throughput(args.steps, world, ms)

    # stage times (CUDA events on the plan's launch stream), timed steps
    plan.set_timing(True)
    stages = {"fwd": [], "adj": []}
    launches = 0
    for _ in range(args.steps):
        plan.forward(x_d)
        stages["fwd"].append(plan.stage_times())
        plan.adjoint(k_d)
        stages["adj"].append(plan.stage_times())
    plan.set_timing(False)
    for v in stages["fwd"] + stages["adj"]:
        launches += v["launches"]
    launches_per_step = launches // args.steps

    def avg(kind, key):
        return statistics.mean(s[key] for s in stages[kind])

    g = plan.info
    G_cells = int(np.prod([v for v in g.grid_dims if v]))
    dim = len(dims)
    peak, src = peaks()
    # algorithmic bytes per launch of the two gridding kernels.  General
    # grids: k-space (8 B per sample per coil), coordinates (4 B per axis
    # per sample) and the oversampled grid (8 B per cell per coil), read or
    # written once.  Power-of-two grids (this workload) run
    # k_forward_tma_groups (the same bytes) and k_adjoint_spmm_xfft, which
    # reads the sorted k-space, the interpolation matrix (8 B per entry,
    # kw^d entries per sample) and the row offsets (4 B per cell) and writes
    # the x-transformed rows (8 B per coil per kept output, G / G_x * N_x
    # per coil).
    gbytes = 8 * M * C + 4 * dim * M + 8 * G_cells * C
    pow2 = all((v & (v - 1)) == 0 for v in g.grid_dims if v)
    if pow2:
        nx_rows = G_cells // g.grid_dims[0] * dims[0]
        abytes = (8 * M * C + 8 * M * inp["kw"] ** dim + 4 * G_cells +
                  8 * C * nx_rows)
        kernels = {
            ("k_forward_tma_groups" if dim == 3 else "k_forward_tma"):
                ("forward interpolation", avg("fwd", "gridding_ms"), gbytes),
            "k_adjoint_spmm_xfft": ("adjoint spread + x transform",
                                    avg("adj", "gridding_ms"), abytes),
        }
    else:
        kernels = {
            "k_forward_interp": ("forward interpolation",
                                 avg("fwd", "gridding_ms"), gbytes),
            "k_adjoint_spmm": ("adjoint gridding", avg("adj", "gridding_ms"),
                               gbytes),
        }
    rooflines = []
    for kname, (what, kms, nbytes) in kernels.items():
        ach = nbytes / (kms * 1e-3) / 1e9
        traffic, tsrc = profile_traffic(args.workload, kname)
        # the gridding bytes of either direction counted as 8MC + 4dM + 8GC:
        # k-space, coordinates and the oversampled grid once each
        sach = gbytes / (kms * 1e-3) / 1e9
        rooflines.append({
            "kernel": kname, "what": what, "bound": "hbm", "achieved": ach,
            "peak": peak, "peak_source": src, "unit": "GB/s",
            "frac": ach / peak, "traffic": traffic,
            "traffic_source": tsrc,
            "algorithmic_bytes": nbytes,
            "gridding_bytes": gbytes, "gridding_achieved": sach,
            "gridding_frac": sach / peak, "launch_ms": kms})
    # the dominant one of this library's kernels (longest per step)
    roofline = max(rooflines, key=lambda r: r["launch_ms"])

    # end-to-end through the public API: every step copies its inputs from
    # pinned host memory and reads both results back to pinned host memory.
    # The operator runs on one stream; host-to-device copies run on a second
    # stream and device-to-host copies on a third, so a step's transfers
    # overlap the operator work of its neighbours (both copy directions and
    # the kernels proceed at once, as in a serving loop).
    xh = torch.from_numpy(inp["x"]).pin_memory()
    kh = torch.from_numpy(inp["k"]).pin_memory()
    out_k = torch.empty((C, M), dtype=torch.complex64).pin_memory()
    out_x = torch.empty(inp["x"].shape, dtype=torch.complex64).pin_memory()
    s_in = torch.cuda.Stream(device=dev)
    s_out = torch.cuda.Stream(device=dev)

    def e2e_step():
        with torch.cuda.stream(s_in):
            xd = xh.to(dev, non_blocking=True)
            ex = torch.cuda.Event()
            ex.record(s_in)
            kd = kh.to(dev, non_blocking=True)
            ek = torch.cuda.Event()
            ek.record(s_in)
        stream.wait_event(ex)
        xd.record_stream(stream)
        kk = plan.forward(xd)
        ef = torch.cuda.Event()
        ef.record(stream)
        stream.wait_event(ek)
        kd.record_stream(stream)
        ii = plan.adjoint(kd)
        ea = torch.cuda.Event()
        ea.record(stream)
        with torch.cuda.stream(s_out):
            s_out.wait_event(ef)
            out_k.copy_(kk, non_blocking=True)
            kk.record_stream(s_out)
            s_out.wait_event(ea)
            out_x.copy_(ii.reshape(out_x.shape), non_blocking=True)
            ii.record_stream(s_out)

    for _ in range(2):
        e2e_step()
    barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s_in.wait_event(e0)
    s_out.wait_event(e0)
    for _ in range(args.steps):
        e2e_step()
    stream.wait_stream(s_in)
    stream.wait_stream(s_out)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = reduce_over_ranks(e0.elapsed_time(e1), dist, dev)
    e2e_value = replica_throughput(args.steps, world, e2e_ms)
    h2d = xh.numel() * 8 + kh.numel() * 8
    d2h = out_k.numel() * 8 + out_x.numel() * 8

    # plain per-call operator (the upstream's flow: one coil per pass, maps
    # copied per coil per call, a synchronisation per coil)
    plain = {"value": None, "unit": UNIT, "steps": args.plain_steps}
    if args.plain_steps > 0:
        plan_p = G.Plan(inp["traj"], dims, inp["kw"], inp["sw"], inp["osf"],
                        None, inp["maps"], G.BALANCED, plain=True, device=dev)
        pms, pwall = timed_steps(lambda: (plan_p.forward(x_d),
                                          plan_p.adjoint(k_d)),
                                 args.plain_steps)
        plan_p.close()
        pms = reduce_over_ranks(pms, dist, dev)
        plain.update(value=world * 1e3 / pms, ms_per_step=pms,
                     wall_value=world * 1e3 / pwall, wall_ms_per_step=pwall,
                     batched_over_plain=value / (world * 1e3 / pms))
    # the host-array API (gnufft_forward_host / gnufft_adjoint_host: the
    # counterpart of the upstream's performForwardGpuNUFFT /
    # performGpuNUFFTAdj on host Arrays): host buffers in and out,
    # synchronous per call
    host_api = None
    if args.host_steps > 0:
        xh_np = inp["x"]
        kh_np = inp["k"]
        hms, hwall = timed_steps(lambda: (plan.forward(xh_np),
                                          plan.adjoint(kh_np)),
                                 args.host_steps)
        hms = reduce_over_ranks(hms, dist, dev)
        host_api = {"value": world * 1e3 / hms, "unit": UNIT,
                    "steps": args.host_steps, "ms_per_step": hms,
                    "wall_value": world * 1e3 / hwall,
                    "wall_ms_per_step": hwall,
                    "note": "Plan.forward / adjoint on NumPy arrays "
                            "(pageable host memory), copies inside each "
                            "call"}
    # plan creation (sector binning, sort, tables, interpolation matrix,
    # deapodization) for this workload and for the 2-D 256^2 x 16-coil
    # radial 402 x 512 workload of the differentiable operator
    creation = {}
    if rank == 0 and args.plan_timing:
        creation["workload_ms"] = plan_creation_ms(
            lambda: G.Plan(inp["traj"], dims, inp["kw"], inp["sw"],
                           inp["osf"], None, inp["maps"], G.BALANCED,
                           device=dev))
        tr4 = radial2d(402, 512)
        rng4 = np.random.default_rng(4)
        m4 = (rng4.standard_normal((16, 256, 256)) + 1j *
              rng4.standard_normal((16, 256, 256))).astype(np.complex64)
        creation["2d256_16coil_radial402x512_ms"] = plan_creation_ms(
            lambda: G.Plan(tr4, (256, 256), 3, 8, 2.0, None, m4, G.BALANCED,
                           device=dev))

    # the upstream library's own GPU operator, built from its sources for
    # sm_100a (oracle/_ref), on the same inputs through its host-array API
    # (performForwardGpuNUFFT / performGpuNUFFTAdj: per-call device
    # allocation and copies, one coil per pass in 3D); wall clock per step
    ref_gpu = None
    if args.ref_gpu_steps > 0:
        ref_gpu = reference_gpu(inp, args.ref_gpu_steps)

    batched = None
    if args.batch_instances > 0 and rank == 0:
        batched = batch_run(dev, args.steps, args.warmup,
                            n_instances=args.batch_instances)
    served = None
    if args.serve_requests > 0:
        served = serving_run(dev, args.serve_requests, seed=rank)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            threads = min(cpu_threads(), C)
            step_cpu = cpu_reference(inp, threads)
            step_cpu()
            tcpu = statistics.mean(step_cpu() for _ in range(2))
            cpu_val = threads / (tcpu * 2 * C)
            t1 = step_cpu(1)
            cpu = {"value": cpu_val, "unit": UNIT, "cores": threads,
                   "kind": "reference",
                   "single_core_value": 1.0 / (t1 * 2 * C),
                   "host_threads": cpu_threads(),
                   "sample": (f"upstream gpuNUFFT_cpu adjoint gridding, "
                              f"{threads} coil(s) x 2 steps on {threads} "
                              f"thread(s), one coil per thread; fwd+adj/s = "
                              f"coils/s / (2 x {C}); FFT and deapodization "
                              f"not counted; single_core_value: one coil on "
                              f"one thread")}
        except Exception as e:  # oracle/_ref absent on this machine
            cpu = {"value": None, "unit": UNIT, "cores": 0,
                   "kind": "reference", "sample": f"unavailable: {e}"}

    clocks = clk.summary()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": workload_label(args.workload),
                       "parallelism": f"replicas x{world}",
                       "l2": "inputs and grids larger than L2 (126 MB)",
                       "timed": "one step (forward + adjoint through the "
                                "public API) captured as a CUDA graph and "
                                "replayed once per timed step"},
            "roofline": roofline,
            "rooflines": rooflines,
            "stages_ms": {
                "forward": {k: avg("fwd", k) for k in
                            ("prepare_ms", "gridding_ms", "fft_ms",
                             "finish_ms")},
                "adjoint": {k: avg("adj", k) for k in
                            ("prepare_ms", "gridding_ms", "fft_ms",
                             "finish_ms")},
            },
            "plain": plain,
            "host_api": host_api,
            "plan_creation_ms": creation,
            "reference_gpu": ref_gpu,
            "served": served,
            "batched_uneven": batched,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "clocks": clocks,
            "gpu_launches": launches_per_step * args.steps,
        }
        print(json.dumps(line), flush=True)
    plan.close()


def serving_run(dev, n_requests, seed=0):
    """Poisson arrivals (mean 50 requests/s) of mixed CG-SENSE requests, 10
    iterations each: 2-D radial/spiral 128-384^2 with 1-32 coils and
    20k-400k samples, or 3-D kooshball 96^3-160^3 with 8-32 coils and
    0.5M-3M samples (two of the ten trajectories of the pool, so about one
    request in five).  Operators are reused per trajectory; maps per (size,
    coils).  Returns the server's statistics: cold (first pass, operators
    built on demand) and warm (the same arrivals again, operators
    resident) latencies side by side."""
    from gpunufft_b200.batch import spiral_trajectory
    from gpunufft_b200.serving import Request, Server
    rng = np.random.default_rng(seed)
    pool = []
    for i in range(10):
        if i < 8:
            size = int(rng.choice([128, 192, 256, 384]))
            M = int(rng.integers(20_000, 400_001))
            if i % 2:
                traj = radial2d(max(1, M // (2 * size)), 2 * size)
            else:
                traj = spiral_trajectory(int(rng.integers(8, 49)), M, rng)
            pool.append(((size, size), traj))
        else:
            size = int(rng.choice([96, 128, 160]))
            M = int(rng.integers(500_000, 3_000_001))
            nr = 2 * size
            pool.append(((size,) * 3, kooshball(max(1, M // nr), nr)))
    import copy

    import torch
    maps_cache = {}

    def maps_for(dims, C):
        key = (dims, C)
        if key not in maps_cache:
            shape = dims[::-1]
            grids = np.meshgrid(*[np.linspace(-0.5, 0.5, n, dtype=np.float32)
                                  for n in shape], indexing="ij")
            m = np.empty((C,) + shape, np.complex64)
            rss = np.zeros(shape, np.float32)
            for c in range(C):
                v = rng.standard_normal(len(shape))
                cen = 0.6 * v / np.linalg.norm(v)
                r2 = sum((g - cc) ** 2 for g, cc in zip(grids, cen))
                m[c] = np.exp(-r2 / 0.3)
                rss += np.abs(m[c]) ** 2
            m /= np.sqrt(rss)
            maps_cache[key] = torch.from_numpy(m).pin_memory()
        return maps_cache[key]

    reqs = []
    t = 0.0
    for i in range(n_requests):
        t += rng.exponential(1 / 50.0)
        dims, traj = pool[int(rng.integers(0, 10))]
        C = (int(rng.integers(8, 33)) if len(dims) == 3 else
             int(rng.integers(1, 33)))
        M = traj.shape[1]
        k = (rng.standard_normal((C, M), dtype=np.float32) + 1j *
             rng.standard_normal((C, M), dtype=np.float32)).astype(
                 np.complex64)
        reqs.append(Request(traj=traj, img_dims=dims,
                            kspace=torch.from_numpy(k).pin_memory(),
                            sens=maps_for(dims, C), n_iter=10, arrival=t,
                            rid=i))
    srv = Server(device=dev, max_slots=8)
    try:
        # first pass: operators and transform plans are built on demand
        srv.run([copy.copy(r) for r in reqs])
        cold = srv.stats()
        # second pass, same arrival pattern: the recurring workload in
        # steady state (operators resident per trajectory)
        srv.run(reqs)
        st = srv.stats()
    finally:
        srv.close()
    out = {
        "cold": {k: cold[k] for k in ("p50_ms", "p99_ms", "throughput_rps",
                                      "plan_cache_misses")},
        "warm": {k: st[k] for k in ("p50_ms", "p99_ms", "throughput_rps",
                                    "plan_cache_hits")},
        "requests": st["requests"], "max_concurrent": st["max_concurrent"],
        "peak_hbm_gb": max(st["peak_hbm_gb"], cold["peak_hbm_gb"]),
        "peak_live_gb": max(st["peak_live_gb"], cold["peak_live_gb"]),
        "peak_admitted_gb": max(st["peak_admitted_gb"],
                                cold["peak_admitted_gb"]),
        "workload": (f"{n_requests} CG-SENSE requests x 10 iterations, "
                     f"Poisson 50/s, 2-D 128-384^2 1-32 coils 20k-400k "
                     f"samples / 3-D 96-160^3 8-32 coils 0.5M-3M samples; "
                     f"cold = first pass (operators built on demand), warm "
                     f"= the same arrivals again (operators resident)")}
    return out


def batch_run(dev, steps, warmup, seed=0, n_instances=64):
    """``n_instances`` uneven 2-D spiral operators (image 96-320^2, 8-32
    coils, 10k-120k samples, osf 1.25-2, kernel width 3-5; sector width and
    forward tile from the autotuner): fwd + adj of every instance per step.
    Headline: the persistent batch (every stage of all instances in one
    launch, one cuFFT call per instance between stages) replayed from a
    CUDA graph; beside it the instances' own launches captured on 8
    streams into one graph, and the plain per-instance loop on one stream.
    Device-timed ms per step of each."""
    import torch

    import gpunufft_b200 as G
    from gpunufft_b200.batch import BatchedOperator, autotune, \
        spiral_instances
    specs = spiral_instances(n_instances, seed=seed)
    rng = np.random.default_rng(seed)
    plans, coils, tuned = [], [], []
    t0 = time.perf_counter()
    for s in specs:
        shape = s["img_dims"][::-1]
        grids = np.meshgrid(*[np.linspace(-0.5, 0.5, n) for n in shape],
                            indexing="ij")
        maps = []
        for c in range(s["n_coils"]):
            a = 2 * math.pi * c / s["n_coils"]
            cen = (0.6 * math.sin(a), 0.6 * math.cos(a))
            r2 = sum((g - cc) ** 2 for g, cc in zip(grids, cen))
            ramp = sum(rng.uniform(-2, 2) * g for g in grids)
            maps.append(np.exp(-r2 / 0.3) * np.exp(1j * ramp))
        maps = np.array(maps)
        maps = (maps / np.sqrt((np.abs(maps) ** 2).sum(0))).astype(
            np.complex64)
        tr = autotune(s["traj"], s["img_dims"], s["n_coils"],
                      s["kernel_width"], s["osf"], sens=maps, reps=2,
                      sector_widths=(6, 8, 12), tile_coils=(0, 8, 16),
                      device=dev)
        tuned.append((tr.sector_width, tr.tile_coils))
        plans.append(G.Plan(s["traj"], s["img_dims"], s["kernel_width"],
                            tr.sector_width, s["osf"], None, maps, G.BALANCED,
                            device=dev, tile_coils=tr.tile_coils))
        coils.append(s["n_coils"])
    tune_s = time.perf_counter() - t0
    bo = BatchedOperator(plans, coils, device=dev, mode="persistent")
    info = bo.info()
    for x in bo.img_in:
        x.copy_(torch.randn_like(x))
    for k in bo.k_in:
        k.copy_(torch.randn_like(k))
    ms_graph, _ = timed_steps(lambda: (bo.replay("forward"),
                                       bo.replay("adjoint")), steps,
                              max(warmup, 1))
    ms_plain, _ = timed_steps(lambda: (bo.plain("forward"),
                                       bo.plain("adjoint")), steps,
                              max(warmup, 1))
    # one more persistent step inside an NVTX range, untimed, so that a
    # profiler can list exactly the launches of one step
    # (ncu --nvtx --nvtx-include "batch_step/")
    torch.cuda.nvtx.range_push("batch_step")
    bo.replay("forward")
    bo.replay("adjoint")
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize(dev)
    bo.close()
    so = BatchedOperator(plans, coils, n_streams=8, device=dev,
                         mode="streams")
    for x in so.img_in:
        x.copy_(torch.randn_like(x))
    for k in so.k_in:
        k.copy_(torch.randn_like(k))
    ms_streams, _ = timed_steps(lambda: (so.replay("forward"),
                                         so.replay("adjoint")), steps,
                                max(warmup, 1))
    del so
    sw_hist = {}
    for sw, tc in tuned:
        key = f"sw{sw}/tile{tc or 'auto'}"
        sw_hist[key] = sw_hist.get(key, 0) + 1
    for p in plans:
        p.close()
    n = len(plans)
    return {"value": n / (ms_graph * 1e-3), "unit": "instances/s",
            "ms_per_step": ms_graph, "instances": n,
            "launches_per_step": {
                "persistent_kernels": info.kernels_forward +
                info.kernels_adjoint,
                "fft_calls": 2 * info.fft_calls,
                "units": dict(zip(("prepare", "interpolation", "gather",
                                   "spread", "finish"), info.units))},
            "streams_graph": {"value": n / (ms_streams * 1e-3),
                              "ms_per_step": ms_streams},
            "plain": {"value": n / (ms_plain * 1e-3),
                      "ms_per_step": ms_plain},
            "graph_over_plain": ms_plain / ms_graph,
            "persistent_over_streams": ms_streams / ms_graph,
            "autotune": {"seconds": tune_s, "choices": sw_hist},
            "workload": f"{n} variable-density 2-D spirals, image 96-320^2, "
                        "8-32 coils, 10k-120k samples, osf 1.25-2, kw 3-5, "
                        "coil maps; one step = forward + adjoint of every "
                        "instance"}


def run_batch_arm(args, rank, world):
    """The uneven spiral batch as the benchmark's workload."""
    import torch
    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    b = batch_run(dev, args.steps, args.warmup, seed=rank)
    if rank == 0:
        print(json.dumps({
            "metric": "uneven batch: instance fwd+adj/s, persistent batch "
                      "from a CUDA graph vs plain per-instance loop",
            "value": world * b["value"], "unit": "instances/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": b["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": b["workload"],
                       "instances": b["instances"]},
            **{k: b[k] for k in ("launches_per_step", "streams_graph",
                                 "plain", "graph_over_plain",
                                 "persistent_over_streams", "autotune")},
        }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="3d128x32",
                    choices=list(WORKLOADS) + ["spirals64"])
    ap.add_argument("--plain-steps", type=int, default=5)
    ap.add_argument("--host-steps", type=int, default=5,
                    help="steps of the host-array API arm (0: skip)")
    ap.add_argument("--batch-instances", type=int, default=64,
                    help="instances of the uneven spiral batch reported "
                         "beside the workload (0: skip)")
    ap.add_argument("--no-plan-timing", dest="plan_timing",
                    action="store_false",
                    help="skip the plan-creation timings")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=40,
                    help="requests of the serving run (0: skip)")
    ap.add_argument("--ref-gpu-steps", type=int, default=5,
                    help="steps of the upstream GPU operator (0: skip)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if args.impl == "reference":
        run_reference_arm(args, rank)
        return
    if args.workload == "spirals64":
        run_batch_arm(args, rank, world)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl",
                                 timeout=datetime.timedelta(seconds=300))
        dist = tdist
    try:
        run_gpu_arm(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
