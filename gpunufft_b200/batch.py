"""Many independent operators run together, and the autotuner that picks
each operator's sector width and tile shape.

``BatchedOperator`` takes operators of uneven sizes (image size, coils,
trajectory length, oversampling, kernel width, sector width; one plan may
appear several times, as frames sharing a trajectory).  By default
(``mode="persistent"``) it runs them through the library's batch entry
points (``gnufft_batch_forward`` / ``gnufft_batch_adjoint``): every stage
of all instances -- forward: prepare, interpolation; adjoint: gather,
spread, finish -- is one persistent launch whose blocks take (instance,
work item) units from a device counter, with one cuFFT call per instance
between the stages; the call is captured once into a CUDA graph and
replayed.  ``mode="streams"`` records the instances' own per-operator
launches on several capture streams into one graph instead.  Inputs and
outputs are static device tensors owned by the batch; ``forward`` /
``adjoint`` copy new data in, replay, and return the (static) outputs.

``autotune`` times fwd + adj for candidate sector widths and forward tile
shapes (coils staged per sector tile) on the instance itself and returns
the fastest.  Results are cached per geometry.
"""
from __future__ import annotations

import ctypes
import dataclasses
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _capi as C
from .operator import Plan


# --------------------------------------------------------------------------
# autotuner
# --------------------------------------------------------------------------
@dataclasses.dataclass
class TuneResult:
    sector_width: int
    tile_coils: int
    ms: float                       # fwd + adj device time of the choice
    table: List[Tuple[int, int, float]]  # every candidate timed


_TUNE_CACHE: Dict[tuple, TuneResult] = {}


def _time_fwd_adj(plan: Plan, n_coils: int, reps: int, device: int) -> float:
    dev = torch.device("cuda", device)
    shape = plan.img_shape if plan.n_sens else (n_coils,) + plan.img_shape
    x = torch.randn(shape, dtype=torch.complex64, device=dev)
    k = torch.randn((n_coils, plan.M), dtype=torch.complex64, device=dev)
    plan.forward(x)
    plan.adjoint(k)
    best = float("inf")
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        plan.forward(x)
        plan.adjoint(k)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def autotune(traj, img_dims: Sequence[int], n_coils: int,
             kernel_width: int = 3, osf: float = 2.0, dens=None, sens=None,
             sector_widths: Sequence[int] = (4, 6, 8, 10, 12, 16),
             tile_coils: Sequence[int] = (0, 2, 4, 8, 16, 32),
             reps: int = 3, device: int = 0,
             use_cache: bool = True) -> TuneResult:
    """Fastest (sector width, forward tile coils) for this operator, by
    timing fwd + adj on random data (CUDA events, best of ``reps``).  Sector
    width first (with the automatic tile), then the tile shape."""
    traj = np.ascontiguousarray(traj, np.float32)
    key = (tuple(int(v) for v in img_dims), int(n_coils), traj.shape,
           int(kernel_width), float(osf), dens is not None,
           sens is not None, tuple(sector_widths), tuple(tile_coils))
    if use_cache and key in _TUNE_CACHE:
        return _TUNE_CACHE[key]
    table = []

    def trial(sw, tc):
        try:
            p = Plan(traj, img_dims, kernel_width, sw, osf, dens, sens,
                     C.BALANCED, device=device, tile_coils=tc)
        except C.GnufftError:
            return None                  # geometry not supported
        try:
            ms = _time_fwd_adj(p, n_coils, reps, device)
        finally:
            p.close()
        table.append((sw, tc, ms))
        return ms

    best_sw, best_ms = None, float("inf")
    for sw in sector_widths:
        ms = trial(sw, 0)
        if ms is not None and ms < best_ms:
            best_sw, best_ms = sw, ms
    if best_sw is None:
        raise RuntimeError("no candidate sector width is supported")
    best_tc = 0
    for tc in tile_coils:
        if tc == 0:
            continue
        ms = trial(best_sw, tc)
        if ms is not None and ms < best_ms:
            best_tc, best_ms = tc, ms
    res = TuneResult(best_sw, best_tc, best_ms, table)
    if use_cache:
        _TUNE_CACHE[key] = res
    return res


# --------------------------------------------------------------------------
# batched execution in one CUDA graph
# --------------------------------------------------------------------------
class BatchedOperator:
    """Independent operators run together (see the module docstring).

    plans: one Plan per instance (built with its own maps if any; a plan
    may repeat); n_coils: coil count per instance; mode: "persistent" (one
    launch per stage for all instances) or "streams" (per-instance launches
    on n_streams capture branches)."""

    def __init__(self, plans: Sequence[Plan], n_coils: Sequence[int],
                 n_streams: int = 8, device: int = 0,
                 mode: str = "persistent"):
        if len(plans) != len(n_coils):
            raise ValueError("one coil count per plan")
        if mode not in ("persistent", "streams"):
            raise ValueError("mode is 'persistent' or 'streams'")
        self.plans = list(plans)
        self.n_coils = [int(c) for c in n_coils]
        self.device = device
        self.mode = mode
        self._batch = None
        dev = torch.device("cuda", device)
        self.img_in, self.k_in, self.k_out, self.img_out = [], [], [], []
        for p, c in zip(self.plans, self.n_coils):
            shape = p.img_shape if p.n_sens else (c,) + p.img_shape
            self.img_in.append(torch.zeros(shape, dtype=torch.complex64,
                                           device=dev))
            self.k_in.append(torch.zeros((c, p.M), dtype=torch.complex64,
                                         device=dev))
        self.streams = [torch.cuda.Stream(device=device)
                        for _ in range(max(1, n_streams))]
        self._graphs: Dict[str, torch.cuda.CUDAGraph] = {}
        self._outs: Dict[str, list] = {}
        if mode == "persistent":
            n = len(self.plans)
            handles = (ctypes.c_void_p * n)(*[p._h.value for p in self.plans])
            coils = (ctypes.c_uint32 * n)(*self.n_coils)
            h = ctypes.c_void_p()
            with torch.cuda.device(device):
                C.check(C.lib().gnufft_batch_create(handles, coils, n,
                                                    ctypes.byref(h)))
            self._batch = h
            for p, c, x in zip(self.plans, self.n_coils, self.img_in):
                self.k_out.append(torch.empty((c, p.M), dtype=torch.complex64,
                                              device=dev))
                self.img_out.append(torch.empty_like(x))

            def ptrs(ts):
                return (ctypes.c_void_p * n)(*[t.data_ptr() for t in ts])
            self._p_img_in, self._p_k_out = ptrs(self.img_in), ptrs(self.k_out)
            self._p_k_in, self._p_img_out = ptrs(self.k_in), ptrs(self.img_out)
        # grow every plan's scratch, create its FFT plans and load the
        # kernels before any capture
        for i in range(len(self.plans)):
            self._call_one("forward", i)
            self._call_one("adjoint", i)
        if self._batch is not None:
            self._call_batch("forward")
            self._call_batch("adjoint")
        torch.cuda.synchronize(device)

    def info(self) -> Optional[C.BatchInfo]:
        """Work units per stage, launches per call and device bytes of the
        persistent batch (None in "streams" mode)."""
        if self._batch is None:
            return None
        info = C.BatchInfo()
        C.check(C.lib().gnufft_batch_get_info(self._batch,
                                              ctypes.byref(info)))
        return info

    def close(self) -> None:
        if self._batch is not None:
            self._graphs.clear()
            C.lib().gnufft_batch_destroy(self._batch)
            self._batch = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _call_one(self, kind: str, i: int):
        p = self.plans[i]
        return (p.forward(self.img_in[i]) if kind == "forward"
                else p.adjoint(self.k_in[i]))

    def _call_batch(self, kind: str) -> list:
        stream = ctypes.c_void_p(
            torch.cuda.current_stream(self.device).cuda_stream)
        L = C.lib()
        if kind == "forward":
            C.check(L.gnufft_batch_forward(self._batch, self._p_img_in,
                                           self._p_k_out, stream))
            return self.k_out
        C.check(L.gnufft_batch_adjoint(self._batch, self._p_k_in,
                                       self._p_img_out, stream))
        return self.img_out

    def _capture(self, kind: str) -> None:
        g = torch.cuda.CUDAGraph()
        main = torch.cuda.Stream(device=self.device)
        main.wait_stream(torch.cuda.current_stream(self.device))
        if self.mode == "persistent":
            with torch.cuda.graph(g, stream=main):
                outs = self._call_batch(kind)
        else:
            outs = [None] * len(self.plans)
            with torch.cuda.graph(g, stream=main):
                for s in self.streams:
                    s.wait_stream(main)
                for i in range(len(self.plans)):
                    with torch.cuda.stream(self.streams[i % len(self.streams)]):
                        outs[i] = self._call_one(kind, i)
                for s in self.streams:
                    main.wait_stream(s)
        torch.cuda.current_stream(self.device).wait_stream(main)
        self._graphs[kind] = g
        self._outs[kind] = outs

    def replay(self, kind: str) -> list:
        """Run every instance's ``kind`` ('forward' or 'adjoint') on the
        static inputs; returns the static outputs (valid until the next
        replay of the same kind)."""
        if kind not in self._graphs:
            self._capture(kind)
        self._graphs[kind].replay()
        return self._outs[kind]

    def forward(self, images: Sequence[torch.Tensor]) -> list:
        for dst, src in zip(self.img_in, images):
            dst.copy_(src.reshape(dst.shape), non_blocking=True)
        return self.replay("forward")

    def adjoint(self, kspaces: Sequence[torch.Tensor]) -> list:
        for dst, src in zip(self.k_in, kspaces):
            dst.copy_(src.reshape(dst.shape), non_blocking=True)
        return self.replay("adjoint")

    def plain(self, kind: str) -> list:
        """The same work as a plain per-instance loop on one stream."""
        return [self._call_one(kind, i) for i in range(len(self.plans))]


# --------------------------------------------------------------------------
# workload: uneven variable-density spirals
# --------------------------------------------------------------------------
def spiral_trajectory(n_interleaves: int, n_samples: int,
                      rng: np.random.Generator) -> np.ndarray:
    """2-D variable-density spiral (radius ~ u^1.6, denser near the centre),
    ``n_interleaves`` rotated copies, ``n_samples`` points in total,
    coordinates in [-0.5, 0.5)."""
    per = max(1, n_samples // n_interleaves)
    u = np.arange(per) / per
    turns = rng.uniform(6, 14)
    r = 0.499 * u ** 1.6
    out = []
    for l in range(n_interleaves):
        th = 2 * np.pi * (turns * u + l / n_interleaves)
        out.append(np.stack([r * np.cos(th), r * np.sin(th)]))
    return np.ascontiguousarray(np.concatenate(out, 1), np.float32)


def spiral_instances(n: int = 64, seed: int = 0):
    """The uneven batch: image size in {96, 160, 256, 320}^2, 8-32 coils,
    8-48 interleaves, 10k-120k samples, osf 1.25-2.0, kernel width 3-5."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        size = int(rng.choice([96, 160, 256, 320]))
        out.append(dict(
            img_dims=(size, size), n_coils=int(rng.integers(8, 33)),
            traj=spiral_trajectory(int(rng.integers(8, 49)),
                                   int(rng.integers(10_000, 120_001)), rng),
            osf=float(np.round(rng.uniform(1.25, 2.0), 2)),
            kernel_width=int(rng.integers(3, 6))))
    return out
