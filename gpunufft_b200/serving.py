"""Serving loop for CG-SENSE reconstruction requests with continuous
batching and memory-based admission.

A request carries a trajectory, multicoil k-space, sensitivity maps and a
CG iteration count (the body of ``matlab/demo/utils/cg_sense_2d.m:40-108``).
The server keeps operators resident per trajectory (sector tables,
interpolation matrix, cuFFT plans: ``PlanCache``), admits queued requests
whenever a slot and enough device memory are free, and advances every
admitted request by one CG iteration per scheduler round, each request on
its own CUDA stream.  Requests that arrive while others are on the GPU join
at the next round; finished requests leave and free their slot and memory
at once, so work of different sizes overlaps on the device.  Every
iteration is stream-ordered and needs no host synchronisation; the
scheduler only polls CUDA events.

Results do not depend on the mix: a request's arithmetic runs on its own
plan instance and stream in a fixed order.
"""
from __future__ import annotations

import collections
import dataclasses
import hashlib
import os
import time
from typing import Deque, Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _capi as C
from .cg_sense import _dot
from .operator import Plan


@dataclasses.dataclass
class Request:
    traj: np.ndarray                 # (dim, M) float32 in [-0.5, 0.5)
    img_dims: Tuple[int, ...]        # (width, height[, depth])
    kspace: np.ndarray               # (C, M) complex64
    sens: np.ndarray                 # (C, [depth,] height, width) complex64
    n_iter: int = 10
    dens: Optional[np.ndarray] = None
    alpha: float = 0.0
    kernel_width: int = 3
    sector_width: int = 8
    osf: float = 2.0
    arrival: float = 0.0             # seconds, relative to the server clock
    rid: int = -1
    # filled in by the server
    result: Optional[np.ndarray] = None
    admitted: float = 0.0
    finished: float = 0.0

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def _key(req: Request) -> str:
    h = hashlib.sha1()
    h.update(np.ascontiguousarray(req.traj, np.float32).tobytes())
    if req.dens is not None:
        h.update(np.ascontiguousarray(req.dens, np.float32).tobytes())
    h.update(repr((tuple(req.img_dims), req.kernel_width, req.sector_width,
                   float(req.osf))).encode())
    return h.hexdigest()


def plan_table_bytes(req: Request) -> int:
    """Upper bound of the device bytes of a new operator for the request's
    trajectory before any call: sorted trajectory, indices (sorted order,
    sector, inverse), density weights, the interpolation matrix (row offsets
    per grid cell, at most (kw + 1)^d entries of 8 bytes per sample), the
    forward work items, their lane order (3-D), column ranges and the list
    of column tiles holding one, deapodization, the lookup table and the
    maps the request sets."""
    dims = [v for v in req.img_dims if v]
    dim = len(dims)
    M = req.traj.shape[1]
    N = int(np.prod(dims))
    grid = [int(v * req.osf) for v in dims]
    G = int(np.prod(grid))
    Cn = req.kspace.shape[0]
    nnz = M * (req.kernel_width + 1) ** dim
    b = 4 * dim * M + 3 * 4 * M + 4 * M + 4 * (G + 1) + 8 * nnz
    if dim == 3:
        b += 4 * M
    b += 16 * (M // 256 + int(np.prod([-(-g // req.sector_width)
                                       for g in grid])) + 1)
    b += 8 * grid[0] * grid[1] + 4 * (grid[0] * grid[1] // 8 + 1)
    b += 4 * N + 4 * 4096 + 8 * Cn * N
    return int(b)


def request_bytes(req: Request, plan: Optional[Plan] = None) -> int:
    """Device bytes a request holds while it runs: its operator (the cached
    instance's own figure, else plan_table_bytes), the operator's scratch
    for the request's coil count (gnufft_call_scratch_bytes), and its
    tensors -- k-space and maps, the CG vectors x, r, p and the
    temporaries of one iteration (forward output, adjoint outputs)."""
    dims = [v for v in req.img_dims if v]
    M = req.traj.shape[1]
    N = int(np.prod(dims))
    Cn = req.kspace.shape[0]
    if plan is not None:
        op = plan.info.device_bytes + plan.call_scratch_bytes(Cn)
    else:
        G = int(np.prod([int(v * req.osf) for v in dims]))
        lanes = Cn if Cn <= 16 else (Cn + 31) // 32 * 32
        # scratch bound: sorted k-space lanes, grid and two transform
        # buffers of a grid each (what gnufft_call_scratch_bytes counts,
        # rounded up)
        op = plan_table_bytes(req) + 8 * M * lanes + 3 * 8 * (Cn + 1) * G
    tensors = 8 * Cn * M + 8 * Cn * N          # k-space, maps
    tensors += 8 * N * 3                       # x, r, p
    tensors += 8 * Cn * M + 8 * N * 4          # one iteration's temporaries
    return int(op + tensors)


class PlanCache:
    """Operators resident per trajectory (sector tables, interpolation
    matrix, transform plans and scratch).  At most ``max_instances``
    instances of one trajectory's operator exist (two: a second request of
    the same trajectory runs beside the first); a request whose
    trajectory's instances are all busy waits for one.  Idle instances stay
    cached until memory is needed.

    With ``plan_dir`` the operators' precomputed tables also persist on
    disk, one ``<key>.npz`` per trajectory (``Plan.save``: the upstream's
    precompute arrays): a miss loads the file when it exists (tables
    validated, ``Plan.from_file``; the sort is skipped) and otherwise
    creates the operator and writes its file, so a restarted server meets
    known trajectories with their tables ready."""

    def __init__(self, device: int = 0, max_instances: int = 2,
                 plan_dir: Optional[str] = None):
        self.device = device
        self.max_instances = max_instances
        self.plan_dir = plan_dir
        self.plans_loaded = 0
        self.plans_saved = 0
        self.free: Dict[str, List[Plan]] = collections.defaultdict(list)
        self.busy: Dict[int, str] = {}
        self.count: Dict[str, int] = collections.defaultdict(int)
        self.lru: "collections.OrderedDict[str, float]" = \
            collections.OrderedDict()
        self.hits = 0
        self.misses = 0

    def available(self, req: Request) -> bool:
        key = _key(req)
        return bool(self.free[key]) or self.count[key] < self.max_instances

    def peek(self, req: Request) -> Optional[Plan]:
        """An idle cached instance for the request's trajectory, if any."""
        ps = self.free.get(_key(req))
        return ps[-1] if ps else None

    def acquire(self, req: Request) -> Plan:
        key = _key(req)
        self.lru[key] = time.perf_counter()
        self.lru.move_to_end(key)
        if self.free[key]:
            self.hits += 1
            p = self.free[key].pop()
        else:
            self.misses += 1
            p = self._new_plan(req, key)
            self.count[key] += 1
        self.busy[id(p)] = key
        return p

    def _new_plan(self, req: Request, key: str) -> Plan:
        path = (os.path.join(self.plan_dir, key + ".npz")
                if self.plan_dir else None)
        if path and os.path.exists(path):
            self.plans_loaded += 1
            return Plan.from_file(path, device=self.device)
        p = Plan(req.traj, req.img_dims, req.kernel_width, req.sector_width,
                 req.osf, req.dens, None, C.BALANCED, device=self.device)
        if path:
            os.makedirs(self.plan_dir, exist_ok=True)
            tmp = os.path.join(self.plan_dir, key + ".tmp.npz")
            p.save(tmp)
            os.replace(tmp, path)  # readers never see a partial file
            self.plans_saved += 1
        return p

    def release(self, p: Plan) -> None:
        key = self.busy.pop(id(p))
        self.free[key].append(p)

    def idle_bytes(self) -> int:
        return sum(p.info.device_bytes for ps in self.free.values()
                   for p in ps)

    def evict_one(self) -> bool:
        """Drop one idle instance, least recently used trajectory first."""
        for key in list(self.lru):
            if self.free.get(key):
                self.free[key].pop().close()
                self.count[key] -= 1
                if not self.free[key] and key not in self.busy.values():
                    del self.lru[key]
                return True
        return False

    def clear(self) -> None:
        for ps in self.free.values():
            for p in ps:
                p.close()
        self.free.clear()
        self.count.clear()


class _Active:
    """A request on the GPU: its plan instance, stream and CG state.

    The CG vectors live in fixed device tensors updated in place, so after
    the first (eager) iteration one iteration is captured as a CUDA graph
    and every later iteration is a single graph launch: the host work per
    iteration no longer grows with the number of kernels in it."""

    def __init__(self, req: Request, plan: Plan, device: int,
                 use_graph: bool = True, admitted_bytes: int = 0):
        self.req = req
        self.plan = plan
        self.admitted_bytes = admitted_bytes
        self.stream = torch.cuda.Stream(device=device)
        self.done_event = torch.cuda.Event()
        self.it = 0
        self.use_graph = use_graph
        self.graph: Optional[torch.cuda.CUDAGraph] = None
        with torch.cuda.stream(self.stream):
            dev = torch.device("cuda", device)
            # pinned host tensors upload asynchronously on this stream
            self.y = torch.as_tensor(req.kspace).to(dev, non_blocking=True)
            self.maps = torch.as_tensor(req.sens).to(dev, non_blocking=True)
            plan.set_sens(self.maps)
            rhs = plan.adjoint(self.y)
            self.x = torch.zeros_like(rhs)
            self.r = rhs
            self.p = rhs.clone()
            self.rr = _dot(self.r, self.r).real

    def _iteration(self) -> None:
        """One CG iteration (matlab/demo/utils/cg_sense_2d.m:76-100) with
        in-place updates of x, r, p and rr."""
        ap = self.plan.adjoint(self.plan.forward(self.p))
        if self.req.alpha:
            ap = ap + self.req.alpha * self.p
        a = self.rr / _dot(self.p, ap)
        self.x.add_(a * self.p)
        self.r.sub_(a * ap)
        rr_new = _dot(self.r, self.r).real
        self.p.mul_(rr_new / self.rr).add_(self.r)
        self.rr.copy_(rr_new)

    def step(self) -> None:
        """Enqueue one CG iteration on this request's stream."""
        with torch.cuda.stream(self.stream):
            if self.graph is not None:
                self.graph.replay()
            elif self.use_graph and self.it == 1 and self.req.n_iter > 2:
                # the first iteration ran eagerly on this stream (every
                # buffer of the plan and of the vector ops exists); capture
                # the second and replay it from now on.  capture_begin /
                # capture_end, not torch.cuda.graph: no device-wide
                # synchronisation while other requests run.
                g = torch.cuda.CUDAGraph()
                g.capture_begin()
                try:
                    self._iteration()
                finally:
                    g.capture_end()
                self.graph = g
                g.replay()
            else:
                self._iteration()
            self.it += 1
            if self.it == self.req.n_iter:
                self.out = torch.empty(self.x.shape, dtype=self.x.dtype,
                                       pin_memory=True)
                self.out.copy_(self.x, non_blocking=True)
                self.done_event.record(self.stream)

    def finished(self) -> bool:
        return self.it == self.req.n_iter and self.done_event.query()

    def release(self) -> None:
        self.graph = None


class Server:
    """Continuous-batching CG-SENSE server on one GPU.

    max_slots: requests on the GPU at once; memory_budget: device bytes the
    server may hold for running requests and cached operators (default:
    90 % of the free memory at start)."""

    def __init__(self, device: int = 0, max_slots: int = 8,
                 memory_budget: Optional[int] = None,
                 plan_dir: Optional[str] = None):
        self.device = device
        torch.cuda.set_device(device)
        free, _ = torch.cuda.mem_get_info(device)
        self.budget = int(memory_budget if memory_budget is not None
                          else 0.9 * free)
        self.max_slots = max_slots
        self.cache = PlanCache(device, plan_dir=plan_dir)
        self.queue: Deque[Request] = collections.deque()
        self.active: List[_Active] = []
        self.done: List[Request] = []
        self.in_use = 0
        self.peak_in_use = 0
        self.peak_device_used = 0
        self.max_concurrent = 0
        self.peak_live = 0
        self.peak_accounted = 0
        self._t0 = time.perf_counter()
        self._free0 = free
        self._torch0 = torch.cuda.memory_allocated(device)

    def now(self) -> float:
        return time.perf_counter() - self._t0

    def submit(self, req: Request) -> None:
        if request_bytes(req) > self.budget:
            raise ValueError("request larger than the server's memory budget")
        if req.arrival <= 0:
            req.arrival = self.now()
        self.queue.append(req)

    def _admit(self) -> None:
        """Admit queued requests in arrival order while slots and memory
        allow; a request whose trajectory's operator is busy stays queued
        without blocking the requests behind it."""
        waiting = collections.deque()
        while self.queue and len(self.active) < self.max_slots:
            req = self.queue.popleft()
            if not self.cache.available(req):
                waiting.append(req)
                continue
            cached = self.cache.peek(req)
            need = request_bytes(req, cached)
            idle = self.cache.idle_bytes()
            if cached is not None:  # counted in `need` from now on
                idle -= cached.info.device_bytes
            while (self.in_use + need + idle > self.budget
                   and self.cache.evict_one()):
                idle = self.cache.idle_bytes()
                cached = self.cache.peek(req)
                need = request_bytes(req, cached)
                if cached is not None:
                    idle -= cached.info.device_bytes
            if self.in_use + need > self.budget:
                waiting.append(req)         # wait for memory to free up
                break
            req.admitted = self.now()
            plan = self.cache.acquire(req)
            self.active.append(_Active(req, plan, self.device,
                                       admitted_bytes=need))
            self.in_use += need
            self.peak_in_use = max(self.peak_in_use, self.in_use)
            self.peak_accounted = max(self.peak_accounted,
                                      self.in_use + self.cache.idle_bytes())
        waiting.extend(self.queue)
        self.queue = waiting
        self.max_concurrent = max(self.max_concurrent, len(self.active))

    def _retire(self) -> None:
        keep = []
        for a in self.active:
            if a.finished():
                a.req.result = a.out.numpy().copy()
                a.req.finished = self.now()
                a.release()
                self.cache.release(a.plan)
                self.in_use -= a.admitted_bytes
                self.done.append(a.req)
            else:
                keep.append(a)
        self.active = keep

    def round(self) -> None:
        """One scheduler round: retire, admit, one iteration per request."""
        self._retire()
        self._admit()
        for a in self.active:
            if a.it < a.req.n_iter:
                a.step()
        free, total = torch.cuda.mem_get_info(self.device)
        self.peak_device_used = max(self.peak_device_used, total - free)
        # what the running requests and cached operators hold: operators'
        # own figures and the tensors torch has allocated (not the memory
        # its caching allocator keeps for reuse)
        live = (sum(a.plan.info.device_bytes for a in self.active) +
                self.cache.idle_bytes() +
                max(0, torch.cuda.memory_allocated(self.device) -
                    self._torch0))
        self.peak_live = max(self.peak_live, live)
        self.peak_accounted = max(self.peak_accounted,
                                  self.in_use + self.cache.idle_bytes())

    def run(self, arrivals: Sequence[Request], timeout: float = 600.0):
        """Replay ``arrivals`` (sorted by ``arrival`` seconds from now) and
        serve until all are done.  Returns the finished requests."""
        pending = collections.deque(sorted(arrivals, key=lambda r: r.arrival))
        self._t0 = time.perf_counter()
        self.done = []
        self.max_concurrent = 0
        n = len(pending)
        while len(self.done) < n:
            t = self.now()
            if t > timeout:
                raise TimeoutError("serving did not finish")
            while pending and pending[0].arrival <= t:
                self.queue.append(pending.popleft())
            if not self.active and not self.queue and pending:
                time.sleep(min(0.001, max(0.0, pending[0].arrival - t)))
                continue
            self.round()
            if self.active and all(a.it == a.req.n_iter for a in self.active):
                time.sleep(0.0002)      # everything enqueued: wait a little
        torch.cuda.synchronize(self.device)
        return list(self.done)

    def stats(self) -> dict:
        lat = np.array([r.latency for r in self.done]) * 1e3
        span = (max(r.finished for r in self.done) -
                min(r.arrival for r in self.done)) if self.done else 0.0
        return {
            "requests": len(self.done),
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "throughput_rps": len(self.done) / span if span > 0 else None,
            "max_concurrent": self.max_concurrent,
            "peak_hbm_gb": self.peak_device_used / 1e9,
            "peak_live_gb": self.peak_live / 1e9,
            "peak_admitted_gb": self.peak_accounted / 1e9,
            "plan_cache_hits": self.cache.hits,
            "plan_cache_misses": self.cache.misses,
            "plans_loaded": self.cache.plans_loaded,
            "plans_saved": self.cache.plans_saved,
        }

    def close(self) -> None:
        torch.cuda.synchronize(self.device)
        for a in self.active:
            a.release()
            self.cache.release(a.plan)
        self.active = []
        self.cache.clear()
