"""Serving: continuous batching of FIRE minimisations and fixed-step dynamics runs.

Requests (Voronoi or vertex model; SPP dynamics for a fixed number of steps, or FIRE to a force
norm) arrive at any time. Each of ``lanes`` worker threads takes a batch when it is free: the
oldest queued request fixes the batch's kind, and every queued request of the same kind joins it,
within a cell budget and the device-memory budget (admission by the footprint the library reports
for that batch shape). Batches run concurrently, each system on its own stream, with all state
resident in HBM from the initial upload to the final read-back. Requests that arrive while
batches run join the next batch that a free lane forms. Memory is returned to the budget when a
batch completes.

Every instance's result depends only on its own request: its initial state and its device noise
are derived from the request's seed, the noise is keyed by the instance seed and the local cell
index, and FIRE keeps per-instance state. So a request gives the same result alone and in a mix,
up to the order of floating-point atomics; with ``Server(deterministic=True)`` (fixed-point force
sums) an SPP request's positions are the same bits in any mix, and reruns of a batch repeat
exactly.

The reference has no serving layer; this drives the same kernels as the class API
(``VoronoiQuadraticEnergy``/``VertexQuadraticEnergy`` with ``selfPropelledParticleDynamics``,
``selfPropelledCellVertexDynamics`` and ``EnergyMinimizerFIRE``).
"""
from __future__ import annotations

import collections
import ctypes as C
import dataclasses
import math
import threading
import time
from concurrent.futures import Future

import numpy as np

from ._lib import FireParams, load
from .models import VertexBatch, VoronoiBatch


@dataclasses.dataclass
class Request:
    model: str                 # "voronoi" or "vertex"
    task: str                  # "spp" (fixed-step self-propelled dynamics) or "fire"
    n: int                     # cells
    p0: float = 3.8            # preferred shape index (A0 = 1)
    seed: int = 0              # initial positions, directors and device noise
    steps: int = 2000          # SPP steps
    v0: float = 0.05
    dt: float = 0.01
    fire_tol: float = 1e-10    # FIRE: stop when sqrt(max |F|^2) <= fire_tol
    fire_max_iterations: int = 10000
    rid: int = -1

    def key(self):
        """Requests with equal keys can share a batch. FIRE batches also group sizes by factor-of-4
        classes so that small requests do not wait for large ones to converge."""
        if self.task == "spp":
            return (self.model, "spp", self.steps, self.dt)
        return (self.model, "fire", self.fire_tol, self.fire_max_iterations, int(math.log(self.n, 4)))


@dataclasses.dataclass
class Result:
    rid: int
    positions: np.ndarray      # cells (Voronoi) or vertices (vertex model)
    energy: float
    work: int                  # cell-steps (SPP) or cell-iterations (FIRE)
    iterations: int            # SPP steps or FIRE iterations
    fmax: float                # FIRE: final sqrt(max |F|^2); SPP: nan
    t_submit: float
    t_start: float
    t_done: float
    batch_requests: int
    batch_cells: int

    @property
    def latency(self):
        return self.t_done - self.t_submit


def initial_state(req):
    """Seeded uniform positions in a square box of side sqrt(N) (mean cell area 1) and directors."""
    rng = np.random.default_rng([int(req.seed) & (2**63 - 1), 17])
    L = math.sqrt(req.n)
    pos = rng.random((req.n, 2)) * L
    theta = rng.uniform(0.0, 2.0 * math.pi, req.n)
    return L, pos, theta


def instance_seed(req):
    return int(np.random.default_rng([int(req.seed) & (2**63 - 1), 29]).integers(0, 2**63))


def footprint(model, sizes, K=16, vmax=30, deterministic=False):
    """Device bytes of a batch with these instance sizes, plus FIRE and staging buffers allocated
    on first use (velocities, per-dof instance index, and in the deterministic mode the fixed-point
    accumulators)."""
    lib = load()
    arr = np.ascontiguousarray(sizes, dtype=np.int32)
    if model == "voronoi":
        base = lib.cg_voronoi_footprint(len(arr), arr.ctypes.data, K)
        dofs = int(arr.sum())
    else:
        base = lib.cg_vertex_footprint(len(arr), arr.ctypes.data, vmax)
        dofs = 2 * int(arr.sum())
    det = (64 * dofs + 24 * len(arr)) if deterministic else 0
    return int(base + 24 * dofs + 8 * int(arr.sum()) + 256 * len(arr) + det + (1 << 16))


def device_memory():
    f, t = C.c_size_t(0), C.c_size_t(0)
    if load().cg_device_memory(C.byref(f), C.byref(t)) != 0:
        raise RuntimeError("cg_device_memory failed")
    return f.value, t.value


def run_batch(reqs, deterministic=False):
    """Run one batch of same-kind requests to completion on its own system (and stream); return
    per-request (positions, energy, iterations, fmax). deterministic: fixed-point force sums and
    fixed-order FIRE reductions (cg_set_deterministic)."""
    model, task = reqs[0].model, reqs[0].task
    states = [initial_state(r) for r in reqs]
    Ns = [r.n for r in reqs]
    boxes = [(L, L) for L, _, _ in states]
    pos = np.concatenate([p for _, p, _ in states])
    if model == "voronoi":
        b = VoronoiBatch(Ns, boxes)
        b.set_positions(pos)
    else:
        b = VertexBatch(Ns, boxes)
        b.from_cells(pos)
    try:
        if deterministic:
            b.set_deterministic(True)
        b.set_preferences(np.concatenate([np.tile([1.0, r.p0], (r.n, 1)) for r in reqs]))
        b.set_instance_seeds([instance_seed(r) for r in reqs])
        if task == "spp":
            b.set_directors(np.concatenate([t for _, _, t in states]))
            b.set_motility(np.concatenate([np.tile([r.v0, 1.0], (r.n, 1)) for r in reqs]))
            if model == "voronoi":
                b.triangulate()
            b.spp_run(reqs[0].steps, dt=reqs[0].dt)
            its = np.full(len(reqs), reqs[0].steps)
            fmax = np.full(len(reqs), np.nan)
        else:
            if model == "voronoi":
                b.triangulate()
            b.fire_minimize(FireParams.defaults(force_cutoff=reqs[0].fire_tol,
                                                max_iterations=reqs[0].fire_max_iterations))
            its, fmax, _ = b.fire_state()  # fmax = sqrt(max |F|^2) per instance
        P = b.positions()
        E = b.energies()
    finally:
        b.close()
    out = []
    off = 0
    for i, r in enumerate(reqs):
        m = r.n if model == "voronoi" else 2 * r.n
        out.append((P[off:off + m].copy(), float(E[i]), int(its[i]), float(fmax[i])))
        off += m
    return out


class Server:
    """Continuous-batching request loop over ``lanes`` concurrent batches.

    memory_budget: bytes of device memory the resident batches may hold (default: 70 % of the
    device's total memory). max_batch_cells / max_batch_requests bound one batch. deterministic:
    run every batch with order-independent sums (reproducible results)."""

    def __init__(self, lanes=4, memory_budget=None, max_batch_cells=1 << 20, max_batch_requests=512,
                 deterministic=False):
        if memory_budget is None:
            _, total = device_memory()
            memory_budget = int(0.7 * total)
        self.budget = int(memory_budget)
        self.deterministic = bool(deterministic)
        self.max_cells = int(max_batch_cells)
        self.max_reqs = int(max_batch_requests)
        self.queue = collections.deque()
        self.cond = threading.Condition()
        self.resident = 0
        self.peak_resident = 0
        self.closing = False
        self.batches = 0
        self._rid = 0
        self.threads = [threading.Thread(target=self._lane, daemon=True) for _ in range(int(lanes))]
        for t in self.threads:
            t.start()

    def submit(self, req: Request) -> Future:
        fut = Future()
        with self.cond:
            if req.rid < 0:
                req.rid = self._rid
            self._rid += 1
            self.queue.append((req, fut, time.perf_counter()))
            self.cond.notify()
        return fut

    def submit_many(self, reqs):
        """Queue several requests at once (they are visible to the lanes together)."""
        futs = []
        with self.cond:
            for req in reqs:
                if req.rid < 0:
                    req.rid = self._rid
                self._rid += 1
                fut = Future()
                self.queue.append((req, fut, time.perf_counter()))
                futs.append(fut)
            self.cond.notify_all()
        return futs

    def close(self):
        with self.cond:
            self.closing = True
            self.cond.notify_all()
        for t in self.threads:
            t.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _take(self):
        """Under the lock: the next batch (same kind as the oldest request, admitted by footprint),
        or None when closing with an empty queue."""
        while True:
            if self.queue:
                head = self.queue[0][0]
                key = head.key()
                picked, cells, fp = [], 0, 0
                for item in self.queue:
                    r = item[0]
                    if r.key() != key:
                        continue
                    if picked and (cells + r.n > self.max_cells or len(picked) >= self.max_reqs):
                        break
                    f = footprint(head.model, [x[0].n for x in picked] + [r.n], deterministic=self.deterministic)
                    if self.resident + f > self.budget:
                        break
                    picked.append(item)
                    cells += r.n
                    fp = f
                if picked:
                    for item in picked:
                        self.queue.remove(item)
                    self.resident += fp
                    self.peak_resident = max(self.peak_resident, self.resident)
                    return picked, fp
                if self.resident == 0:
                    # the oldest request alone exceeds the budget: it can never be admitted
                    req, fut, _ = self.queue.popleft()
                    fut.set_exception(MemoryError(f"request {req.rid} needs more than the memory budget"))
                    continue
            elif self.closing:
                return None
            self.cond.wait()

    def _lane(self):
        while True:
            with self.cond:
                got = self._take()
            if got is None:
                return
            items, fp = got
            reqs = [it[0] for it in items]
            t_start = time.perf_counter()
            try:
                outs = run_batch(reqs, self.deterministic)
                err = None
            except Exception as e:  # the failure belongs to this batch's requests
                outs, err = None, e
            t_done = time.perf_counter()
            with self.cond:
                self.resident -= fp
                self.batches += 1
                self.cond.notify_all()
            cells = sum(r.n for r in reqs)
            for k, (r, fut, t_sub) in enumerate(items):
                if err is not None:
                    fut.set_exception(err)
                    continue
                P, E, its, fmax = outs[k]
                fut.set_result(Result(r.rid, P, E, r.n * its, its, fmax, t_sub, t_start, t_done,
                                      len(reqs), cells))


def request_stream(n_requests, seed=2026, n_min=100, n_max=65536, fire_fraction=0.5, vertex_fraction=0.4,
                   steps=2000, fire_tol=1e-10, fire_max_iterations=10000):
    """The serving workload: Voronoi 60 % / vertex 40 %, N log-uniform in [n_min, n_max], p0 uniform
    in [3.6, 4.0], each request FIRE to fire_tol or `steps` SPP steps (v0 = 0.05, dt = 0.01); all
    seeds derived from (seed, request id)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_requests):
        model = "vertex" if rng.random() < vertex_fraction else "voronoi"
        task = "fire" if rng.random() < fire_fraction else "spp"
        n = int(round(math.exp(rng.uniform(math.log(n_min), math.log(n_max)))))
        out.append(Request(model, task, n, p0=float(rng.uniform(3.6, 4.0)),
                           seed=int(np.random.default_rng([seed, i]).integers(0, 2**62)),
                           steps=steps, fire_tol=fire_tol, fire_max_iterations=fire_max_iterations, rid=i))
    return out


def serve_poisson(requests, rate, lanes=4, memory_budget=None):
    """Submit `requests` at Poisson arrival times of the given rate (requests/s) and wait for all.
    Returns (results in request order, makespan seconds, server stats)."""
    arr_rng = np.random.default_rng(12345)
    gaps = arr_rng.exponential(1.0 / rate, len(requests)) if rate and rate > 0 else np.zeros(len(requests))
    with Server(lanes=lanes, memory_budget=memory_budget) as srv:
        t0 = time.perf_counter()
        t_next = t0
        futs = []
        for r, g in zip(requests, gaps):
            t_next += g
            d = t_next - time.perf_counter()
            if d > 0:
                time.sleep(d)
            futs.append(srv.submit(r))
        res = [f.result() for f in futs]
        stats = {"batches": srv.batches, "peak_resident_bytes": srv.peak_resident, "budget_bytes": srv.budget}
    makespan = max(r.t_done for r in res) - t0
    return res, makespan, stats


def summarize(results, makespan):
    lat = np.array([r.latency for r in results])
    work = sum(r.work for r in results)
    return {"requests": len(results), "p50_latency_s": float(np.percentile(lat, 50)),
            "p99_latency_s": float(np.percentile(lat, 99)), "mean_latency_s": float(lat.mean()),
            "cell_steps_per_s": work / makespan, "makespan_s": makespan, "work_cell_steps": int(work),
            "mean_batch_requests": float(np.mean([r.batch_requests for r in results]))}
