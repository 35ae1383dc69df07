"""Serving: continuous batching of FIRE minimisations and fixed-step dynamics runs.

Requests (Voronoi or vertex model; SPP dynamics for a fixed number of steps, or FIRE to a force
norm) arrive at any time. Each of ``lanes`` worker threads runs one batch at a time: a system
holding many requests as instances, all state resident in HBM. A batch runs in chunks (SPP: a
number of steps; FIRE: a number of iterations). At every chunk end:
  * requests that have finished (SPP: their steps done; FIRE: converged or at the iteration cap)
    leave the batch and their results are returned at once;
  * queued requests of the batch's kind join it, as the device-memory budget allows (admission
    by the footprint the library reports for the new batch shape);
  * when requests joined, or finished ones hold half the batch, the batch is rebuilt as a new
    system: the running requests move into it with their whole state
    (cg_copy_instances) and continue exactly where they stopped, the new ones start fresh
    (cg_fire_begin_instances for FIRE), and the old system's memory returns to the budget.
A free lane takes the oldest queued request's kind and every queued request of that kind. Batches
run concurrently, each system on its own stream.

Every instance's result depends only on its own request: its initial state and its device noise
are derived from the request's seed, the noise is keyed by the instance seed, its own step count
and the local cell index, and FIRE keeps per-instance state that moves with the instance. So a
request gives the same result alone and in a mix, whether it started a batch or joined one, up to
the order of floating-point atomics; with ``Server(deterministic=True)`` (fixed-point force sums)
an SPP request's positions are the same bits in any mix.

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
    batch_requests: int        # requests in the batch during this request's last chunk
    batch_cells: int
    joined: bool = False       # admitted into a batch that was already running
    capped: bool = False       # FIRE: stopped at the iteration cap above the force threshold

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


SPP_CHUNK = 100     # SPP steps per chunk: requests join and leave a batch at chunk ends
FIRE_CHUNK = 256    # FIRE iterations per chunk


def spp_chunk(steps):
    """The chunk length of an SPP batch: the largest divisor of the request's steps up to SPP_CHUNK
    (every request of a batch has the same steps, so all finish at chunk ends)."""
    for c in range(min(SPP_CHUNK, steps), 0, -1):
        if steps % c == 0:
            return c
    return 1


def fire_params(req):
    return FireParams.defaults(force_cutoff=req.fire_tol, max_iterations=req.fire_max_iterations)


@dataclasses.dataclass
class _Slot:
    req: Request
    fut: Future
    t_sub: float
    t_start: float
    done: int = 0          # SPP steps done
    joined: bool = False
    index: int = -1        # instance index in the batch's current system


class RunningBatch:
    """One serving batch: a system and its requests as instances (in slot order). build() makes a
    new system from the slots still running (moved with their state) and new slots (fresh)."""

    def __init__(self, model, task, deterministic=False):
        self.model, self.task, self.det = model, task, bool(deterministic)
        self.b = None
        self.slots = []
        self.prm = None

    def build(self, fresh):
        """Replace the system by one holding the running slots (state moved) followed by `fresh`."""
        lib = load()
        surv = list(self.slots)
        order = surv + list(fresh)
        init = [initial_state(sl.req) for sl in order]
        Ns = [sl.req.n for sl in order]
        boxes = [(L, L) for L, _, _ in init]
        if self.model == "voronoi":
            nb = VoronoiBatch(Ns, boxes)
            pos = [p for _, p, _ in init]
            if surv:  # the running slots' current positions (their rows then come with the copy)
                P = self.b.positions()
                off = self.b.offsets
                for j, sl in enumerate(surv):
                    pos[j] = P[off[sl.index]:off[sl.index + 1]]
            nb.set_positions(np.concatenate(pos))
        else:
            # rows as wide as the running system's (they grow when a T1 transition needs it)
            nb = VertexBatch(Ns, boxes, vmax=self.b.row_capacity() if surv else 30)
            # the running slots' vertex state is overwritten by the copy below; their initial
            # cells only give the new system its shape
            nb.from_cells(np.concatenate([p for _, p, _ in init]))
        try:
            if self.det:
                nb.set_deterministic(True)
            nb.set_preferences(np.concatenate([np.tile([1.0, sl.req.p0], (sl.req.n, 1)) for sl in order]))
            nb.set_instance_seeds([instance_seed(sl.req) for sl in order])
            if self.task == "spp":
                nb.set_directors(np.concatenate([t for _, _, t in init]))
                nb.set_motility(np.concatenate([np.tile([sl.req.v0, 1.0], (sl.req.n, 1)) for sl in order]))
            if self.model == "voronoi":
                nb.triangulate()
            for j, sl in enumerate(surv):
                rc = lib.cg_copy_instances(nb.handle, j, self.b.handle, sl.index, 1)
                if rc != 0:
                    raise RuntimeError(f"cg_copy_instances failed: {lib.cg_last_error_string().decode()}")
            if self.task == "fire":
                self.prm = fire_params(order[0].req)
                if surv:
                    rc = lib.cg_fire_begin_instances(nb.handle, C.byref(self.prm), len(surv), len(fresh))
                    if rc != 0:
                        raise RuntimeError(lib.cg_last_error_string().decode())
                else:
                    nb.fire_begin(self.prm)
        except Exception:
            nb.close()
            raise
        if self.b is not None:
            self.b.close()
        self.b = nb
        self.slots = order
        for j, sl in enumerate(order):
            sl.index = j

    def run_chunk(self):
        """One chunk; returns the mask of slots that have finished."""
        if self.task == "spp":
            n = spp_chunk(self.slots[0].req.steps)
            self.b.spp_run(n, dt=self.slots[0].req.dt)
            for sl in self.slots:
                sl.done += n
            return np.array([sl.done >= sl.req.steps for sl in self.slots])
        self.b.fire_advance(self.prm, FIRE_CHUNK)
        its, fmax, _ = self.b.fire_state()
        self.its, self.fmax = its, fmax
        return np.array([its[sl.index] >= sl.req.fire_max_iterations or fmax[sl.index] <= sl.req.fire_tol
                         for sl in self.slots])

    def results(self, mask, t_done):
        """(slot, Result) of the slots in mask (mask follows self.slots); they leave the batch. A slot's
        instance in the system is sl.index: slots that left earlier stay in the system (frozen for
        FIRE) until the next rebuild."""
        P = self.b.positions()
        E = self.b.energies()
        off = self.b.offsets if self.model == "voronoi" else 2 * self.b.offsets
        cells = sum(sl.req.n for sl in self.slots)
        out, keep = [], []
        for m, sl in zip(mask, self.slots):
            if not m:
                keep.append(sl)
                continue
            j = sl.index
            r = sl.req
            if self.task == "spp":
                its, fm, capped = r.steps, float("nan"), False
            else:
                its, fm = int(self.its[j]), float(self.fmax[j])
                capped = fm > r.fire_tol
            res = Result(r.rid, P[off[j]:off[j + 1]].copy(), float(E[j]), r.n * its, its, fm, sl.t_sub,
                         sl.t_start, t_done, len(self.slots), cells, sl.joined, capped)
            out.append((sl, res))
        self.slots = keep
        return out

    def close(self):
        if self.b is not None:
            self.b.close()
            self.b = None


def run_batch(reqs, deterministic=False):
    """Run one batch of same-kind requests to completion on its own system (and stream); return
    per-request (positions, energy, iterations, fmax). deterministic: fixed-point force sums and
    fixed-order FIRE reductions (cg_set_deterministic)."""
    rb = RunningBatch(reqs[0].model, reqs[0].task, deterministic)
    now = time.perf_counter()
    slots = [_Slot(r, None, now, now) for r in reqs]
    rb.build(slots)
    done = {}
    try:
        while rb.slots:
            m = rb.run_chunk()
            if m.any():
                for sl, res in rb.results(m, time.perf_counter()):
                    done[id(sl)] = res
    finally:
        rb.close()
    return [(done[id(sl)].positions, done[id(sl)].energy, done[id(sl)].iterations, done[id(sl)].fmax)
            for sl in slots]


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
        self.rebuilds = 0    # batches rebuilt around their running requests
        self.joined = 0      # requests admitted into a running batch
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
                picked, fp = self._pick(head.key(), head.model, [])
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

    def _pick(self, key, model, running):
        """Under the lock: queued requests of this key that fit beside the `running` sizes, while the
        footprint of the resulting batch plus everything resident stays within the budget (a
        rebuilt batch's old system stays resident until the rebuild is done)."""
        picked, sizes = [], list(running)
        fp = footprint(model, sizes, deterministic=self.deterministic) if sizes else 0
        for item in self.queue:
            r = item[0]
            if r.key() != key:
                continue
            if sizes and (sum(sizes) + r.n > self.max_cells or len(sizes) >= self.max_reqs):
                break
            f = footprint(model, sizes + [r.n], deterministic=self.deterministic)
            if self.resident + f > self.budget:
                break
            picked.append(item)
            sizes.append(r.n)
            fp = f
        return picked, fp

    def _lane(self):
        while True:
            with self.cond:
                got = self._take()
            if got is None:
                return
            items, fp = got
            key = items[0][0].key()
            t0 = time.perf_counter()
            rb = RunningBatch(items[0][0].model, items[0][0].task, self.deterministic)
            fresh = [_Slot(r, fut, t_sub, t0) for r, fut, t_sub in items]
            try:
                rb.build(fresh)
                with self.cond:
                    self.batches += 1
                while rb.slots:
                    mask = rb.run_chunk()
                    freed = 0
                    if mask.any():
                        for sl, res in rb.results(mask, time.perf_counter()):
                            sl.fut.set_result(res)
                            freed += sl.req.n
                    if not rb.slots:
                        break
                    # admission into the running batch: queued requests of its kind, and a rebuild
                    # that returns the finished requests' memory while others wait
                    with self.cond:
                        running = [sl.req.n for sl in rb.slots]
                        picked, fp_new = self._pick(key, rb.model, running)
                        # finished requests still in the system (stepped, or frozen FIRE instances
                        # whose forces are still evaluated) once they hold half of it
                        dead = rb.b.Ntot - sum(running)
                        shrink = freed > 0 and dead >= sum(running)
                        rebuild = bool(picked) or shrink
                        if rebuild:
                            for item in picked:
                                self.queue.remove(item)
                            self.resident += fp_new  # held with the old system until the rebuild ends
                            self.peak_resident = max(self.peak_resident, self.resident)
                    if rebuild:
                        now = time.perf_counter()
                        joiners = [_Slot(r, fut, t_sub, now, joined=True) for r, fut, t_sub in picked]
                        try:
                            rb.build(joiners)
                        except Exception as e:
                            for sl in joiners:
                                sl.fut.set_exception(e)
                            raise
                        finally:
                            # the old system is gone (or, on failure, closed below): its memory
                            # returns to the budget and the new footprint is what this lane holds
                            with self.cond:
                                self.resident -= fp
                                self.rebuilds += 1
                                self.joined += len(joiners)
                                self.cond.notify_all()
                            fp = fp_new
            except Exception as e:  # the failure belongs to this batch's requests
                for sl in rb.slots + fresh:
                    if sl.fut is not None and not sl.fut.done():
                        sl.fut.set_exception(e)
            finally:
                rb.close()
                with self.cond:
                    self.resident -= fp
                    self.cond.notify_all()


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
        stats = {"batches": srv.batches, "rebuilds": srv.rebuilds, "joined_running_batch": srv.joined,
                 "peak_resident_bytes": srv.peak_resident, "budget_bytes": srv.budget}
    makespan = max(r.t_done for r in res) - t0
    return res, makespan, stats


def summarize(results, makespan, requests=None):
    """Latency percentiles (all requests; and FIRE requests that reached their threshold apart from
    those stopped at the iteration cap), aggregate cell-steps/s, batching statistics."""
    lat = np.array([r.latency for r in results])
    work = sum(r.work for r in results)
    out = {"requests": len(results), "p50_latency_s": float(np.percentile(lat, 50)),
           "p99_latency_s": float(np.percentile(lat, 99)), "mean_latency_s": float(lat.mean()),
           "cell_steps_per_s": work / makespan, "makespan_s": makespan, "work_cell_steps": int(work),
           "mean_batch_requests": float(np.mean([r.batch_requests for r in results])),
           "joined_running_batch_fraction": float(np.mean([r.joined for r in results]))}
    if requests is not None:
        fire = [r for q, r in zip(requests, results) if q.task == "fire"]
        spp = [r for q, r in zip(requests, results) if q.task == "spp"]
        conv = [r for r in fire if not r.capped]
        out["fire_requests"] = len(fire)
        out["fire_capped_fraction"] = float(np.mean([r.capped for r in fire])) if fire else None
        if conv:
            lc = np.array([r.latency for r in conv])
            out["fire_converged_p50_latency_s"] = float(np.percentile(lc, 50))
            out["fire_converged_p99_latency_s"] = float(np.percentile(lc, 99))
        if spp:
            ls = np.array([r.latency for r in spp])
            out["spp_p50_latency_s"] = float(np.percentile(ls, 50))
            out["spp_p99_latency_s"] = float(np.percentile(ls, 99))
    return out
