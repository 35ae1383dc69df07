"""Benchmark of the Voronoi SPP timestep on B200 (cell-steps/s).

Workload (default): the single large monolayer -- N = 262144 cells, periodic box 512 x 512, seeded
uniform positions, A0 = 1, p0 = 3.8, KA = KP = 1, v0 = 0.1, Dr = 1, dt = 0.01, SPP dynamics with a
Delaunay test/repair every step. Synthetic seeded data (the reference ships no dataset).

A "step" = one full timestep of the whole monolayer: fused geometry + forces + exact Delaunay test,
local repair, SPP integrate + move. The L2 (126 MB) is flushed (a 256 MB write) between timed steps.
Timing: CUDA events on the system's stream around each step, max over ranks.

--impl reference: the reference's CPU path on this host (oracle/_ref build of the reference's own
sources when present, else the oracle port), bounded sample of the same workload.
Multi-GPU: independent replicas, one per rank (weak scaling; the path has no exchange step).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-steps/s batched vs plain on 1 B200 at ≤1e-6 force err; p50/p99 latency"
N_CELLS = 262144
BOX = 512.0
P0, V0, DR, DT, MU = 3.8, 0.1, 1.0, 0.01, 1.0
# compulsory bytes of the fused geometry+force(+test) pass per cell: R pos 16, nn 4, nbr 24 (z=6),
# A0/P0 16; W A/P 16, F 16
FORCE_PASS_BYTES = 92
L2_FLUSH_BYTES = 256 << 20
REPAIR_TUNE_STEPS = 5  # cg_autotune_repair runs 12 x this many real steps
RUNAHEAD_CYCLES = 50_000_000  # ~25 ms device spin before a timed loop so no host gap is timed


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks sampled during the timed region."""

    def __init__(self, gpu_index=0):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
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

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_system(cg, torch, stream, precision, n_cells=N_CELLS, box=BOX, seed=1):
    b = cg.VoronoiBatch([n_cells], [(box, box)], K=16, precision=precision)
    rng = np.random.default_rng(seed)
    b.set_positions(rng.random((n_cells, 2)) * box)
    b.set_directors(rng.uniform(0, 2 * np.pi, n_cells))
    b.set_motility(np.tile([V0, DR], (n_cells, 1)))
    b.set_preferences(np.tile([1.0, P0], (n_cells, 1)))
    b.set_seed(seed)
    b._lib.cg_set_stream(b.handle, stream.cuda_stream)
    b.triangulate()
    return b


def save_state(b, path):
    """The prepared monolayer (positions, directors, Delaunay rows) as a compressed .npz."""
    b.enforce_topology()
    nn, nbr = b.topology()
    np.savez_compressed(path, pos=b.positions(), theta=b.directors(), nn=nn, nbr=nbr)


def load_state(cg, stream, precision, path):
    """A system of the default workload's parameters in a state saved by save_state."""
    d = np.load(path)
    b = cg.VoronoiBatch([N_CELLS], [(BOX, BOX)], K=int(d["nbr"].shape[1]), precision=precision)
    b.set_positions(d["pos"])
    b.set_directors(d["theta"])
    b.set_motility(np.tile([V0, DR], (N_CELLS, 1)))
    b.set_preferences(np.tile([1.0, P0], (N_CELLS, 1)))
    b.set_seed(1)
    b._lib.cg_set_stream(b.handle, stream.cuda_stream)
    b.set_topology(d["nn"], d["nbr"])
    return b


def time_steps(cg, torch, b, stream, steps, flush, max_attempts=8, dt=DT):
    """Device time of `steps` completed steps with an L2 flush between steps. A step that halts (the
    device repair could not finish it) is recovered by the host global rebuild (cg_poll), as the
    reference falls back to globalTriangulationCGAL; the halted attempt's time and the recovery's
    time (CUDA events around cg_poll: host round trips included) are both counted, and the halted
    step is then run again. Returns (total_s, completed, kernels, record of halts/recovery)."""
    import ctypes as C
    lib = b._lib
    total, done, kernels = 0.0, 0, 0
    rec = {"attempts": 0, "halts": 0, "recovery_s": 0.0}
    c0 = b.counters()
    while done < steps and rec["attempts"] < max_attempts:
        rec["attempts"] += 1
        want = steps - done
        s0 = C.c_int(0)
        lib.cg_poll(b.handle, C.byref(s0), None, 0)
        k0 = lib.cg_kernels_launched(b.handle)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(want)]
        with torch.cuda.stream(stream):
            torch.cuda._sleep(RUNAHEAD_CYCLES)  # let the host enqueue ahead of the device
            for i in range(want):
                flush.zero_()
                ev[i][0].record(stream)
                cg._lib.check(lib.cg_spp_enqueue(b.handle, 1, dt, MU))
                ev[i][1].record(stream)
        stream.synchronize()
        kernels += lib.cg_kernels_launched(b.handle) - k0
        s1, h = C.c_int(0), C.c_int(0)
        lib.cg_poll(b.handle, C.byref(s1), C.byref(h), 0)
        done += s1.value - s0.value
        total += sum(a.elapsed_time(e) for a, e in ev) / 1e3
        if h.value:
            rec["halts"] += 1
            r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            r0.record(stream)
            cg._lib.check(lib.cg_poll(b.handle, None, None, 1))  # global rebuild
            r1.record(stream)
            r1.synchronize()
            t = r0.elapsed_time(r1) / 1e3
            rec["recovery_s"] += t
            total += t
    c1 = b.counters()
    rec["global_rebuilds"] = int(c1.get("global_rebuilds", 0) - c0.get("global_rebuilds", 0))
    rec["restarred_cells"] = int(c1.get("cells_restarred", 0) - c0.get("cells_restarred", 0))
    rec["rows_changed"] = int(c1.get("rows_changed", 0) - c0.get("rows_changed", 0))
    return total, done, kernels, rec


def time_force_pass(cg, torch, b, stream, reps, flush):
    lib = b._lib
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    with torch.cuda.stream(stream):
        torch.cuda._sleep(RUNAHEAD_CYCLES)
        for i in range(reps):
            flush.zero_()
            ev[i][0].record(stream)
            cg._lib.check(lib.cg_launch_force_pass(b.handle, 1))
            ev[i][1].record(stream)
    stream.synchronize()
    return sum(a.elapsed_time(e) for a, e in ev) / reps / 1e3


def e2e_steps(cg, torch, b, stream, steps):
    """Public API with host buffers, every step: that step's noise copied in from pinned host memory
    (cg_spp_enqueue_host: copy stream, double-buffered, so the copy of step i+1 overlaps step i) and
    the per-instance energy after the step copied out to pinned host memory. The noise is drawn on
    the host before the timed region."""
    import ctypes as C
    lib = b._lib
    gen = np.random.default_rng(7)
    noise = torch.from_numpy(gen.standard_normal((steps, b.Ntot))).pin_memory()
    energy = torch.zeros((steps, 1), dtype=torch.float64).pin_memory()
    # warm-up (untimed): the first step on each of the two staging buffers captures its graph
    warm = torch.from_numpy(gen.standard_normal((2, b.Ntot))).pin_memory()
    for i in range(2):
        cg._lib.check(lib.cg_spp_enqueue_host(b.handle, C.c_void_p(warm[i].data_ptr()), DT, MU, None))
    s0 = C.c_int(0)
    lib.cg_poll(b.handle, C.byref(s0), None, 1)
    st, en = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    st.record(stream)
    for i in range(steps):
        cg._lib.check(lib.cg_spp_enqueue_host(b.handle, C.c_void_p(noise[i].data_ptr()), DT, MU,
                                              C.c_void_p(energy[i].data_ptr())))
    en.record(stream)
    en.synchronize()
    s1, h = C.c_int(0), C.c_int(0)
    lib.cg_poll(b.handle, C.byref(s1), C.byref(h), 1)
    ok = s1.value - s0.value
    if not np.all(np.isfinite(energy.numpy()[:ok])):
        ok = 0
    return st.elapsed_time(en) / 1e3, ok, 8 * b.Ntot, 8


def bench_serving(n_requests, lanes=4, calib=16):
    """Serving: Poisson request stream through the continuous-batching server (cellgpu_b200.serve).
    The arrival rate is 0.8x the service rate measured on a closed burst of `calib` requests from
    the same stream (the whole 10^4-request stream holds ~33 GB, far below 70 % of HBM, so the
    memory-filling rate of the workload spec cannot be reached; the rate saturates the GPU instead)."""
    import copy
    from cellgpu_b200 import serve as S
    reqs = S.request_stream(n_requests)
    burst = [copy.deepcopy(r) for r in S.request_stream(calib, seed=99)]
    res_c, span_c, _ = S.serve_poisson(burst, rate=0, lanes=lanes)
    rate = 0.8 * calib / span_c
    res, makespan, stats = S.serve_poisson(reqs, rate, lanes=lanes)
    out = S.summarize(res, makespan, reqs)
    out.update({"arrival_rate_per_s": rate, "lanes": lanes, "calibration_burst_s": span_c,
                "batches": stats["batches"], "rebuilds": stats["rebuilds"],
                "joined_running_batch": stats["joined_running_batch"],
                "peak_resident_bytes": stats["peak_resident_bytes"], "budget_bytes": stats["budget_bytes"],
                "workload": f"{n_requests} requests: 60% Voronoi / 40% vertex, N log-uniform [100, 65536], "
                            "p0 U[3.6,4.0], FIRE to 1e-10 (max 10^4 iterations) or 2000 SPP steps "
                            "(v0 0.05, dt 0.01), Poisson arrivals"})
    return out


def c4_ensemble(seed=4, n_inst=512):
    """512 monolayers, N log-uniform in [64, 8192], box sqrt(N), p0 U[3.6,4.0], v0 U[0.01,0.1]."""
    rng = np.random.default_rng(seed)
    Ns = np.round(np.exp(rng.uniform(np.log(64), np.log(8192), n_inst))).astype(int)
    boxes = [(float(np.sqrt(n)), float(np.sqrt(n))) for n in Ns]
    pos = [rng.random((n, 2)) * np.sqrt(n) for n in Ns]
    theta = [rng.uniform(0, 2 * np.pi, n) for n in Ns]
    p0 = rng.uniform(3.6, 4.0, n_inst)
    v0 = rng.uniform(0.01, 0.1, n_inst)
    return Ns, boxes, pos, theta, p0, v0


def time_enqueued(torch, stream, fn, reps, flush=None):
    """Device time of `reps` calls of fn (each enqueueing work on `stream`), runahead first."""
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    with torch.cuda.stream(stream):
        torch.cuda._sleep(RUNAHEAD_CYCLES)
        for i in range(reps):
            if flush is not None:
                flush.zero_()
            ev[i][0].record(stream)
            fn()
            ev[i][1].record(stream)
    stream.synchronize()
    return sum(a.elapsed_time(e) for a, e in ev) / 1e3


def bench_batched(cg, torch, flush, steps=5000, equil=150, plain_steps=20, plain_sample=48):
    """The batched-ensemble config: 512 monolayers run for `steps` steps in total. Batched arm: one
    system for all instances, one launch sequence per step; the first `equil` steps from the
    uniform random state are untimed (they rearrange the tissues wholesale), the remaining
    steps - equil are timed with the L2 flushed between steps, halts and their recovery included
    (time_steps). Plain arm: the single-instance drop-in, one system per monolayer, started from
    the batched arm's equilibrated state; a sample of instances, one step of each per round, the L2
    flushed between rounds as between the batched steps. FP64 and mixed precision."""
    import ctypes as C
    Ns, boxes, pos, theta, p0, v0 = c4_ensemble()
    total = int(Ns.sum())
    out = {"n_instances": len(Ns), "cells": total, "steps_total": steps, "steps_untimed": equil}
    for name, prec in (("fp64", cg.CG_FP64), ("mixed", cg.CG_MIXED)):
        b = cg.VoronoiBatch(list(Ns), boxes, precision=prec)
        b.set_positions(np.concatenate(pos))
        b.set_directors(np.concatenate(theta))
        b.set_motility(np.concatenate([np.tile([v, 1.0], (n, 1)) for n, v in zip(Ns, v0)]))
        b.set_preferences(np.concatenate([np.tile([1.0, p], (n, 1)) for n, p in zip(Ns, p0)]))
        st = torch.cuda.Stream()
        b._lib.cg_set_stream(b.handle, st.cuda_stream)
        b.triangulate()
        b.spp_run(equil - 12 * REPAIR_TUNE_STEPS, dt=DT, mu=MU)
        b.spatial_sort()
        out[f"batched_{name}_autotune"] = b.autotune()
        # the repair grids are timed on real steps: the last 12 x REPAIR_TUNE_STEPS untimed ones
        out[f"batched_{name}_autotune_repair"] = b.autotune_repair(REPAIR_TUNE_STEPS, dt=DT, mu=MU)
        t, done, _, rec = time_steps(cg, torch, b, st, steps - equil, flush)
        out[f"batched_{name}"] = total * done / t
        out[f"batched_{name}_ms_per_step"] = 1e3 * t / max(done, 1)
        out[f"batched_{name}_timed_steps"] = done
        out[f"batched_{name}_timed_window"] = rec
        if name == "fp64":
            keep_state = (b.positions(), b.directors())
        del b
    # plain: the single-instance drop-in, one system per monolayer, sampled over a subset (the
    # sort keeps every cell inside its instance's index range)
    rng = np.random.default_rng(11)
    sample = rng.choice(len(Ns), plain_sample, replace=False)
    systems = []
    allpos, allth = keep_state
    offs = np.concatenate([[0], np.cumsum(Ns)])
    st = torch.cuda.Stream()
    for i in sample:
        s = cg.VoronoiBatch([int(Ns[i])], [boxes[i]])
        s.set_positions(allpos[offs[i]:offs[i + 1]])
        s.set_directors(allth[offs[i]:offs[i + 1]])
        s.set_motility(np.tile([v0[i], 1.0], (Ns[i], 1)))
        s.set_preferences(np.tile([1.0, p0[i]], (Ns[i], 1)))
        s._lib.cg_set_stream(s.handle, st.cuda_stream)
        s.triangulate()
        s.spp_run(5, dt=DT, mu=MU)
        systems.append(s)

    def one_round():
        for s in systems:
            cg._lib.check(s._lib.cg_spp_enqueue(s.handle, 1, DT, MU))

    t = time_enqueued(torch, st, one_round, plain_steps, flush)
    halted = 0
    for s in systems:
        h = C.c_int(0)
        s._lib.cg_poll(s.handle, None, C.byref(h), 1)
        halted += h.value
    cells = int(Ns[sample].sum())
    out["plain_fp64"] = cells * plain_steps / t
    out["plain_sample_instances"] = len(sample)
    out["plain_steps"] = plain_steps
    out["plain_halted_instances"] = halted
    out["plain_l2"] = "flushed between rounds (one step of every sampled instance per round)"
    out["batched_over_plain_fp64"] = out["batched_fp64"] / out["plain_fp64"]
    out["batched_mixed_over_plain_fp64"] = out["batched_mixed"] / out["plain_fp64"]
    return out


def profile_c4_steps(cg, torch, steps):
    """A profiler target: the 512-monolayer ensemble prepared as bench_batched prepares it (150 steps from the
    random state, spatial sort, autotune, repair autotune), 200 further steps, then `steps` steps
    with supplied noise through plain launches, so that every kernel is a launch of its own, with
    the CUDA profiler switched on for those steps only (ncu --profile-from-start off). Returns the
    counters of those steps."""
    Ns, boxes, pos, theta, p0, v0 = c4_ensemble()
    b = cg.VoronoiBatch(list(Ns), boxes, precision=cg.CG_FP64)
    b.set_positions(np.concatenate(pos))
    b.set_directors(np.concatenate(theta))
    b.set_motility(np.concatenate([np.tile([v, 1.0], (n, 1)) for n, v in zip(Ns, v0)]))
    b.set_preferences(np.concatenate([np.tile([1.0, p], (n, 1)) for n, p in zip(Ns, p0)]))
    b.triangulate()
    b.spp_run(150, dt=DT, mu=MU)
    b.spatial_sort()
    b.autotune()
    b.autotune_repair(REPAIR_TUNE_STEPS, dt=DT, mu=MU)
    b.spp_run(200, dt=DT, mu=MU)
    noise = torch.randn(steps, int(Ns.sum()), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    c0 = b.counters()
    torch.cuda.profiler.start()
    b.spp_run(steps, dt=DT, mu=MU, noise=noise)
    torch.cuda.synchronize()
    torch.cuda.profiler.stop()
    c1 = b.counters()
    return {k: c1[k] - c0[k] for k in c1}


def bench_c1(cg, torch, flush, steps=1000, cpu=True):
    """The reference's own small case (plain FP64, single instance, the drop-in's latency case): N = 300
    cells in a box of side sqrt(N) from seeded uniform positions, A0 = 1, p0 = 3.8, SPP v0 = 0.05,
    Dr = 1, dt = 0.01, `steps` steps with a Delaunay test/repair every step. GPU: every step timed,
    L2 flushed between steps, halts and recovery included; CPU: the reference's CPU path (local
    test-and-repair and the default global retriangulation) on one core, same workload."""
    n = 300
    L = float(np.sqrt(n))
    rng = np.random.default_rng(1)
    b = cg.VoronoiBatch([n], [(L, L)], K=16)
    b.set_positions(rng.random((n, 2)) * L)
    b.set_directors(rng.uniform(0, 2 * np.pi, n))
    b.set_motility(np.tile([0.05, 1.0], (n, 1)))
    b.set_preferences(np.tile([1.0, 3.8], (n, 1)))
    st = torch.cuda.Stream()
    b._lib.cg_set_stream(b.handle, st.cuda_stream)
    b.triangulate()
    for _ in range(3):  # warm-up: graph capture
        cg._lib.check(b._lib.cg_spp_enqueue(b.handle, 1, 0.01, MU))
    b._lib.cg_poll(b.handle, None, None, 1)
    t, done, _, rec = time_steps(cg, torch, b, st, steps, flush, dt=0.01)
    out = {"workload": "voronoi_spp_N300 (box sqrt(300), v0 0.05, 1000 steps)", "cells": n, "steps": done,
           "gpu_cell_steps_per_s": n * done / t, "gpu_ms_per_step": 1e3 * t / max(done, 1),
           "timed_window": rec, "l2": "flushed between timed steps"}
    b.close()
    if cpu:
        try:
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import ref_harness
            if ref_harness.available():
                loc = ref_harness.bench_c1(steps, local_repair=True)
                glo = ref_harness.bench_c1(steps, local_repair=False)
                out["cpu_reference_local"] = loc
                out["cpu_reference_global"] = glo
                best = max(loc["value"], glo["value"])
                out["gpu_over_cpu_reference_best_mode"] = out["gpu_cell_steps_per_s"] / best
        except Exception as e:
            out["cpu_reference_error"] = str(e)
    return out


def bench_vertex(cg, torch, flush, steps=10000, fire=True):
    """The vertex-model config: Nc = 16384 cells / 32768 vertices from the Voronoi dual of seeded
    uniform points in a box of side 128, A0 = 1, p0 U[3.7,3.9] per cell, T1 threshold 0.04,
    Brownian T = 1e-3, dt = 0.005 for 10^4 steps (the whole run is timed: the first ~10^3 steps
    relax the random dual with many T1 flips, the rest is the steady state), then FIRE to
    sqrt(max|F|^2) <= 1e-12 (at most 10^5 iterations)."""
    Nc, L = 16384, 128.0
    rng = np.random.default_rng(3)
    b = cg.VertexBatch([Nc], [(L, L)], vmax=30)
    st = torch.cuda.Stream()
    b._lib.cg_set_stream(b.handle, st.cuda_stream)
    b.from_cells(rng.random((Nc, 2)) * L)
    b.set_preferences(np.stack([np.ones(Nc), rng.uniform(3.7, 3.9, Nc)], 1))
    b.set_t1_threshold(0.04)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    segments = []
    done = 0
    f0 = 0
    ev0.record(st)
    for seg in (1000, steps - 1000):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        b.brownian_run(seg, dt=0.005, mu=1.0, T=1e-3)
        e1.record(st)
        e1.synchronize()
        f1 = b.counters()["t1_flips"]
        segments.append({"steps": seg, "ms_per_step": e0.elapsed_time(e1) / seg, "t1_flips": f1 - f0})
        f0 = f1
        done += seg
    ev1.record(st)
    ev1.synchronize()
    t = ev0.elapsed_time(ev1) / 1e3
    out = {"cells": Nc, "vertices": 2 * Nc, "steps": done, "brownian_cell_steps_per_s": Nc * done / t,
           "brownian_ms_per_step": 1e3 * t / done, "t1_flips": b.counters()["t1_flips"],
           "segments": segments}
    if fire:
        p = cg.FireParams.defaults(force_cutoff=1e-12, max_iterations=100000)
        ev0.record(st)
        b.fire_minimize(p)
        ev1.record(st)
        ev1.synchronize()
        it, fmax, fnorm = b.fire_state()
        tf = ev0.elapsed_time(ev1) / 1e3
        out.update({"fire_iterations": int(it[0]), "fire_fmax": float(fmax[0]), "fire_fnorm_mean_conv": float(fnorm[0]),
                    "fire_s": tf, "fire_cell_iterations_per_s": Nc * int(it[0]) / tf})
    return out


def replica_aggregate(total_s, done, n_cells, world, device):
    """Whole-job throughput of `world` independent replicas (one per rank, no exchange on the step
    path): the time is the max over ranks of the device-timed region, the work is the sum of the
    cell-steps every rank completed. Collective: every rank calls it at the same point."""
    units = float(done * n_cells)
    if world > 1:
        import torch
        import torch.distributed as dist
        t = torch.tensor([total_s], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        u = torch.tensor([units], dtype=torch.float64, device=device)
        dist.all_reduce(u, op=dist.ReduceOp.SUM)
        total_s, units = float(t.item()), float(u.item())
    return (units / total_s if total_s > 0 else 0.0), total_s


def bench_deterministic(cg, torch, stream, flush, precision, steps, equilibrate, sort):
    """The same monolayer with order-independent fixed-point force sums (cg_set_deterministic, the
    mode Simulation::setReproducible selects), prepared and timed as the main line: per-step device
    time with the L2 flushed between steps."""
    b = make_system(cg, torch, stream, precision, seed=1)
    b.set_deterministic(True)
    if equilibrate > 0:
        b.spp_run(equilibrate, dt=DT, mu=MU)
    if sort:
        b.spatial_sort()
    for _ in range(3):
        cg._lib.check(b._lib.cg_spp_enqueue(b.handle, 1, DT, MU))
    b._lib.cg_poll(b.handle, None, None, 1)
    torch.cuda.synchronize()
    total, done, _, rec = time_steps(cg, torch, b, stream, steps, flush)
    b.close()
    return {"value": N_CELLS * done / total if total > 0 else 0.0, "unit": "cell-steps/s",
            "ms_per_step": 1e3 * total / max(done, 1), "steps": done, "timed_window": rec,
            "force_sums": "fixed point (deterministic mode)"}


def workload_config(precision, world, sort=True, deterministic=False):
    return {"workload": "voronoi_spp_N262144_L512", "n_cells": N_CELLS, "box": BOX, "p0": P0, "v0": V0,
            "Dr": DR, "dt": DT, "precision": precision, "l2": "flushed (256 MB write) between timed steps",
            "spatial_sort": "Hilbert order once after equilibration" if sort else "none",
            "force_sums": "fixed point (deterministic mode)" if deterministic else "floating-point atomics",
            "parallelism": f"replicas{world}"}


def cpu_baseline_port(n_cells=N_CELLS, box=BOX, steps=3, seed=1):
    """Oracle port of the reference CPU path, 1 thread, on the same monolayer."""
    from oracle import oracle as O
    rng = np.random.default_rng(seed)
    pos = rng.random((n_cells, 2)) * box
    theta = rng.uniform(0, 2 * np.pi, n_cells)
    nn, nbr = O.periodic_delaunay(pos, (box, box), 16)
    mot = np.tile([V0, DR], (n_cells, 1))
    pref = np.tile([1.0, P0], (n_cells, 1))
    noise = np.random.default_rng(seed + 1).standard_normal((steps, n_cells))
    t0 = time.perf_counter()
    O.voronoi_spp_run(pos, (box, box), nn, nbr, theta, mot, pref, noise, dt=DT, mu=MU)
    t = time.perf_counter() - t0
    return {"value": n_cells * steps / t, "unit": "cell-steps/s", "cores": 1, "kind": "port",
            "sample": f"{steps} SPP steps of the N={n_cells} monolayer (full Delaunay rebuild per step)"}


def cpu_reference(steps, all_cores=False, global_steps=0):
    """The reference's CPU path (oracle/_ref, its own sources) on a relaxed sample of the workload:
    one instance on one core, or one instance per host core; the oracle port when _ref is absent.
    On one core the record is the faster of the local test-and-repair mode and the default global
    retriangulation mode (`global_steps` steps of it on the same state), with the other beside it."""
    ref = os.path.join(ROOT, "oracle", "_ref", "libcgref.so")
    if os.path.exists(ref):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import ref_harness  # noqa
        if all_cores:
            return ref_harness.bench_c2_all_cores(steps)
        state = ref_harness.relaxed_c2_state(n_tile=N_CELLS // 16, reps=4, v0=V0, seed=1)
        rec = ref_harness.bench_c2(steps, state=state)
        if global_steps > 0:
            glo = ref_harness.bench_c2(global_steps, state=state, local_repair=False)
            rec["global_mode"] = {k: glo[k] for k in ("value", "unit", "sample")}
            if glo["value"] > rec["value"]:  # report the faster mode as the baseline
                glo["local_mode"] = {k: rec[k] for k in ("value", "unit", "sample")}
                rec = glo
        return rec
    return cpu_baseline_port(steps=steps)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--deterministic", action="store_true",
                    help="order-independent fixed-point force sums (cg_set_deterministic), the mode "
                         "Simulation.setReproducible(true) selects")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-steps", type=int, default=0,
                    help="run this many SPP steps through plain kernel launches (supplied noise, no "
                         "graph) after preparing the state, then exit (profiling)")
    ap.add_argument("--no-repair-tune", action="store_true",
                    help="keep the default repair-round grids (no cg_autotune_repair before timing)")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the batched-ensemble and vertex-model measurements")
    ap.add_argument("--serve-requests", type=int, default=2000,
                    help="requests in the serving extra (about 2.5 minutes for 2000); 0 skips it")
    ap.add_argument("--serve-only", action="store_true",
                    help="run only the serving stream and print its JSON line")
    ap.add_argument("--case", default="c2", choices=["c1", "c2", "c3", "c4"],
                    help="c2: the headline line (default); c1 / c3 / c4: only the small plain case, the "
                         "vertex-model or the batched-ensemble measurement, printed as one JSON line")
    ap.add_argument("--c3-steps", type=int, default=10000, help="Brownian steps of the c3 case")
    ap.add_argument("--c4-profile-steps", type=int, default=0,
                    help="with --case c4: prepare the ensemble, run this many plain-launch steps with "
                         "the CUDA profiler on, print their counters and exit (a profiler target)")
    ap.add_argument("--no-sort", action="store_true",
                    help="time the equilibrated monolayer in its creation order (no spatial re-sort)")
    ap.add_argument("--equilibrate", type=int, default=300,
                    help="untimed SPP steps from the random initial state before warm-up")
    ap.add_argument("--state-out", default=None,
                    help="save the prepared (equilibrated, sorted) monolayer to this .npz")
    ap.add_argument("--state-in", default=None,
                    help="start from a monolayer saved by --state-out instead of preparing one "
                         "(profiling runs: few launches before the measured ones)")
    ap.add_argument("--force-pass-only", type=int, default=0,
                    help="after preparing the state, launch the fused force pass this many times and "
                         "exit (a profiler target)")
    args = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        if rank != 0:
            return
        t0 = time.perf_counter()
        steps = max(1, min(args.steps, 20))
        base = cpu_reference(steps, all_cores=True)
        line = {"metric": METRIC, "value": base["value"], "unit": "cell-steps/s", "n_gpus": args.gpus,
                "steps": steps, "warmup": 0, "ms_per_step": 1e3 * N_CELLS / base["value"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic", "impl": "reference",
                "config": workload_config(args.precision, args.gpus),
                "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "wall_s": time.perf_counter() - t0}
        print(json.dumps(line))
        return

    import torch

    import cellgpu_b200 as cg
    from cellgpu_b200 import build as cgbuild

    if not os.path.exists(cgbuild.LIB):
        raise SystemExit("libcellgpu_b200.so missing: run __graft_entry__.build()")
    torch.cuda.set_device(local)
    if args.case != "c2":
        if rank == 0:
            flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
            if args.case == "c1":
                out = {"c1_plain": bench_c1(cg, torch, flush, cpu=not args.no_cpu_baseline)}
            elif args.case == "c3":
                out = {"c3_vertex": bench_vertex(cg, torch, flush, steps=max(1001, args.c3_steps))}
            elif args.c4_profile_steps > 0:
                out = {"c4_profile_counters": profile_c4_steps(cg, torch, args.c4_profile_steps)}
            else:
                out = {"c4_ensemble": bench_batched(cg, torch, flush)}
            print(json.dumps({"metric": METRIC, "impl": "ours", "n_gpus": 1, "case": args.case, **out}))
        return
    if args.serve_only:
        if rank == 0:
            out = bench_serving(max(1, args.serve_requests))
            print(json.dumps({"metric": "p50/p99 latency and cell-steps/s of a served request stream",
                              "impl": "ours", "n_gpus": 1, "c5_serving": out}))
        return
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    stream = torch.cuda.Stream()
    precision = cg.CG_FP64 if args.precision == "fp64" else cg.CG_MIXED
    if args.state_in:
        b = load_state(cg, stream, precision, args.state_in)
    else:
        b = make_system(cg, torch, stream, precision, seed=1 + rank)
    if args.deterministic:
        b.set_deterministic(True)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    if not args.state_in:
        # relax the random initial state (untimed): its first steps rearrange the tissue wholesale
        if args.equilibrate > 0:
            b.spp_run(args.equilibrate, dt=DT, mu=MU)
        # Hilbert-order the cells of the equilibrated monolayer once (untimed; the reference's
        # spatial sorting, Simple2DCell::spatiallySortCells): neighbours sit close in memory
        if not args.no_sort:
            b.spatial_sort()
    if args.state_out and rank == 0:
        save_state(b, args.state_out)
    if args.force_pass_only > 0:
        for _ in range(args.force_pass_only):
            cg._lib.check(b._lib.cg_launch_force_pass(b.handle, 1))
        torch.cuda.synchronize()
        print(json.dumps({"force_pass_launches": args.force_pass_only, "n_cells": N_CELLS}))
        return
    if args.plain_steps > 0:
        # profiling aid: SPP steps through plain kernel launches (supplied noise, no step graph, so
        # every repair kernel can be profiled), then exit
        gen = torch.Generator(device="cuda")
        gen.manual_seed(7)
        noise = torch.randn((args.plain_steps, N_CELLS), dtype=torch.float64, device="cuda", generator=gen)
        b.spp_run(args.plain_steps, dt=DT, mu=MU, noise=noise)
        torch.cuda.synchronize()
        print(json.dumps({"plain_steps": args.plain_steps, "n_cells": N_CELLS}))
        return
    # repair-round grids timed on real steps (untimed; 12 x REPAIR_TUNE_STEPS more relaxation steps)
    repair_tune = None if args.no_repair_tune else b.autotune_repair(REPAIR_TUNE_STEPS, dt=DT, mu=MU)
    # warm-up (untimed; graph capture happens here)
    for _ in range(max(3, args.warmup)):
        cg._lib.check(b._lib.cg_spp_enqueue(b.handle, 1, DT, MU))
    b._lib.cg_poll(b.handle, None, None, 1)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        total, done, kernels, timed_window = time_steps(cg, torch, b, stream, args.steps, flush)
    torch.cuda.synchronize()
    value, total = replica_aggregate(total, done, N_CELLS, world, "cuda")
    # dominant kernel: fused geometry + force + exact test
    t_force = time_force_pass(cg, torch, b, stream, 20, flush)
    hbm, kind = peaks()
    achieved = FORCE_PASS_BYTES * N_CELLS / t_force / 1e9
    # end to end through the host-buffer API
    e2e_t, e2e_ok, h2d, d2h = e2e_steps(cg, torch, b, stream, max(3, args.steps // 5))
    e2e_value, _ = replica_aggregate(e2e_t, e2e_ok, N_CELLS, world, "cuda")
    counters = b.counters()
    # mixed-precision force error on this (relaxed) state, against FP64
    F64 = None
    try:
        import ctypes as C
        bm = cg.VoronoiBatch([N_CELLS], [(BOX, BOX)], K=16, precision=cg.CG_MIXED if precision == cg.CG_FP64 else cg.CG_FP64)
        b.enforce_topology()  # the mixed perimeter derivative assumes a Delaunay triangulation
        nn, nbr = b.topology()
        bm.set_positions(b.positions())
        bm.set_topology(nn, nbr)
        bm.set_preferences(np.tile([1.0, P0], (N_CELLS, 1)))
        b.compute_forces()
        bm.compute_forces()
        Fa, Fb = b.forces(), bm.forces()
        F64, Fmx = (Fa, Fb) if precision == cg.CG_FP64 else (Fb, Fa)
        scale = float(np.sqrt(np.mean(np.sum(F64 ** 2, axis=1))))
        d = np.linalg.norm(Fmx - F64, axis=1)
        mixed_err = {"max": float(np.max(d / np.maximum(np.linalg.norm(F64, axis=1), scale))),
                     "rms": float(np.sqrt(np.mean(d ** 2)) / scale), "F_scale_rms": scale}
        del bm
    except Exception as e:
        mixed_err = {"error": str(e)}
    extras = {}
    if not args.no_extras and world == 1 and not args.deterministic:
        try:
            extras["c2_deterministic"] = bench_deterministic(cg, torch, stream, flush, precision, args.steps,
                                                             args.equilibrate, not args.no_sort)
        except Exception as e:
            extras["c2_deterministic"] = {"error": str(e)}
    if not args.no_extras and world == 1:
        try:
            extras["c1_plain"] = bench_c1(cg, torch, flush, cpu=not args.no_cpu_baseline)
        except Exception as e:
            extras["c1_plain"] = {"error": str(e)}
        try:
            extras["c4_ensemble"] = bench_batched(cg, torch, flush)
        except Exception as e:
            extras["c4_ensemble"] = {"error": str(e)}
        try:
            extras["c3_vertex"] = bench_vertex(cg, torch, flush)
        except Exception as e:
            extras["c3_vertex"] = {"error": str(e)}
        if args.serve_requests > 0:
            try:
                extras["c5_serving"] = bench_serving(args.serve_requests)
            except Exception as e:
                extras["c5_serving"] = {"error": str(e)}
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    cpu = None
    if not args.no_cpu_baseline and world == 1:
        try:
            cpu = cpu_reference(20, global_steps=3)
        except Exception as e:  # the baseline must not take the bench down
            cpu = {"error": str(e)}
    c4 = extras.get("c4_ensemble", {})
    ratios = {k: c4[k] for k in ("batched_over_plain_fp64", "batched_mixed_over_plain_fp64") if k in c4}
    # the force pass timed above: one thread per cell for FP64 with atomic sums, else 8-lane groups
    thread_form = precision == cg.CG_FP64 and not args.deterministic
    force_kernel = "k_voro_thread (force+test)" if thread_form else "k_voro_groups (force+test)"
    prof = os.path.join(ROOT, "profiles", "force_pass_traffic.json")
    traffic = None
    if os.path.exists(prof):
        with open(prof) as f:
            tr = json.load(f)
        traffic = tr.get("traffic_bytes_per_launch" if thread_form else "group_form_traffic_bytes_per_launch")
    line = {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": done,
        "warmup": max(3, args.warmup), "ms_per_step": 1e3 * total / max(done, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if precision == cg.CG_FP64 else "f32+f64",
        "data": "synthetic",
        "config": workload_config(args.precision, world, not args.no_sort, args.deterministic),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "kernel": force_kernel,
                     "kernel_ms": t_force * 1e3, "peak_kind": kind},
        "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(kernels),
        "clocks": clk.summary(),
        "batched_fp64_over_plain_fp64": ratios.get("batched_over_plain_fp64"),
        "batched_mixed_over_plain_fp64": ratios.get("batched_mixed_over_plain_fp64"),
        "timed_window": timed_window,
        "counters": counters,
        "equilibrate_steps": args.equilibrate,
        "repair_autotune": repair_tune,
        "mixed_force_error_vs_fp64": mixed_err,
        **extras,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line))


if __name__ == "__main__":
    main()
