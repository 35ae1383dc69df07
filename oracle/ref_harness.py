"""TEST INFRASTRUCTURE ONLY: ctypes front end of oracle/_ref/libcgref.so, the reference's own CPU
sources (abaso/cellGPU src/...) compiled in place with the DelaunayCGAL stand-in (oracle/shim).
Only tests/ and bench.py's CPU-baseline / reference arm load it."""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libcgref.so")
_lib = None
_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def available():
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        L.ref_reproducible_normals.argtypes = [C.c_int, _dp]
        L.ref_voronoi_new.restype = C.c_void_p
        L.ref_voronoi_new.argtypes = [C.c_int, C.c_double, C.c_double]
        L.ref_free.argtypes = [C.c_void_p]
        L.ref_voronoi_set_state.argtypes = [C.c_void_p, _dp, C.c_void_p]
        L.ref_voronoi_set_motility.argtypes = [C.c_void_p, C.c_double, C.c_double]
        L.ref_voronoi_set_preferences.argtypes = [C.c_void_p, _dp]
        L.ref_voronoi_forces.restype = C.c_double
        L.ref_voronoi_forces.argtypes = [C.c_void_p, _dp, _dp]
        L.ref_voronoi_get.argtypes = [C.c_void_p, _dp, C.c_void_p, C.c_int, _ip, _ip]
        L.ref_voronoi_set_exclusions.argtypes = [C.c_void_p, _ip]
        L.ref_voronoi_external_forces.argtypes = [C.c_void_p, _dp]
        L.ref_voronoi_observables.argtypes = [C.c_void_p, _dp, C.c_double, _dp]
        L.ref_voronoi_spp_run.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int]
        L.ref_fire.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                               C.c_double, C.c_int, C.c_double, C.c_int]
        L.ref_vertex_new.restype = C.c_void_p
        L.ref_vertex_new.argtypes = [C.c_int, C.c_double, C.c_double]
        L.ref_vertex_counts.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ref_vertex_get.argtypes = [C.c_void_p, C.c_void_p, _dp, _ip, _ip, _ip, _ip]
        L.ref_vertex_set_positions.argtypes = [C.c_void_p, _dp]
        L.ref_vertex_set_preferences.argtypes = [C.c_void_p, _dp]
        L.ref_vertex_set_t1.argtypes = [C.c_void_p, C.c_double]
        L.ref_vertex_forces.restype = C.c_double
        L.ref_vertex_forces.argtypes = [C.c_void_p, _dp, _dp]
        L.ref_vertex_brownian_run.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double, C.c_double]
        L.ref_vertex_set_tension.argtypes = [C.c_void_p, _ip, C.c_double, C.c_int, C.c_void_p]
        L.ref_voronoi_tension_forces.restype = C.c_double
        L.ref_voronoi_tension_forces.argtypes = [C.c_int, _dp, _ip, _dp, C.c_double, C.c_int, C.c_void_p, _dp,
                                                 _dp]
        _lib = L
    return _lib


def voronoi_tension_forces(pos, types, pref, gamma=0.0, gammas=None):
    """The reference's VoronoiQuadraticEnergyWithTension (CPU branch) on one state: forces, A/P and
    computeEnergy(). gammas: an ntypes x ntypes matrix, else one gamma for unlike types."""
    pos = np.ascontiguousarray(pos, np.float64)
    n = len(pos)
    F = np.zeros((n, 2))
    AP = np.zeros((n, 2))
    g = None if gammas is None else np.ascontiguousarray(gammas, np.float64)
    nt = 0 if g is None else int(round(np.sqrt(g.size)))
    with quiet():
        E = lib().ref_voronoi_tension_forces(n, pos, np.ascontiguousarray(types, np.int32),
                                             np.ascontiguousarray(pref, np.float64), float(gamma), nt,
                                             None if g is None else g.ctypes.data_as(C.c_void_p), F, AP)
    return F, AP, E


class quiet:
    """Silence the reference's own console output (C stdio on fd 1) for the duration of a call, so a
    caller that prints one JSON line keeps its stdout clean."""

    def __enter__(self):
        import sys
        sys.stdout.flush()
        self._libc = C.CDLL(None)
        self._libc.fflush(None)
        self._saved = os.dup(1)
        self._null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self._null, 1)
        return self

    def __exit__(self, *exc):
        self._libc.fflush(None)
        os.dup2(self._saved, 1)
        os.close(self._saved)
        os.close(self._null)
        return False


def reproducible_normals(n):
    out = np.zeros(n)
    lib().ref_reproducible_normals(n, out)
    return out


class RefVoronoi:
    """VoronoiQuadraticEnergy of the reference, CPU branch."""

    def __init__(self, N, A0=1.0, P0=3.8):
        self.N = N
        self.h = lib().ref_voronoi_new(N, A0, P0)

    def __del__(self):
        try:
            lib().ref_free(self.h)
        except Exception:
            pass

    def set_state(self, pos, theta=None):
        pos = np.ascontiguousarray(pos, np.float64)
        th = None if theta is None else np.ascontiguousarray(theta, np.float64)
        lib().ref_voronoi_set_state(self.h, pos, None if th is None else th.ctypes.data_as(C.c_void_p))
        self._th = th

    def set_motility(self, v0, Dr):
        lib().ref_voronoi_set_motility(self.h, v0, Dr)

    def set_preferences(self, pref):
        lib().ref_voronoi_set_preferences(self.h, np.ascontiguousarray(pref, np.float64))

    def forces(self):
        F = np.zeros((self.N, 2))
        AP = np.zeros((self.N, 2))
        E = lib().ref_voronoi_forces(self.h, F, AP)
        return F, AP, E

    def set_exclusions(self, exes):
        lib().ref_voronoi_set_exclusions(self.h, np.ascontiguousarray(exes, np.int32))

    def external_forces(self):
        out = np.zeros((self.N, 2))
        lib().ref_voronoi_external_forces(self.h, out)
        return out

    def observables(self, initial, cutoff=0.5):
        """reportq, reportVarq, reportVarAP (A, P) and dynamicalFeatures' MSD and overlap against
        `initial`, on the current state."""
        out = np.zeros(6)
        lib().ref_voronoi_observables(self.h, np.ascontiguousarray(initial, np.float64), cutoff, out)
        return dict(zip(("mean_q", "var_q", "var_A", "var_P", "msd", "overlap"), out))

    def state(self, K=16):
        pos = np.zeros((self.N, 2))
        th = np.zeros(self.N)
        nn = np.zeros(self.N, np.int32)
        nbr = np.zeros((self.N, K), np.int32)
        st = lib().ref_voronoi_get(self.h, pos, th.ctypes.data_as(C.c_void_p), K, nn, nbr)
        if st:
            raise RuntimeError("row longer than K")
        return pos, th, nn, nbr

    def spp_run(self, steps, dt=0.01, local_repair=True):
        lib().ref_voronoi_spp_run(self.h, steps, dt, 1 if local_repair else 0)

    def fire(self, dt=0.01, alpha_start=0.99, dt_max=0.1, dt_inc=1.05, dt_dec=0.95, alpha_dec=0.9, n_min=5,
             force_cutoff=1e-7, max_iterations=1000):
        lib().ref_fire(self.h, 0, dt, alpha_start, dt_max, dt_inc, dt_dec, alpha_dec, n_min, force_cutoff,
                       max_iterations)


class RefVertex:
    """VertexQuadraticEnergy of the reference, CPU branch, initialised from the Delaunay dual."""

    def __init__(self, Nc, A0=1.0, P0=3.8):
        self.h = lib().ref_vertex_new(Nc, A0, P0)
        nc, nv, vm = C.c_int(), C.c_int(), C.c_int()
        lib().ref_vertex_counts(self.h, C.byref(nc), C.byref(nv), C.byref(vm))
        self.Nc, self.Nv, self.vmax = nc.value, nv.value, vm.value

    def __del__(self):
        try:
            lib().ref_free(self.h)
        except Exception:
            pass

    def state(self):
        cp = np.zeros((self.Nc, 2))
        vp = np.zeros((self.Nv, 2))
        vn = np.zeros(3 * self.Nv, np.int32)
        vcn = np.zeros(3 * self.Nv, np.int32)
        cvn = np.zeros(self.Nc, np.int32)
        cv = np.zeros((self.Nc, self.vmax), np.int32)
        lib().ref_vertex_get(self.h, cp.ctypes.data_as(C.c_void_p), vp, vn, vcn, cvn, cv)
        return cp, vp, vn, vcn, cvn, cv

    def set_positions(self, vpos):
        lib().ref_vertex_set_positions(self.h, np.ascontiguousarray(vpos, np.float64))

    def set_preferences(self, pref):
        lib().ref_vertex_set_preferences(self.h, np.ascontiguousarray(pref, np.float64))

    def set_t1(self, t):
        lib().ref_vertex_set_t1(self.h, t)

    def forces(self):
        F = np.zeros((self.Nv, 2))
        AP = np.zeros((self.Nc, 2))
        E = lib().ref_vertex_forces(self.h, F, AP)
        return F, AP, E

    def brownian_run(self, steps, dt=0.005, T=1e-3, mu=1.0):
        lib().ref_vertex_brownian_run(self.h, steps, dt, T, mu)

    def set_tension(self, types, gamma=0.0, gammas=None):
        """VertexQuadraticEnergyWithTension: cell types, one gamma or an ntypes x ntypes matrix."""
        g = None if gammas is None else np.ascontiguousarray(gammas, np.float64)
        nt = 0 if g is None else int(round(np.sqrt(g.size)))
        lib().ref_vertex_set_tension(self.h, np.ascontiguousarray(types, np.int32), float(gamma), nt,
                                     None if g is None else g.ctypes.data_as(C.c_void_p))

    def fire(self, dt=0.01, alpha_start=0.99, dt_max=0.1, dt_inc=1.05, dt_dec=0.95, alpha_dec=0.9, n_min=5,
             force_cutoff=1e-7, max_iterations=1000):
        lib().ref_fire(self.h, 1, dt, alpha_start, dt_max, dt_inc, dt_dec, alpha_dec, n_min, force_cutoff,
                       max_iterations)


def relaxed_c2_state(n_tile=16384, reps=4, relax_steps=120, v0=0.1, seed=1):
    """Steady-state sample of the large monolayer made by the reference itself: a tile of n_tile
    cells (side L/reps) from seeded uniform positions, relaxed with the reference CPU SPP path, then
    tiled reps x reps (periodic images agree, so the tiling is a valid periodic state of N = n_tile
    reps^2 cells in a box reps times larger). The reference's per-step cost on a relaxed state is
    ~1.75x lower than on the first steps from uniform positions, so this is the fair sample."""
    Lt = float(np.sqrt(n_tile))
    rng = np.random.default_rng(seed)
    with quiet():
        r = RefVoronoi(n_tile)
        r.set_state(rng.random((n_tile, 2)) * Lt, rng.uniform(0, 2 * np.pi, n_tile))
        r.set_motility(v0, 1.0)
        r.spp_run(relax_steps, 0.01, True)
    pos, th, _, _ = r.state()
    del r
    shifts = np.array([(i * Lt, j * Lt) for j in range(reps) for i in range(reps)])
    full = (pos[None, :, :] + shifts[:, None, :]).reshape(-1, 2)
    return full, np.tile(th, reps * reps), Lt * reps


def bench_c2(steps, n_cells=262144, box=512.0, v0=0.1, seed=1, barrier=None, local_repair=True, state=None):
    """The reference's CPU SPP path on the large monolayer in a relaxed state (relaxed_c2_state);
    returns the cpu_baseline record. local_repair: the test-and-repair mode that voronoi.cpp:106-107
    switches to (setCPU(false)); otherwise the reference's default CPU mode, a global
    retriangulation every step (src/models/voronoiModelBase.cpp:556-564). With a barrier
    (multi-process runs) every worker starts its timed steps together."""
    reps = 4
    if state is None:
        state = relaxed_c2_state(n_tile=n_cells // (reps * reps), reps=reps, v0=v0, seed=seed)
    pos, th, L = state
    assert abs(L - box) < 1e-9 and len(pos) == n_cells
    with quiet():
        r = RefVoronoi(n_cells)
        r.set_state(pos, th)
        r.set_motility(v0, 1.0)
        r.spp_run(1, 0.01, local_repair)  # first step builds the updater
    if barrier is not None:
        barrier.wait()
    with quiet():
        t0 = time.perf_counter()
        r.spp_run(steps, 0.01, local_repair)
        t1 = time.perf_counter()
    t = t1 - t0
    mode = "local test-and-repair" if local_repair else "global retriangulation every step (default CPU mode)"
    return {"value": n_cells * steps / t, "unit": "cell-steps/s", "cores": 1, "kind": "reference",
            "sample": f"{steps} SPP steps of the N={n_cells} monolayer, reference CPU path ({mode}), "
                      f"relaxed state (N/16 tile relaxed 120 steps by the reference, tiled 4x4), 1 thread",
            "mode": "local" if local_repair else "global",
            "t0": t0, "t1": t1, "cell_steps": n_cells * steps}


def bench_c1(steps=1000, n_cells=300, v0=0.05, seed=1, local_repair=True):
    """The reference's own small case: N = 300 cells in a box of side sqrt(N) from seeded uniform
    positions, A0 = 1, p0 = 3.8, SPP v0 = 0.05, Dr = 1, dt = 0.01, `steps` steps, reference CPU path,
    one thread (local test-and-repair, or the default global retriangulation every step)."""
    L = float(np.sqrt(n_cells))
    rng = np.random.default_rng(seed)
    with quiet():
        r = RefVoronoi(n_cells)
        r.set_state(rng.random((n_cells, 2)) * L, rng.uniform(0, 2 * np.pi, n_cells))
        r.set_motility(v0, 1.0)
        r.spp_run(1, 0.01, local_repair)
        t0 = time.perf_counter()
        r.spp_run(steps, 0.01, local_repair)
        t1 = time.perf_counter()
    return {"value": n_cells * steps / (t1 - t0), "unit": "cell-steps/s", "cores": 1, "kind": "reference",
            "ms_per_step": 1e3 * (t1 - t0) / steps, "mode": "local" if local_repair else "global",
            "sample": f"{steps} SPP steps of N={n_cells} (box sqrt(N), v0 {v0}), reference CPU path, 1 thread"}


_BARRIER = None


def _init_worker(b):
    global _BARRIER
    _BARRIER = b


def _c2_worker_b(args):
    steps, seed = args
    return bench_c2(steps, seed=seed, barrier=_BARRIER)


def bench_c2_all_cores(steps, max_procs=256, gb_per_proc=1.0):
    """One independent reference instance per host core (the reference is single-threaded), as many
    as memory allows; all start their timed steps together. Aggregate = all cell-steps / the span
    from the first start to the last finish."""
    import multiprocessing as mp
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available / 2**30
    except Exception:
        avail = 8.0
    procs = int(max(1, min(cores, max_procs, avail * 0.7 // gb_per_proc)))
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(procs)
    with ctx.Pool(procs, initializer=_init_worker, initargs=(barrier,)) as pool:
        res = pool.map(_c2_worker_b, [(steps, 1 + i) for i in range(procs)])
    span = max(r["t1"] for r in res) - min(r["t0"] for r in res)
    cell_steps = sum(r["cell_steps"] for r in res)
    return {"value": cell_steps / span, "unit": "cell-steps/s", "cores": procs, "kind": "reference",
            "sample": f"{procs} independent instances (one per core; {cores} cores available), each {steps} "
                      f"SPP steps of the N=262144 monolayer in a relaxed state, reference CPU path, "
                      f"1 thread per instance",
            "per_instance": [r["value"] for r in res]}
