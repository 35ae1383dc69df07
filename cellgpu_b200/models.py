"""Host-side mirror of the reference's class API (abaso/cellGPU ``inc/Simulation.h``,
``inc/models/voronoiQuadraticEnergy.h``, ``inc/updaters/selfPropelledParticleDynamics.h`` ...) over the
C ABI. Every compute call goes to the sm_100a library; there is no CPU branch.

Names follow the reference so code written against it reads the same:

    model = VoronoiQuadraticEnergy(300, 1.0, 3.8, reprod=True)   # Voronoi2D is an alias
    spp = selfPropelledParticleDynamics(300)
    sim = Simulation(); sim.setConfiguration(model); sim.addUpdater(spp, model)
    sim.setIntegrationTimestep(0.01)
    for t in range(1000): sim.performTimestep()
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import CG_FP64, CG_MIXED, FireParams, check, device_noise, load, ptr


def _f64(a, shape):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(shape))


class VoronoiBatch:
    """A device-resident batch of independent Voronoi monolayers (one launch per step for all).

    ``N`` is a list of cell counts, ``boxes`` a list of (Lx, Ly). A batch of one is the plain
    drop-in of the reference's single-monolayer path.
    """

    def __init__(self, N, boxes, K=16, precision=CG_FP64):
        self._lib = load()
        self.N = [int(n) for n in N]
        self.boxes = np.asarray(boxes, dtype=np.float64).reshape(len(self.N), 2)
        self.K = int(K)
        self.precision = precision
        h = C.c_void_p()
        n_arr = np.asarray(self.N, dtype=np.int32)
        check(self._lib.cg_voronoi_create(len(self.N), ptr(n_arr), ptr(np.ascontiguousarray(self.boxes)),
                                          self.K, precision, C.byref(h)))
        self._h = h
        self.Ntot = sum(self.N)
        self.offsets = np.concatenate([[0], np.cumsum(self.N)]).astype(np.int64)

    # -- lifetime
    def close(self):
        if getattr(self, "_h", None):
            self._lib.cg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    # -- line tension (VoronoiQuadraticEnergyWithTension)
    def set_cell_types(self, types):
        t = np.ascontiguousarray(types, dtype=np.int32).reshape(self.Ntot)
        check(self._lib.cg_set_cell_types(self._h, ptr(t)))

    def set_tension(self, gamma):
        """gamma per unit length on every edge between cells of different types (0: off)."""
        check(self._lib.cg_set_tension(self._h, float(gamma)))

    def set_exclusions(self, excluded):
        """Particle exclusions (voronoiModelBase::setExclusions): cells with excluded[c] != 0 get
        zero motility and, after every force evaluation, F = 0 with the computed force kept as the
        external force -F. None clears the flags."""
        if excluded is None:
            check(self._lib.cg_set_exclusions(self._h, None))
            return
        e = np.ascontiguousarray(excluded, np.int32).reshape(-1)
        if e.size != self.Ntot:
            raise ValueError("one flag per cell")
        check(self._lib.cg_set_exclusions(self._h, ptr(e)))

    def external_forces(self):
        out = np.zeros((self.Ntot, 2))
        check(self._lib.cg_get_external_forces(self._h, ptr(out)))
        return out

    def set_tension_matrix(self, gamma):
        """symmetric ntypes x ntypes matrix of edge tensions between types (empty: off)."""
        g = np.ascontiguousarray(gamma, dtype=np.float64)
        n = 0 if g.size == 0 else int(round(np.sqrt(g.size)))
        check(self._lib.cg_set_tension_matrix(self._h, n, ptr(g.reshape(-1)) if n else None))

    # -- autotuning of launch parameters
    def autotune(self):
        """Time the force pass's block shapes and the cell-list bin sides on the current state and
        keep the fastest; returns the timings (ms) and the choices."""
        t = np.zeros(6)
        c = np.zeros(2, np.int32)
        check(self._lib.cg_autotune(self._h, ptr(t), ptr(c)))
        return {"force_pass_ms": t[:3].tolist(), "triangulation_ms": t[3:].tolist(),
                "force_shape": ["2 warps/block", "4 warps/block", "thread per cell"][int(c[0])],
                "bin_side": [0.8, 1.0, 1.25][int(c[1])]}

    def autotune_repair(self, steps=10, dt=0.01, mu=1.0):
        """Time the repair round's launch grids on real SPP steps (device noise) and keep the
        fastest. The system advances by 12 * steps steps. Returns ms per step for each (star grid,
        commit grid) pair and the chosen grids."""
        t = np.zeros(6)
        c = np.zeros(2, np.int32)
        check(self._lib.cg_autotune_repair(self._h, int(steps), float(dt), float(mu), ptr(t), ptr(c)))
        return {"ms_per_step": t.tolist(), "star_grid": int(c[0]), "commit_grid": int(c[1])}

    # -- spatial re-sorting
    def spatial_sort(self):
        """Reorder every instance's cells along a Hilbert curve (arrays and topology move with them)."""
        check(self._lib.cg_spatial_sort(self._h))

    def tags(self):
        """For every current index, the index the cell had when the batch was created."""
        out = np.zeros(self.Ntot, np.int32)
        check(self._lib.cg_get_tags(self._h, ptr(out)))
        return out

    # -- observables (per instance, on the device)
    OBS_FIELDS = ("mean_q", "var_q", "mean_A", "mean_P", "var_A", "var_P", "msd", "overlap")

    def set_reference_positions(self):
        """Capture the current positions as the reference of msd / overlap."""
        check(self._lib.cg_set_reference_positions(self._h))

    def observables(self, cutoff=0.5):
        """Per instance: mean and variance of q = P/sqrt(A), mean and variance of A and P (stored
        areas/perimeters of the last force evaluation), MSD and overlap fraction against the
        reference positions. Returns a dict of arrays."""
        out = np.zeros((len(self.N), len(self.OBS_FIELDS)))
        check(self._lib.cg_observables(self._h, float(cutoff), ptr(out)))
        return {k: out[:, i] for i, k in enumerate(self.OBS_FIELDS)}

    # -- snapshots (exact resume: device noise is keyed per instance and counted by step)
    def snapshot(self) -> bytes:
        """The whole state of the batch as bytes; ``restore(bytes)`` continues it exactly."""
        n = self._lib.cg_snapshot_size(self._h)
        buf = C.create_string_buffer(n)
        check(self._lib.cg_snapshot(self._h, buf, n))
        return buf.raw

    # -- state
    def set_positions(self, pos):
        pos = _f64(pos, (self.Ntot, 2))
        check(self._lib.cg_set_positions(self._h, ptr(pos)))

    def positions(self):
        out = np.zeros((self.Ntot, 2))
        check(self._lib.cg_get_positions(self._h, ptr(out)))
        return out

    def set_preferences(self, APpref):
        a = _f64(APpref, (self.Ntot, 2))
        check(self._lib.cg_set_cell_preferences(self._h, ptr(a)))

    def set_moduli(self, KA, KP):
        check(self._lib.cg_set_moduli(self._h, float(KA), float(KP)))

    def set_motility(self, motility):
        m = _f64(motility, (self.Ntot, 2))
        check(self._lib.cg_set_motility(self._h, ptr(m)))

    def set_directors(self, theta):
        t = _f64(theta, (self.Ntot,))
        check(self._lib.cg_set_directors(self._h, ptr(t)))

    def directors(self):
        out = np.zeros(self.Ntot)
        check(self._lib.cg_get_directors(self._h, ptr(out)))
        return out

    def set_seed(self, seed):
        check(self._lib.cg_set_seed(self._h, int(seed) & (2**64 - 1)))

    def set_deterministic(self, on=True):
        """Order-independent (fixed-point) force sums: the same inputs then give bit-identical
        forces and trajectories on every run (cg_set_deterministic)."""
        check(self._lib.cg_set_deterministic(self._h, 1 if on else 0))

    @property
    def deterministic(self):
        return bool(self._lib.cg_get_deterministic(self._h))

    def set_instance_seeds(self, seeds):
        """Philox key of each instance's device noise (its noise is then independent of where the
        instance sits in a batch)."""
        arr = np.ascontiguousarray([int(x) & (2**64 - 1) for x in seeds], dtype=np.uint64)
        if len(arr) != len(self.N):
            raise ValueError("one seed per instance")
        check(self._lib.cg_set_instance_seeds(self._h, arr.ctypes.data))

    def forces(self):
        out = np.zeros((self.Ntot, 2))
        check(self._lib.cg_get_forces(self._h, ptr(out)))
        return out

    def area_perimeter(self):
        out = np.zeros((self.Ntot, 2))
        check(self._lib.cg_get_area_perimeter(self._h, ptr(out)))
        return out

    def topology(self):
        """(nn, nbr): row lengths and rows of K entries. K is the system's current row capacity,
        which grows from 16 to 32 when a cell gets more than 16 neighbours."""
        self.K = int(self._lib.cg_neighbor_capacity(self._h))
        nn = np.zeros(self.Ntot, np.int32)
        nbr = np.zeros((self.Ntot, self.K), np.int32)
        check(self._lib.cg_get_topology(self._h, ptr(nn), ptr(nbr)))
        return nn, nbr

    def set_topology(self, nn, nbr):
        self.K = int(self._lib.cg_neighbor_capacity(self._h))
        nn = np.ascontiguousarray(nn, np.int32)
        nbr = np.asarray(nbr, np.int32).reshape(self.Ntot, -1)
        if nbr.shape[1] > self.K:
            raise ValueError(f"rows of {nbr.shape[1]} entries exceed the capacity {self.K}")
        rows = np.full((self.Ntot, self.K), -1, np.int32)
        rows[:, :nbr.shape[1]] = nbr
        check(self._lib.cg_set_topology(self._h, ptr(nn), ptr(rows)))

    def energies(self):
        out = np.zeros(len(self.N))
        check(self._lib.cg_get_energies(self._h, ptr(out)))
        return out

    def counters(self):
        out = (C.c_longlong * 8)()
        check(self._lib.cg_counters(self._h, out, 8))
        keys = ["tests_failed", "cells_restarred", "rows_changed", "repair_rounds", "global_rebuilds",
                "t1_flips", "fire_iterations", "round_epilogues"]
        return dict(zip(keys, list(out)))

    # -- compute
    def triangulate(self):
        check(self._lib.cg_triangulate(self._h))

    def compute_forces(self):
        check(self._lib.cg_compute_forces(self._h))

    def enforce_topology(self):
        check(self._lib.cg_enforce_topology(self._h))

    def spp_run(self, n_steps, dt=0.01, mu=1.0, noise=None):
        """n_steps SPP steps; noise: optional device tensor (torch, float64) of n_steps*N normals,
        step-major (row t holds step t's normals of every cell)."""
        noise = device_noise(noise, int(n_steps) * self.Ntot)
        check(self._lib.cg_spp_run(self._h, int(n_steps), float(dt), float(mu), ptr(noise)))

    def synchronize(self):
        check(self._lib.cg_synchronize(self._h))

    def device_bytes(self):
        return int(self._lib.cg_device_bytes(self._h))

    # -- FIRE
    def fire_minimize(self, params=None, **kw):
        p = params if params is not None else FireParams.defaults(**kw)
        check(self._lib.cg_fire_minimize(self._h, C.byref(p)))

    def fire_begin(self, params=None, **kw):
        """Start a FIRE minimisation that fire_advance continues in pieces."""
        p = params if params is not None else FireParams.defaults(**kw)
        check(self._lib.cg_fire_begin(self._h, C.byref(p)))
        return p

    def fire_advance(self, params, iterations):
        """Up to `iterations` more FIRE iterations (fewer if every instance stops); returns the
        number of stopped instances."""
        n = C.c_int(0)
        check(self._lib.cg_fire_advance(self._h, C.byref(params), int(iterations), C.byref(n)))
        return n.value

    def fire_state(self):
        n = len(self.N)
        it = np.zeros(n, np.int32)
        fm = np.zeros(n)
        fn = np.zeros(n)
        check(self._lib.cg_fire_state(self._h, ptr(it), ptr(fm), ptr(fn)))
        return it, fm, fn


class VertexBatch(VoronoiBatch):
    """A device-resident batch of vertex-model monolayers: Nc[i] cells, 2 Nc[i] vertices each."""

    def __init__(self, Nc, boxes, vmax=30, precision=CG_FP64):
        self._lib = load()
        self.N = [int(n) for n in Nc]
        self.boxes = np.asarray(boxes, dtype=np.float64).reshape(len(self.N), 2)
        self.K = self.vmax = int(vmax)
        self.precision = precision
        h = C.c_void_p()
        n_arr = np.asarray(self.N, dtype=np.int32)
        check(self._lib.cg_vertex_create(len(self.N), ptr(n_arr), ptr(np.ascontiguousarray(self.boxes)),
                                         self.vmax, precision, C.byref(h)))
        self._h = h
        self.Ntot = sum(self.N)
        self.Nv = 2 * self.Ntot
        self.offsets = np.concatenate([[0], np.cumsum(self.N)]).astype(np.int64)

    def from_cells(self, cell_pos):
        p = _f64(cell_pos, (self.Ntot, 2))
        check(self._lib.cg_vertex_from_voronoi(self._h, ptr(p)))

    def set_positions(self, vpos):
        p = _f64(vpos, (self.Nv, 2))
        check(self._lib.cg_set_positions(self._h, ptr(p)))

    def positions(self):
        out = np.zeros((self.Nv, 2))
        check(self._lib.cg_get_positions(self._h, ptr(out)))
        return out

    def forces(self):
        out = np.zeros((self.Nv, 2))
        check(self._lib.cg_get_forces(self._h, ptr(out)))
        return out

    def row_capacity(self):
        """Current cell-row width (vmax): it grows when a T1 transition needs longer rows."""
        self.K = self.vmax = int(self._lib.cg_neighbor_capacity(self._h))
        return self.vmax

    def vertex_topology(self):
        vn = np.zeros(3 * self.Nv, np.int32)
        vcn = np.zeros(3 * self.Nv, np.int32)
        cvn = np.zeros(self.Ntot, np.int32)
        cv = np.zeros((self.Ntot, self.row_capacity()), np.int32)
        check(self._lib.cg_get_vertex_topology(self._h, ptr(vn), ptr(vcn), ptr(cvn), ptr(cv)))
        return vn, vcn, cvn, cv

    def set_vertex_topology(self, vn, vcn, cvn, cv):
        vn = np.ascontiguousarray(vn, np.int32)
        vcn = np.ascontiguousarray(vcn, np.int32)
        cvn = np.ascontiguousarray(cvn, np.int32)
        cv = np.ascontiguousarray(cv, np.int32).reshape(self.Ntot, -1)
        if cv.shape[1] != self.row_capacity():
            w = np.full((self.Ntot, self.vmax), -1, np.int32)
            k = min(self.vmax, cv.shape[1])
            w[:, :k] = cv[:, :k]
            cv = w
        check(self._lib.cg_set_vertex_topology(self._h, ptr(vn), ptr(vcn), ptr(cvn), ptr(cv)))

    def set_t1_threshold(self, t):
        check(self._lib.cg_set_t1_threshold(self._h, float(t)))

    def brownian_run(self, n_steps, dt=0.005, mu=1.0, T=1e-3, noise=None):
        """noise: optional device tensor (torch, float64) with n_steps*2*Nv normals (x then y per
        vertex), step-major."""
        noise = device_noise(noise, int(n_steps) * 2 * self.Nv)
        check(self._lib.cg_brownian_run(self._h, int(n_steps), float(dt), float(mu), float(T), ptr(noise)))

    def spp_run(self, n_steps, dt=0.01, mu=1.0, noise=None):
        """n_steps SPP steps of the cell-vertex model; noise: optional device tensor (torch,
        float64) of n_steps*Nc director normals, step-major."""
        noise = device_noise(noise, int(n_steps) * self.Ntot)
        check(self._lib.cg_vertex_spp_run(self._h, int(n_steps), float(dt), float(mu), ptr(noise)))


def restore(snapshot: bytes):
    """A new VoronoiBatch or VertexBatch holding the state saved by ``snapshot()``."""
    lib = load()
    buf = C.create_string_buffer(bytes(snapshot), len(snapshot))
    h = C.c_void_p()
    check(lib.cg_restore(buf, len(snapshot), C.byref(h)))
    n_inst = lib.cg_num_instances(h)
    Ns = np.zeros(n_inst, np.int32)
    boxes = np.zeros((n_inst, 2))
    check(lib.cg_get_instances(h, ptr(Ns), ptr(boxes)))
    vertex = lib.cg_model_kind(h) == 1
    b = (VertexBatch if vertex else VoronoiBatch).__new__(VertexBatch if vertex else VoronoiBatch)
    b._lib = lib
    b._h = h
    b.N = [int(n) for n in Ns]
    b.boxes = boxes
    b.K = lib.cg_neighbor_capacity(h)
    b.precision = lib.cg_precision(h)
    b.Ntot = sum(b.N)
    b.offsets = np.concatenate([[0], np.cumsum(b.N)]).astype(np.int64)
    if vertex:
        b.vmax = b.K
        b.Nv = 2 * b.Ntot
    return b


def random_positions(N, box, seed):
    """Seeded uniform positions in [0,Lx)x[0,Ly), x then y per cell like
    Simple2DCell::setCellPositionsRandomly (src/models/Simple2DCell.cpp:85-100), from numpy's PCG64."""
    rng = np.random.default_rng(seed)
    u = rng.random((N, 2))
    return u * np.asarray(box, dtype=np.float64).reshape(1, 2)


class VoronoiQuadraticEnergy:
    """Voronoi (SPV) model with E = sum KA (A-A0)^2 + KP (P-P0)^2
    (inc/models/voronoiQuadraticEnergy.h; src/models/voronoiQuadraticEnergy.cpp:28-35)."""

    def __init__(self, n, A0=1.0, P0=3.8, reprod=False, seed=None, K=16, precision=CG_FP64, box=None):
        L = float(np.sqrt(n))
        self.box = (L, L) if box is None else tuple(box)
        self.Ncells = int(n)
        self.reproducible = reprod
        if seed is None:
            seed = 13377 if reprod else int(np.random.SeedSequence().entropy % (2**31))
        self.seed = seed
        self.batch = VoronoiBatch([n], [self.box], K=K, precision=precision)
        self.batch.set_seed(seed)
        self.batch.set_positions(random_positions(n, self.box, seed))
        rng = np.random.default_rng(seed + 1)
        self.batch.set_directors(rng.uniform(0, 2 * np.pi, n))  # Simple2DActiveCell.cpp:55-70
        self.setCellPreferencesUniform(A0, P0)
        self.setv0Dr(0.05, 1.0)
        self.KA, self.KP = 1.0, 1.0
        self.batch.triangulate()
        self.forcesUpToDate = False

    # reference API
    def getNumberOfDegreesOfFreedom(self):
        return self.Ncells

    def setCellPreferencesUniform(self, A0, P0):
        self.batch.set_preferences(np.tile([A0, P0], (self.Ncells, 1)))
        self.forcesUpToDate = False

    def setCellPreferences(self, APpref):
        self.batch.set_preferences(APpref)
        self.forcesUpToDate = False

    def setModuliUniform(self, KA, KP):
        self.KA, self.KP = KA, KP
        self.batch.set_moduli(KA, KP)
        self.forcesUpToDate = False

    def setv0Dr(self, v0, Dr):
        self.batch.set_motility(np.tile([v0, Dr], (self.Ncells, 1)))

    def setCellMotility(self, v0s, Drs):
        self.batch.set_motility(np.stack([v0s, Drs], axis=1))

    def setCellPositions(self, pos):
        self.batch.set_positions(pos)
        self.batch.triangulate()
        self.forcesUpToDate = False

    def returnPositions(self):
        return self.batch.positions()

    getCellPositions = returnPositions

    def computeForces(self):
        if self.forcesUpToDate:
            return
        self.batch.compute_forces()
        self.forcesUpToDate = True

    def returnForces(self):
        return self.batch.forces()

    getForces = returnForces

    def returnAreaPeri(self):
        return self.batch.area_perimeter()

    def computeEnergy(self):
        self.computeForces()
        return float(self.batch.energies()[0])

    def enforceTopology(self):
        self.batch.enforce_topology()

    def globalTriangulation(self):
        self.batch.triangulate()

    def neighbors(self):
        return self.batch.topology()

    def setExclusions(self, exes):
        """voronoiModelBase::setExclusions (src/models/voronoiModelBase.cpp:85-104): cells with
        exes[i] != 0 stop self-propelling (v0 = Dr = 0); their force is zeroed after every force
        evaluation and kept as the external force (returnExternalForces)."""
        self.batch.set_exclusions(exes)
        self.forcesUpToDate = False

    def returnExternalForces(self):
        return self.batch.external_forces()


Voronoi2D = VoronoiQuadraticEnergy


class _SurfaceTension:
    """setCellType / setSurfaceTension / setUseSurfaceTension of the reference's
    *QuadraticEnergyWithTension classes: one gamma for every unlike pair, or a symmetric matrix of
    tensions between types (setSurfaceTension with a flattened list), applied while
    setUseSurfaceTension(True)."""

    def _init_tension(self):
        self.gamma = 0.0
        self.Tension = False
        self.simpleTension = True
        self.tensionMatrix = None
        self.batch.set_cell_types(np.zeros(self.Ncells, np.int32))

    def _apply(self):
        if not self.Tension:
            self.batch.set_tension(0.0)
        elif self.simpleTension:
            self.batch.set_tension(self.gamma)
        else:
            self.batch.set_tension_matrix(self.tensionMatrix)
        self.forcesUpToDate = False

    def setCellType(self, types):
        self.batch.set_cell_types(types)
        self.forcesUpToDate = False

    def setUseSurfaceTension(self, use_tension):
        self.Tension = bool(use_tension)
        self._apply()

    def setSurfaceTension(self, g):
        if np.ndim(g) == 0:
            self.gamma, self.simpleTension = float(g), True
        else:
            flat = np.asarray(g, np.float64).reshape(-1)
            n = int(round(np.sqrt(flat.size)))
            if n * n != flat.size:
                raise ValueError("the tension matrix must be square")
            self.tensionMatrix, self.simpleTension = flat.reshape(n, n), False
        self._apply()

    def getSurfaceTension(self):
        return self.gamma


class VoronoiQuadraticEnergyWithTension(_SurfaceTension, VoronoiQuadraticEnergy):
    """Voronoi model with line tension between cells of different types
    (inc/models/voronoiQuadraticEnergyWithTension.h)."""

    def __init__(self, n, A0=1.0, P0=3.8, reprod=False, **kw):
        VoronoiQuadraticEnergy.__init__(self, n, A0, P0, reprod, **kw)
        self._init_tension()


class selfPropelledParticleDynamics:
    """SPP equations of motion (src/updaters/selfPropelledParticleDynamics.cpp:45-101)."""

    def __init__(self, n=None):
        self.deltaT = 0.01
        self.mu = 1.0
        self.model = None
        self.noise = None

    def setDeltaT(self, dt):
        self.deltaT = dt

    def setMu(self, mu):
        self.mu = mu

    def set2DModel(self, model):
        self.model = model

    def integrateEquationsOfMotion(self, n_steps=1):
        self.model.batch.spp_run(n_steps, self.deltaT, self.mu, self.noise)
        self.model.forcesUpToDate = False


class VertexQuadraticEnergy:
    """Vertex (AVM) model (inc/models/vertexQuadraticEnergy.h; src/models/vertexQuadraticEnergy.cpp:18-24):
    cells from seeded random points, vertices from their Delaunay dual."""

    def __init__(self, n, A0=1.0, P0=3.8, reprod=False, seed=None, vmax=30, box=None):
        L = float(np.sqrt(n))
        self.box = (L, L) if box is None else tuple(box)
        self.Ncells = int(n)
        if seed is None:
            seed = 13377 if reprod else int(np.random.SeedSequence().entropy % (2**31))
        self.seed = seed
        self.batch = VertexBatch([n], [self.box], vmax=vmax)
        self.batch.set_seed(seed)
        self.batch.from_cells(random_positions(n, self.box, seed))
        rng = np.random.default_rng(seed + 1)
        self.batch.set_directors(rng.uniform(0, 2 * np.pi, n))
        self.setCellPreferencesUniform(A0, P0)
        self.setT1Threshold(0.01)

    def getNumberOfDegreesOfFreedom(self):
        return self.batch.Nv

    def setCellPreferencesUniform(self, A0, P0):
        self.batch.set_preferences(np.tile([A0, P0], (self.Ncells, 1)))

    def setCellPreferences(self, APpref):
        self.batch.set_preferences(APpref)

    def setModuliUniform(self, KA, KP):
        self.batch.set_moduli(KA, KP)

    def setT1Threshold(self, t):
        self.batch.set_t1_threshold(t)

    def setv0Dr(self, v0, Dr):
        self.batch.set_motility(np.tile([v0, Dr], (self.Ncells, 1)))

    def computeForces(self):
        self.batch.compute_forces()

    def returnForces(self):
        return self.batch.forces()

    def returnPositions(self):
        return self.batch.positions()

    def computeEnergy(self):
        self.batch.compute_forces()
        return float(self.batch.energies()[0])

    def enforceTopology(self):
        self.batch.enforce_topology()


class VertexQuadraticEnergyWithTension(_SurfaceTension, VertexQuadraticEnergy):
    """Vertex model with line tension on edges between cells of different types
    (inc/models/vertexQuadraticEnergyWithTension.h). computeEnergy includes the tension (gamma l
    over every unlike edge once), which the reference leaves unimplemented."""

    def __init__(self, n, A0=1.0, P0=3.8, reprod=False, **kw):
        VertexQuadraticEnergy.__init__(self, n, A0, P0, reprod, **kw)
        self._init_tension()


class brownianParticleDynamics:
    """Brownian dynamics (src/updaters/brownianParticleDynamics.cpp:46-109), vertex model."""

    def __init__(self, n=None):
        self.deltaT, self.mu, self.T = 0.01, 1.0, 0.0
        self.model = None

    def setDeltaT(self, dt):
        self.deltaT = dt

    def setMu(self, mu):
        self.mu = mu

    def setT(self, T):
        self.T = T

    def set2DModel(self, model):
        self.model = model

    def integrateEquationsOfMotion(self, n_steps=1):
        self.model.batch.brownian_run(n_steps, self.deltaT, self.mu, self.T)


class selfPropelledCellVertexDynamics(selfPropelledParticleDynamics):
    """SPP of the vertex model (src/updaters/selfPropelledCellVertexDynamics.cpp:28-122)."""


class EnergyMinimizerFIRE:
    """FIRE minimiser (src/updaters/EnergyMinimizerFIRE2D.cpp), CPU conventions, on the GPU."""

    def __init__(self, model=None):
        self.model = model
        self.params = FireParams.defaults()

    def set2DModel(self, model):
        self.model = model

    def setMaximumIterations(self, n):
        self.params.max_iterations = int(n)

    def setForceCutoff(self, fc):
        self.params.force_cutoff = fc

    def setDeltaT(self, dt):
        self.params.dt = dt
        self.params.dt_min = 0.01 * dt

    def setAlphaStart(self, a):
        self.params.alpha_start = a

    def setDeltaTMax(self, t):
        self.params.dt_max = t

    def setDeltaTInc(self, t):
        self.params.dt_inc = t

    def setDeltaTDec(self, t):
        self.params.dt_dec = t

    def setAlphaDec(self, a):
        self.params.alpha_dec = a

    def setNMin(self, n):
        self.params.n_min = int(n)

    def minimize(self):
        self.model.batch.fire_minimize(self.params)

    def integrateEquationsOfMotion(self, n_steps=1):
        self.minimize()


class Simulation:
    """Owns a configuration and its updaters (inc/Simulation.h:18-87; performTimestep,
    src/Simulation.cpp:141-166). GPU only: setCPUOperation(True) is rejected."""

    def __init__(self):
        self.configuration = None
        self.updaters = []
        self.integrationTimestep = 0.01
        self.Time = 0.0
        self.integerTimestep = 0

    def setConfiguration(self, model):
        self.configuration = model

    def addUpdater(self, updater, model=None):
        updater.set2DModel(model if model is not None else self.configuration)
        self.updaters.append(updater)

    def setIntegrationTimestep(self, dt):
        self.integrationTimestep = dt
        for u in self.updaters:
            if hasattr(u, "setDeltaT"):
                u.setDeltaT(dt)

    def setCPUOperation(self, flag):
        if flag:
            raise NotImplementedError("cellgpu_b200 runs on the GPU only")

    def setReproducible(self, flag):
        """Reproducible runs (Simulation::setReproducible): besides fixed seeds, the forces are
        summed in an order-independent way, so reruns give bit-identical trajectories."""
        if self.configuration is not None:
            self.configuration.reproducible = bool(flag)
            self.configuration.batch.set_deterministic(bool(flag))

    def setSortPeriod(self, sp):
        """Spatially re-sort the (Voronoi) configuration every sp steps (src/Simulation.cpp:154-164);
        sp <= 0 never sorts, as the reference's default."""
        self.sortPeriod = int(sp)

    def performTimestep(self):
        self.performTimesteps(1)

    def performTimesteps(self, n):
        """n steps of every updater back to back on the device, with a spatial re-sort whenever
        the step counter reaches a multiple of the sort period."""
        sp = getattr(self, "sortPeriod", -1)
        while n > 0:
            chunk = n
            if sp > 0:
                chunk = min(n, sp - self.integerTimestep % sp)
            for u in self.updaters:
                u.integrateEquationsOfMotion(chunk)
            self.integerTimestep += chunk
            self.Time += chunk * self.integrationTimestep
            n -= chunk
            if sp > 0 and self.integerTimestep % sp == 0 and isinstance(self.configuration, VoronoiQuadraticEnergy):
                self.configuration.batch.spatial_sort()
