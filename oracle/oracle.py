"""TEST INFRASTRUCTURE ONLY: ctypes front end of the CPU oracle (``oracle/cg_oracle.c``).

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` import
this module, and only as the checker. The product (``cellgpu_b200``) never imports it.

Every function takes and returns numpy arrays in the reference's layouts: positions ``(N, 2)``
float64, neighbour rows ``(N, K)`` int32 with ``n_idx(k, c) = c*K + k``
(inc/utility/indexer.h:38-41), box as ``(Lx, Ly)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libcgoracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class FireParams(C.Structure):
    """Mirror of ``cgo_fire_params``; defaults of EnergyMinimizerFIRE::initializeParameters
    (src/updaters/EnergyMinimizerFIRE2D.cpp:24-41)."""

    _fields_ = [
        ("dt", C.c_double), ("dt_max", C.c_double), ("dt_min", C.c_double), ("dt_inc", C.c_double),
        ("dt_dec", C.c_double), ("alpha", C.c_double), ("alpha_start", C.c_double),
        ("alpha_dec", C.c_double), ("force_cutoff", C.c_double), ("n_min", C.c_int),
        ("max_iterations", C.c_int), ("iterations", C.c_int), ("n_since_negative_power", C.c_int),
        ("power", C.c_double), ("force_max", C.c_double),
    ]

    @classmethod
    def defaults(cls, **kw):
        p = cls(dt=0.01, dt_max=0.1, dt_min=0.01 * 0.01, dt_inc=1.05, dt_dec=0.95, alpha=0.99,
                alpha_start=0.99, alpha_dec=0.9, force_cutoff=1e-7, n_min=5, max_iterations=1000,
                iterations=0, n_since_negative_power=0, power=0.0, force_max=100.0)
        for k, v in kw.items():
            setattr(p, k, v)
        if "dt" in kw and "dt_min" not in kw:
            p.dt_min = kw["dt"] * 0.01  # setDeltaT sets deltaTMin = dt*0.01 (EnergyMinimizerFIRE2D.h:42)
        if "alpha_start" in kw and "alpha" not in kw:
            p.alpha = kw["alpha_start"]
        return p


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.cgo_local_star.argtypes = [C.c_int, _dp, C.c_int, _ip]
        L.cgo_local_star_bruteforce.argtypes = [C.c_int, _dp, C.c_int, _ip]
        L.cgo_periodic_delaunay.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, _ip]
        L.cgo_topology_mismatch.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, _ip]
        L.cgo_voronoi_geometry.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, _ip, _dp]
        L.cgo_voronoi_forces.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, _ip, _dp, _dp, C.c_double,
                                         C.c_double, _dp]
        L.cgo_voronoi_energy.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_double]
        L.cgo_voronoi_energy.restype = C.c_double
        L.cgo_voronoi_tension_forces.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, _ip, _dp, _dp, C.c_double,
                                                 C.c_double, _ip, C.c_int, C.c_double, C.c_void_p, _dp]
        L.cgo_voronoi_tension_energy.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, _ip, _dp, _dp, C.c_double,
                                                 C.c_double, _ip, C.c_int, C.c_double, C.c_void_p]
        L.cgo_voronoi_tension_energy.restype = C.c_double
        L.cgo_spp_step.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double]
        L.cgo_voronoi_spp_run.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, _ip, _dp, _dp, _dp,
                                          C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _dp,
                                          _dp, _dp]
        L.cgo_brownian_disp.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_double, _dp]
        L.cgo_vertex_from_delaunay.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, _ip, C.c_int, _dp, _ip,
                                               _ip, _ip, _ip]
        L.cgo_vertex_geometry.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, _ip, _dp]
        L.cgo_vertex_forces.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int, _ip, _ip, _ip, _dp, _dp,
                                        C.c_double, C.c_double, _dp]
        L.cgo_vertex_tension_forces.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int, _ip, _ip, _ip, _dp, _dp,
                                                C.c_double, C.c_double, _ip, C.c_int, C.c_double, C.c_void_p,
                                                _dp]
        L.cgo_vertex_tension_energy.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, _ip, _ip, _dp, _dp, C.c_double,
                                                C.c_double, _ip, C.c_int, C.c_double, C.c_void_p]
        L.cgo_vertex_tension_energy.restype = C.c_double
        L.cgo_vertex_t1.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_double, C.c_int, _ip, _ip, _ip, _ip,
                                    C.c_int, _ip]
        L.cgo_vertex_brownian_run.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int, _ip, _ip, _ip, _ip,
                                              _dp, C.c_double, C.c_double, C.c_double, C.c_double,
                                              C.c_double, C.c_double, C.c_int, _dp, _dp, _dp,
                                              C.POINTER(C.c_int)]
        L.cgo_vertex_spp_run.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int, _ip, _ip, _ip, _ip, _dp,
                                         C.c_double, C.c_double, _dp, _dp, C.c_double, C.c_double,
                                         C.c_double, C.c_int, _dp]
        L.cgo_fire_voronoi.argtypes = [C.c_int, _dp, _dp, C.c_int, _ip, _ip, _dp, C.c_double, C.c_double,
                                       C.POINTER(FireParams), _dp, _dp, _dp]
        L.cgo_fire_vertex.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int, _ip, _ip, _ip, _ip, _dp,
                                      C.c_double, C.c_double, C.c_double, C.POINTER(FireParams), _dp, _dp,
                                      _dp]
        _lib = L
    return _lib


def _box(box):
    b = np.asarray(box, dtype=np.float64).reshape(-1)
    if b.size == 1:
        b = np.array([b[0], b[0]])
    return np.ascontiguousarray(b)


def _f64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a if shape is None else a.reshape(shape)


def local_star(rel, brute=False):
    rel = _f64(rel)
    out = np.zeros(rel.shape[0] + 1, np.int32)
    f = lib().cgo_local_star_bruteforce if brute else lib().cgo_local_star
    z = f(rel.shape[0], rel, out.size, out)
    return out[:z] if z > 0 else z


def periodic_delaunay(pos, box, K=16):
    pos = _f64(pos)
    N = pos.shape[0]
    nn = np.zeros(N, np.int32)
    nbr = np.full((N, K), -1, np.int32)
    st = lib().cgo_periodic_delaunay(N, pos, _box(box), K, nn, nbr)
    if st:
        raise RuntimeError(f"oracle Delaunay failed ({st})")
    return nn, nbr


def topology_mismatch(pos, box, nn, nbr):
    pos = _f64(pos)
    nbr = np.ascontiguousarray(nbr, np.int32)
    return lib().cgo_topology_mismatch(pos.shape[0], pos, _box(box), nbr.shape[1],
                                       np.ascontiguousarray(nn, np.int32), nbr)


def canonical_rows(nn, nbr):
    """Rotate each CCW row to start at its smallest index; pad with -1."""
    nn = np.asarray(nn)
    nbr = np.asarray(nbr)
    out = np.full_like(nbr, -1)
    for i in range(nn.shape[0]):
        z = int(nn[i])
        r = nbr[i, :z]
        s = int(np.argmin(r))
        out[i, :z] = np.roll(r, -s)
    return out


def voronoi_geometry(pos, box, nn, nbr):
    pos = _f64(pos)
    nbr = np.ascontiguousarray(nbr, np.int32)
    AP = np.zeros((pos.shape[0], 2))
    lib().cgo_voronoi_geometry(pos.shape[0], pos, _box(box), nbr.shape[1],
                               np.ascontiguousarray(nn, np.int32), nbr, AP)
    return AP


def voronoi_forces(pos, box, nn, nbr, AP, APpref, KA=1.0, KP=1.0):
    pos = _f64(pos)
    nbr = np.ascontiguousarray(nbr, np.int32)
    F = np.zeros((pos.shape[0], 2))
    st = lib().cgo_voronoi_forces(pos.shape[0], pos, _box(box), nbr.shape[1],
                                  np.ascontiguousarray(nn, np.int32), nbr, _f64(AP), _f64(APpref),
                                  KA, KP, F)
    if st:
        raise RuntimeError("oracle: inconsistent triangulation")
    return F


def voronoi_energy(AP, APpref, KA=1.0, KP=1.0):
    AP = _f64(AP)
    return lib().cgo_voronoi_energy(AP.shape[0], AP, _f64(APpref), KA, KP)


def _tension_args(types, gamma, gammas):
    types = np.ascontiguousarray(types, np.int32)
    if gammas is None:
        return types, 0, float(gamma), None, None
    g = np.ascontiguousarray(gammas, np.float64)
    return types, int(round(np.sqrt(g.size))), 0.0, g.ctypes.data_as(C.c_void_p), g


def voronoi_tension_forces(pos, box, nn, nbr, AP, APpref, types, gamma=0.0, gammas=None, KA=1.0, KP=1.0):
    """Forces with line tension between unlike cells: one gamma, or the ntypes x ntypes matrix
    gammas (row = own type)."""
    pos = _f64(pos)
    nbr = np.ascontiguousarray(nbr, np.int32)
    F = np.zeros((pos.shape[0], 2))
    types, nt, g, tp, _keep = _tension_args(types, gamma, gammas)
    st = lib().cgo_voronoi_tension_forces(pos.shape[0], pos, _box(box), nbr.shape[1],
                                          np.ascontiguousarray(nn, np.int32), nbr, _f64(AP), _f64(APpref), KA,
                                          KP, types, nt, g, tp, F)
    if st:
        raise RuntimeError("oracle: inconsistent triangulation")
    return F


def voronoi_tension_energy(pos, box, nn, nbr, AP, APpref, types, gamma=0.0, gammas=None, KA=1.0, KP=1.0):
    pos = _f64(pos)
    nbr = np.ascontiguousarray(nbr, np.int32)
    types, nt, g, tp, _keep = _tension_args(types, gamma, gammas)
    return lib().cgo_voronoi_tension_energy(pos.shape[0], pos, _box(box), nbr.shape[1],
                                            np.ascontiguousarray(nn, np.int32), nbr, _f64(AP), _f64(APpref), KA,
                                            KP, types, nt, g, tp)


def spp_step(pos, box, F, theta, motility, noise, dt=0.01, mu=1.0):
    """One self-propelled step in place (pos, theta) with the forces F and one normal per cell."""
    lib().cgo_spp_step(pos.shape[0], pos, _box(box), _f64(F), theta, _f64(motility), _f64(noise), dt, mu)


def voronoi_spp_run(pos, box, nn, nbr, theta, motility, APpref, noise, dt=0.01, mu=1.0, KA=1.0,
                    KP=1.0):
    """Advance n_steps = noise.shape[0] SPP steps in place; returns (F, AP) of the last force pass."""
    pos = _f64(pos)
    N = pos.shape[0]
    noise = _f64(noise).reshape(-1, N)
    F = np.zeros((N, 2))
    AP = np.zeros((N, 2))
    st = lib().cgo_voronoi_spp_run(N, pos, _box(box), nbr.shape[1], nn, nbr, theta, _f64(motility),
                                   _f64(APpref), KA, KP, dt, mu, noise.shape[0], noise, F, AP)
    if st:
        raise RuntimeError(f"oracle SPP run failed ({st})")
    return F, AP


def apply_exclusions(F, excluded):
    """Particle exclusions after a force evaluation (src/models/voronoiQuadraticEnergy.cpp:368-377,
    gpu_sum_forces_with_exclusions_kernel, src/models/voronoiQuadraticEnergy.cu:59-93): an excluded
    cell's force becomes the external force -F and its force is zeroed. Returns (F, external)."""
    ex = np.asarray(excluded) != 0
    F = np.array(F, dtype=np.float64, copy=True)
    ext = np.zeros_like(F)
    ext[ex] = -F[ex]
    F[ex] = 0.0
    return F, ext


def voronoi_spp_run_exclusions(pos, box, nn, nbr, theta, motility, APpref, noise, excluded, dt=0.01, mu=1.0,
                               KA=1.0, KP=1.0):
    """voronoi_spp_run with particle exclusions (motility must already hold v0 = Dr = 0 for the
    excluded cells, as voronoiModelBase::setExclusions sets it, src/models/voronoiModelBase.cpp:85-104):
    per step the geometry, the forces, the exclusions, one SPP step, and the Delaunay triangulation
    of the new positions, in place. Returns (F, external, AP) of the last force evaluation."""
    noise = _f64(noise).reshape(-1, pos.shape[0])
    F = ext = AP = None
    for t in range(noise.shape[0]):
        AP = voronoi_geometry(pos, box, nn, nbr)
        F, ext = apply_exclusions(voronoi_forces(pos, box, nn, nbr, AP, APpref, KA, KP), excluded)
        spp_step(pos, box, F, theta, motility, noise[t], dt, mu)
        nn[:], nbr[:] = periodic_delaunay(pos, box, nbr.shape[1])
    return F, ext, AP


def vertex_from_delaunay(pos, box, nn, nbr, vmax=30):
    pos = _f64(pos)
    N = pos.shape[0]
    nbr = np.ascontiguousarray(nbr, np.int32)
    Nv = 2 * N
    vpos = np.zeros((Nv, 2))
    vn = np.zeros(3 * Nv, np.int32)
    vcn = np.zeros(3 * Nv, np.int32)
    cvn = np.zeros(N, np.int32)
    cv = np.full((N, vmax), -1, np.int32)
    st = lib().cgo_vertex_from_delaunay(N, pos, _box(box), nbr.shape[1],
                                        np.ascontiguousarray(nn, np.int32), nbr, vmax, vpos, vn, vcn,
                                        cvn, cv)
    if st < 0:
        raise RuntimeError(f"oracle vertex init failed ({st})")
    return vpos, vn, vcn, cvn, cv


def vertex_geometry(vpos, box, cvn, cv):
    vpos = _f64(vpos)
    cv = np.ascontiguousarray(cv, np.int32)
    AP = np.zeros((cv.shape[0], 2))
    lib().cgo_vertex_geometry(cv.shape[0], vpos, _box(box), cv.shape[1],
                              np.ascontiguousarray(cvn, np.int32), cv, AP)
    return AP


def vertex_forces(vpos, box, cvn, cv, vcn, AP, APpref, KA=1.0, KP=1.0):
    vpos = _f64(vpos)
    cv = np.ascontiguousarray(cv, np.int32)
    F = np.zeros_like(vpos)
    lib().cgo_vertex_forces(cv.shape[0], vpos.shape[0], vpos, _box(box), cv.shape[1],
                            np.ascontiguousarray(cvn, np.int32), cv, np.ascontiguousarray(vcn, np.int32),
                            _f64(AP), _f64(APpref), KA, KP, F)
    return F


def vertex_tension_forces(vpos, box, cvn, cv, vcn, AP, APpref, types, gamma=0.0, gammas=None, KA=1.0, KP=1.0):
    """Vertex forces with line tension on edges between cells of different types."""
    vpos = _f64(vpos)
    cv = np.ascontiguousarray(cv, np.int32)
    F = np.zeros_like(vpos)
    types, nt, g, tp, _keep = _tension_args(types, gamma, gammas)
    lib().cgo_vertex_tension_forces(cv.shape[0], vpos.shape[0], vpos, _box(box), cv.shape[1],
                                    np.ascontiguousarray(cvn, np.int32), cv, np.ascontiguousarray(vcn, np.int32),
                                    _f64(AP), _f64(APpref), KA, KP, types, nt, g, tp, F)
    return F


def vertex_tension_energy(vpos, box, cvn, cv, vcn, AP, APpref, types, gamma=0.0, gammas=None, KA=1.0, KP=1.0):
    vpos = _f64(vpos)
    cv = np.ascontiguousarray(cv, np.int32)
    types, nt, g, tp, _keep = _tension_args(types, gamma, gammas)
    return lib().cgo_vertex_tension_energy(cv.shape[0], vpos, _box(box), cv.shape[1],
                                           np.ascontiguousarray(cvn, np.int32), cv,
                                           np.ascontiguousarray(vcn, np.int32), _f64(AP), _f64(APpref), KA, KP,
                                           types, nt, g, tp)


def vertex_t1(vpos, box, threshold, vn, vcn, cvn, cv, max_events=4096):
    """In-place sequential T1 sweep; returns the list of (vertex1, vertex2) events."""
    ev = np.zeros(2 * max_events, np.int32)
    n = lib().cgo_vertex_t1(cv.shape[0], vpos.shape[0], vpos, _box(box), threshold, cv.shape[1], vn, vcn,
                            cvn, cv, max_events, ev)
    if n < 0:
        raise RuntimeError(f"oracle T1 failed ({n})")
    return ev[: 2 * min(n, max_events)].reshape(-1, 2)


def vertex_brownian_run(vpos, box, vn, vcn, cvn, cv, APpref, noise, dt=0.005, mu=1.0, T=1e-3,
                        t1_threshold=0.04, KA=1.0, KP=1.0):
    Nv = vpos.shape[0]
    Nc = cv.shape[0]
    noise = _f64(noise).reshape(-1, Nv, 2)
    F = np.zeros((Nv, 2))
    AP = np.zeros((Nc, 2))
    nt1 = C.c_int(0)
    st = lib().cgo_vertex_brownian_run(Nc, Nv, vpos, _box(box), cv.shape[1], vn, vcn, cvn, cv,
                                       _f64(APpref), KA, KP, dt, mu, T, t1_threshold, noise.shape[0],
                                       noise, F, AP, C.byref(nt1))
    if st:
        raise RuntimeError(f"oracle vertex run failed ({st})")
    return F, AP, nt1.value


def vertex_spp_run(vpos, box, vn, vcn, cvn, cv, APpref, theta, motility, noise, dt=0.01, mu=1.0,
                   t1_threshold=0.04, KA=1.0, KP=1.0):
    Nv = vpos.shape[0]
    Nc = cv.shape[0]
    noise = _f64(noise).reshape(-1, Nc)
    st = lib().cgo_vertex_spp_run(Nc, Nv, vpos, _box(box), cv.shape[1], vn, vcn, cvn, cv, _f64(APpref), KA, KP,
                                  theta, _f64(motility), dt, mu, t1_threshold, noise.shape[0], noise)
    if st:
        raise RuntimeError(f"oracle vertex SPP failed ({st})")


def fire_voronoi(pos, box, nn, nbr, APpref, params, vel=None, KA=1.0, KP=1.0):
    pos = _f64(pos)
    N = pos.shape[0]
    vel = np.zeros((N, 2)) if vel is None else vel
    F = np.zeros((N, 2))
    AP = np.zeros((N, 2))
    st = lib().cgo_fire_voronoi(N, pos, _box(box), nbr.shape[1], nn, nbr, _f64(APpref), KA, KP,
                                C.byref(params), vel, F, AP)
    if st:
        raise RuntimeError(f"oracle FIRE failed ({st})")
    return F, AP, vel


def fire_vertex(vpos, box, vn, vcn, cvn, cv, APpref, params, t1_threshold=0.04, vel=None, KA=1.0,
                KP=1.0):
    Nv = vpos.shape[0]
    Nc = cv.shape[0]
    vel = np.zeros((Nv, 2)) if vel is None else vel
    F = np.zeros((Nv, 2))
    AP = np.zeros((Nc, 2))
    st = lib().cgo_fire_vertex(Nc, Nv, vpos, _box(box), cv.shape[1], vn, vcn, cvn, cv, _f64(APpref), KA,
                               KP, t1_threshold, C.byref(params), vel, F, AP)
    if st:
        raise RuntimeError(f"oracle vertex FIRE failed ({st})")
    return F, AP, vel
