"""GPU parity of line tension -- Voronoi model (VoronoiQuadraticEnergyWithTension) and vertex model
(VertexQuadraticEnergyWithTension) -- against the reference's outputs (tests/golden/tension_N*.npz,
tests/golden/vertex_tension_Nc*.npz) and the oracle, through the C ABI.

Tolerances: FP64 forces force_error <= 1e-10, areas/perimeters relative 1e-12, energy relative
1e-12 (summation order differs); mixed precision RMS force error <= 1e-6 of FP64.
"""
import glob
import os

import numpy as np
import pytest

from helpers import canonical, force_error, monolayer

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def _golden():
    return dict(np.load(sorted(glob.glob(os.path.join(GOLD, "tension_N*.npz")))[0]))


def _tension_batch(g, mode, precision=0):
    from cellgpu_b200 import VoronoiBatch
    N = int(g["N"])
    b = VoronoiBatch([N], [tuple(g["box"])], K=16, precision=precision)
    b.set_positions(g["pos"])
    b.set_preferences(g["pref"])
    b.triangulate()
    b.set_cell_types(g["types"])
    if mode == "simple":
        b.set_tension(float(g["gamma"]))
    else:
        b.set_tension_matrix(g["gammas"])
    return b


@pytest.mark.parametrize("mode", ["simple", "matrix"])
def test_tension_forces_match_reference(cglib, mode):
    g = _golden()
    b = _tension_batch(g, mode)
    b.compute_forces()
    np.testing.assert_allclose(b.area_perimeter(), g["AP_" + mode], rtol=1e-12, atol=1e-12)
    assert force_error(b.forces(), g["F_" + mode]) < 1e-10
    E = b.energies()[0]
    assert abs(E - float(g["E_" + mode])) < 1e-12 * abs(E)


def test_tension_off_and_like_types(cglib, oracle):
    """gamma = 0, an empty matrix, or one type everywhere give the plain quadratic forces."""
    g = _golden()
    pos, box, pref = g["pos"], tuple(g["box"]), g["pref"]
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    AP = oracle.voronoi_geometry(pos, box, nn, nbr)
    F0 = oracle.voronoi_forces(pos, box, nn, nbr, AP, pref)
    b = _tension_batch(g, "simple")
    b.set_tension(0.0)
    b.compute_forces()
    assert force_error(b.forces(), F0) < 1e-10
    b.set_tension_matrix(g["gammas"])
    b.set_tension_matrix(np.zeros((0, 0)))
    b.compute_forces()
    assert force_error(b.forces(), F0) < 1e-10
    b.set_tension(0.3)
    b.set_cell_types(np.full(len(pos), 2))
    b.compute_forces()
    assert force_error(b.forces(), F0) < 1e-10
    assert abs(b.energies()[0] - oracle.voronoi_energy(AP, pref)) < 1e-12 * b.energies()[0]


def test_tension_argument_checks(cglib):
    from cellgpu_b200 import CellGPUError
    g = _golden()
    b = _tension_batch(g, "matrix")
    with pytest.raises(CellGPUError):
        b.set_cell_types(np.full(int(g["N"]), 3))  # outside the 3 x 3 matrix
    with pytest.raises(CellGPUError):
        b.set_cell_types(np.full(int(g["N"]), -1))
    asym = g["gammas"].copy()
    asym[0, 1] += 0.05
    with pytest.raises(CellGPUError):
        b.set_tension_matrix(asym)


def test_tension_mixed_precision(cglib):
    g = _golden()
    b64 = _tension_batch(g, "matrix", precision=0)
    b32 = _tension_batch(g, "matrix", precision=1)
    b64.compute_forces()
    b32.compute_forces()
    F64, F32 = b64.forces(), b32.forces()
    rms = np.sqrt(np.mean(np.sum((F32 - F64) ** 2, 1))) / np.sqrt(np.mean(np.sum(F64 ** 2, 1)))
    assert rms < 1e-6


@pytest.mark.parametrize("mode", ["simple", "matrix"])
def test_tension_spp_each_step_matches_oracle(cglib, oracle, torch, mode):
    """SPP steps with tension (the captured step graph carries the tension arguments): each GPU
    step against the oracle's step from the same state, re-synchronised after each step."""
    N, steps, dt = 500, 12, 0.01
    pos, box = monolayer(N, 21)
    rng = np.random.default_rng(21)
    types = rng.integers(0, 3, N)
    theta = rng.uniform(0, 2 * np.pi, N)
    mot = np.tile([0.1, 1.0], (N, 1))
    pref = np.tile([1.0, 3.8], (N, 1))
    gammas = np.array([[0.0, 0.1, 0.3], [0.1, 0.0, 0.2], [0.3, 0.2, 0.0]])
    kw = dict(gamma=0.15) if mode == "simple" else dict(gammas=gammas)
    from cellgpu_b200 import VoronoiBatch
    b = VoronoiBatch([N], [box], K=16, precision=0)
    b.set_positions(pos)
    b.set_directors(theta)
    b.set_motility(mot)
    b.set_preferences(pref)
    b.triangulate()
    b.set_cell_types(types)
    if mode == "simple":
        b.set_tension(0.15)
    else:
        b.set_tension_matrix(gammas)
    noise = rng.normal(size=(steps, N))
    opos, oth = pos.copy(), theta.copy()
    onn, onbr = oracle.periodic_delaunay(opos, box, 16)
    for s in range(steps):
        AP = oracle.voronoi_geometry(opos, box, onn, onbr)
        F = oracle.voronoi_tension_forces(opos, box, onn, onbr, AP, pref, types, **kw)
        E = oracle.voronoi_tension_energy(opos, box, onn, onbr, AP, pref, types, **kw)
        oracle.spp_step(opos, box, F, oth, mot, noise[s], dt=dt)
        onn, onbr = oracle.periodic_delaunay(opos, box, 16)
        b.spp_run(1, dt=dt, mu=1.0, noise=torch.tensor(noise[s:s + 1], device="cuda:0"))
        assert force_error(b.forces(), F) < 1e-10
        assert abs(b.energies()[0] - E) < 1e-12 * abs(E)
        assert np.abs(b.positions() - opos).max() < 1e-12
        b.enforce_topology()
        nn, nbr = b.topology()
        assert np.array_equal(canonical(nn, nbr), canonical(onn, onbr))
        b.set_positions(opos)
        b.set_directors(oth)
        b.set_topology(onn, onbr)


def test_tension_survives_snapshot_and_sort(cglib):
    """Cell types and the tension matrix travel in snapshots (a restored batch continues the same
    trajectory) and move with the cells when the batch is spatially re-sorted."""
    from cellgpu_b200 import restore
    g = _golden()
    N = int(g["N"])
    b = _tension_batch(g, "matrix")
    b.set_directors(np.random.default_rng(4).uniform(0, 2 * np.pi, N))
    b.set_motility(np.tile([0.1, 1.0], (N, 1)))
    b.spp_run(10, dt=0.01)
    snap = b.snapshot()
    b.spp_run(15, dt=0.01)
    r = restore(snap)
    r.spp_run(15, dt=0.01)
    assert np.abs(r.positions() - b.positions()).max() < 1e-9
    b.enforce_topology()
    r.enforce_topology()
    b.compute_forces()
    r.compute_forces()
    assert abs(r.energies()[0] - b.energies()[0]) < 1e-9 * abs(b.energies()[0])
    F0, E0 = b.forces(), b.energies()[0]
    b.spatial_sort()
    tags = b.tags()
    assert not np.array_equal(tags, np.arange(N))
    b.compute_forces()
    assert force_error(b.forces(), F0[tags]) < 1e-12
    assert abs(b.energies()[0] - E0) < 1e-12 * abs(E0)


def _vertex_golden():
    return dict(np.load(sorted(glob.glob(os.path.join(GOLD, "vertex_tension_Nc*.npz")))[0]))


def _vertex_tension_batch(g, mode):
    from cellgpu_b200 import VertexBatch
    Nc = int(g["Nc"])
    b = VertexBatch([Nc], [tuple(g["box"])], vmax=int(g["vmax"]))
    b.set_vertex_topology(g["vn"], g["vcn"], g["cvn"], g["cv"])
    b.set_positions(g["vpos"])
    b.set_preferences(g["pref"])
    b.set_cell_types(g["types"])
    if mode == "simple":
        b.set_tension(float(g["gamma"]))
    else:
        b.set_tension_matrix(g["gammas"])
    return b


@pytest.mark.parametrize("mode", ["simple", "matrix"])
def test_vertex_tension_forces_match_reference(cglib, oracle, mode):
    g = _vertex_golden()
    b = _vertex_tension_batch(g, mode)
    b.compute_forces()
    np.testing.assert_allclose(b.area_perimeter(), g["AP_" + mode], rtol=1e-12, atol=1e-12)
    assert force_error(b.forces(), g["F_" + mode]) < 1e-10
    kw = dict(gamma=float(g["gamma"])) if mode == "simple" else dict(gammas=g["gammas"])
    E = oracle.vertex_tension_energy(g["vpos"], tuple(g["box"]), g["cvn"], g["cv"], g["vcn"], g["AP_" + mode],
                                     g["pref"], g["types"], **kw)
    assert abs(b.energies()[0] - E) < 1e-12 * abs(E)
    assert E > float(g["E_" + mode])  # the quadratic part plus a positive tension


def test_vertex_tension_dynamics_and_resume(cglib, oracle, torch):
    """Brownian steps with T1 transitions and tension: the forces of the state reached are the
    oracle's on that state; a snapshot taken mid-run restores types and matrix and continues the
    same trajectory."""
    from cellgpu_b200 import restore
    g = _vertex_golden()
    b = _vertex_tension_batch(g, "matrix")
    b.set_t1_threshold(0.04)
    b.brownian_run(20, dt=0.005, mu=1.0, T=2e-3)
    snap = b.snapshot()
    b.brownian_run(20, dt=0.005, mu=1.0, T=2e-3)
    r = restore(snap)
    r.brownian_run(20, dt=0.005, mu=1.0, T=2e-3)
    assert np.abs(r.positions() - b.positions()).max() < 1e-9
    b.compute_forces()
    vn, vcn, cvn, cv = b.vertex_topology()
    vp = b.positions()
    box = tuple(g["box"])
    AP = oracle.vertex_geometry(vp, box, cvn, cv)
    F = oracle.vertex_tension_forces(vp, box, cvn, cv, vcn, AP, g["pref"], g["types"], gammas=g["gammas"])
    assert force_error(b.forces(), F) < 1e-10


def test_vertex_tension_class_api(cglib):
    """VertexQuadraticEnergyWithTension: tension raises the energy and leaves the net force zero."""
    from cellgpu_b200 import VertexQuadraticEnergyWithTension
    m = VertexQuadraticEnergyWithTension(200, 1.0, 3.8, True)
    E0 = m.computeEnergy()
    m.setCellType(np.arange(200) % 2)
    m.setSurfaceTension(0.3)
    m.setUseSurfaceTension(True)
    E1 = m.computeEnergy()
    assert E1 > E0
    assert np.abs(m.returnForces().sum(axis=0)).max() < 1e-10
    m.setUseSurfaceTension(False)
    assert abs(m.computeEnergy() - E0) < 1e-12 * E0
