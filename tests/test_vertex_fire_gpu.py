"""GPU parity of the vertex (AVM) model and of FIRE against the reference's CPU outputs
(tests/golden, generated from the reference's own sources) and the oracle, through the C ABI.

Tolerances (written here):
  * vertex wiring (vn, vcn, cvn, cv rows) and T1 events: bit-exact;
  * vertex positions after Brownian steps with the reference's own noise: 1e-12 absolute
    (forces differ from the reference only in the order the three force sets are summed);
  * vertex forces / areas / perimeters: force_error <= 1e-12, |dAP| <= 1e-12;
  * FIRE (CPU conventions): converges to the same threshold; final energy within 1e-9 relative and
    positions within 1e-6 of the reference's (trajectories near convergence are smooth, but the
    power reduction is summed in another order).
"""
import glob
import os

import numpy as np
import pytest

from helpers import canonical, force_error, jittered_lattice, monolayer

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _gold(pattern):
    f = sorted(glob.glob(os.path.join(HERE, "golden", pattern)))[0]
    return dict(np.load(f))


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def _vertex_from_golden(g):
    from cellgpu_b200 import VertexBatch
    Nc = int(g["Nc"])
    b = VertexBatch([Nc], [tuple(g["box"])], vmax=int(g["vmax"]))
    b.from_cells(g["cellpos"] if "cellpos" in g else None)
    return b


def test_vertex_init_forces_brownian_golden(cglib, torch):
    g = _gold("vertex_Nc*.npz")
    Nc, vmax = int(g["Nc"]), int(g["vmax"])
    b = _vertex_from_golden(g)
    vn, vcn, cvn, cv = b.vertex_topology()
    assert np.abs(b.positions() - g["vpos"]).max() < 1e-12
    assert np.array_equal(vn, g["vn"]) and np.array_equal(vcn, g["vcn"]) and np.array_equal(cvn, g["cvn"])
    for c in range(Nc):
        assert np.array_equal(cv[c, :cvn[c]], g["cv"][c, :cvn[c]])
    b.set_preferences(g["pref"])
    b.compute_forces()
    assert force_error(b.forces(), g["F0"]) < 1e-12
    assert np.abs(b.area_perimeter() - g["AP0"]).max() < 1e-12
    assert abs(b.energies()[0] - float(g["E0"])) < 1e-10
    b.set_t1_threshold(float(g["t1"]))
    steps = int(g["steps"])
    noise = torch.tensor(g["noise"].reshape(steps, -1), device="cuda:0")
    b.brownian_run(steps, dt=float(g["dt"]), mu=1.0, T=float(g["T"]), noise=noise)
    vn, vcn, cvn, cv = b.vertex_topology()
    assert np.abs(b.positions() - g["vpos1"]).max() < 1e-12
    assert np.array_equal(vn, g["vn1"]) and np.array_equal(vcn, g["vcn1"]) and np.array_equal(cvn, g["cvn1"])
    for c in range(Nc):
        assert np.array_equal(cv[c, :cvn[c]], g["cv1"][c, :cvn[c]])
    assert b.counters()["t1_flips"] > 0


def test_vertex_many_t1_matches_oracle(cglib, oracle, torch):
    """A hot Brownian run (large noise, large threshold): many T1 flips per step, each sweep replayed
    in the reference's order; positions and wiring must follow the oracle's sequential sweep."""
    from cellgpu_b200 import VertexBatch
    pos, box = jittered_lattice(16, 18, 0.3, 3)
    Nc = len(pos)
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    vpos, vn, vcn, cvn, cv = oracle.vertex_from_delaunay(pos, box, nn, nbr, vmax=16)
    b = VertexBatch([Nc], [box], vmax=16)
    b.from_cells(pos)
    assert np.abs(b.positions() - vpos).max() < 1e-12
    pref = np.tile([1.0, 3.85], (Nc, 1))
    b.set_preferences(pref)
    b.set_t1_threshold(0.08)
    rng = np.random.default_rng(5)
    steps = 25
    noise = rng.normal(size=(steps, 2 * Nc, 2))
    b.brownian_run(steps, dt=0.01, mu=1.0, T=0.02, noise=torch.tensor(noise.reshape(steps, -1), device="cuda:0"))
    F, AP, nt1 = oracle.vertex_brownian_run(vpos, box, vn, vcn, cvn, cv, pref, noise, dt=0.01, T=0.02,
                                           t1_threshold=0.08)
    gvn, gvcn, gcvn, gcv = b.vertex_topology()
    assert nt1 > 10
    assert np.abs(b.positions() - vpos).max() < 1e-10
    assert np.array_equal(gvn, vn) and np.array_equal(gvcn, vcn) and np.array_equal(gcvn, cvn)
    assert b.counters()["t1_flips"] == nt1


def test_vertex_spp_matches_oracle(cglib, oracle, torch):
    from cellgpu_b200 import VertexBatch
    pos, box = jittered_lattice(12, 14, 0.25, 4)
    Nc = len(pos)
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    vpos, vn, vcn, cvn, cv = oracle.vertex_from_delaunay(pos, box, nn, nbr, vmax=16)
    b = VertexBatch([Nc], [box], vmax=16)
    b.from_cells(pos)
    rng = np.random.default_rng(8)
    theta = rng.uniform(0, 2 * np.pi, Nc)
    mot = np.tile([0.3, 1.0], (Nc, 1))
    pref = np.tile([1.0, 3.8], (Nc, 1))
    b.set_directors(theta)
    b.set_motility(mot)
    b.set_preferences(pref)
    b.set_t1_threshold(0.04)
    steps = 20
    noise = rng.normal(size=(steps, Nc))
    b.spp_run(steps, dt=0.01, mu=1.0, noise=torch.tensor(noise, device="cuda:0"))
    oracle.vertex_spp_run(vpos, box, vn, vcn, cvn, cv, pref, theta, mot, noise, dt=0.01, t1_threshold=0.04)
    assert np.abs(b.positions() - vpos).max() < 1e-10
    assert np.abs(b.directors() - theta).max() < 1e-12
    gvn, gvcn, gcvn, _ = b.vertex_topology()
    assert np.array_equal(gvn, vn) and np.array_equal(gcvn, cvn)


def test_fire_voronoi_golden(cglib):
    from cellgpu_b200 import FireParams, VoronoiBatch
    g = _gold("fire_voronoi_*.npz")
    N = int(g["N"])
    b = VoronoiBatch([N], [tuple(g["box"])])
    b.set_positions(g["pos"])
    b.triangulate()
    b.fire_minimize(FireParams.defaults(force_cutoff=float(g["cutoff"]), max_iterations=int(g["max_iterations"])))
    it, fmax, _ = b.fire_state()
    assert fmax[0] <= float(g["cutoff"])
    E = b.energies()[0]
    assert abs(E - float(g["E1"])) < 1e-9 * max(1.0, abs(E))
    d = b.positions() - g["pos1"]
    d -= np.round(d / g["box"]) * g["box"]
    assert np.abs(d).max() < 1e-6
    nn, nbr = b.topology()
    assert np.array_equal(canonical(nn, nbr), canonical(g["nn1"], g["nbr1"]))


def test_fire_refuses_mixed_precision(cglib):
    """FIRE moves FP64 positions with FP64 forces: a mixed-precision Voronoi system (FP32 forces)
    is refused with an argument error instead of being read as FP64."""
    from cellgpu_b200 import CG_MIXED, CellGPUError, FireParams, VoronoiBatch
    pos, box = monolayer(300, 81)
    b = VoronoiBatch([len(pos)], [box], precision=CG_MIXED)
    b.set_positions(pos)
    b.triangulate()
    with pytest.raises(CellGPUError):
        b.fire_minimize(FireParams.defaults(force_cutoff=1e-10, max_iterations=100))


def test_fire_vertex_golden(cglib):
    from cellgpu_b200 import FireParams, VertexBatch
    g = _gold("fire_vertex_*.npz")
    Nc = int(g["Nc"])
    b = VertexBatch([Nc], [tuple(g["box"])], vmax=int(g["vmax"]))
    b.set_positions(g["vpos"])
    b.set_vertex_topology(g["vn"], g["vcn"], g["cvn"], g["cv"])
    b.set_t1_threshold(0.01)
    b.fire_minimize(FireParams.defaults(force_cutoff=float(g["cutoff"]), max_iterations=int(g["max_iterations"])))
    it, fmax, _ = b.fire_state()
    assert fmax[0] <= float(g["cutoff"])
    E = b.energies()[0]
    assert abs(E - float(g["E1"])) < 1e-9 * max(1.0, abs(E))


def test_fire_batch_instances_independent(cglib):
    """Instances of different sizes minimise independently in one batch and reach the threshold."""
    from cellgpu_b200 import FireParams, VoronoiBatch
    Ns = [120, 300, 64]
    rng = np.random.default_rng(4)
    boxes = [(np.sqrt(n), np.sqrt(n)) for n in Ns]
    pos = np.concatenate([rng.random((n, 2)) * np.sqrt(n) for n in Ns])
    b = VoronoiBatch(Ns, boxes)
    b.set_positions(pos)
    b.triangulate()
    b.fire_minimize(FireParams.defaults(force_cutoff=1e-10, max_iterations=4000))
    it, fmax, _ = b.fire_state()
    assert np.all(fmax <= 1e-10)
    assert len(set(it.tolist())) > 1
    # each instance alone reaches the same energy
    E = b.energies()
    off = 0
    for i, n in enumerate(Ns):
        s = VoronoiBatch([n], [boxes[i]])
        s.set_positions(pos[off:off + n])
        s.triangulate()
        s.fire_minimize(FireParams.defaults(force_cutoff=1e-10, max_iterations=4000))
        assert abs(s.energies()[0] - E[i]) < 1e-8 * max(1.0, E[i])
        off += n


def test_vertex_full_size_matches_oracle(cglib, oracle, torch):
    """The vertex workload at full size (16384 cells, L = 128, p0 ~ U[3.7, 3.9]) from the random
    dual: the device dual equals the oracle's, and 5 Brownian steps with supplied noise (about 2300
    T1 flips, most of them in these first steps) follow the oracle's sequential sweep: positions
    within 1e-10, wiring and flip count exact."""
    from cellgpu_b200 import VertexBatch
    Nc = 16384
    pos, box = monolayer(Nc, 70, L=128.0)
    nn, nbr = oracle.periodic_delaunay(pos, box, 32)
    vpos, vn, vcn, cvn, cv = oracle.vertex_from_delaunay(pos, box, nn, nbr, vmax=30)
    b = VertexBatch([Nc], [box], vmax=30)
    b.from_cells(pos)
    assert np.abs(b.positions() - vpos).max() < 1e-12
    gvn, gvcn, gcvn, gcv = b.vertex_topology()
    assert np.array_equal(gvn, vn) and np.array_equal(gvcn, vcn) and np.array_equal(gcvn, cvn)
    pref = np.column_stack([np.ones(Nc), np.random.default_rng(71).uniform(3.7, 3.9, Nc)])
    b.set_preferences(pref)
    b.set_t1_threshold(0.04)
    steps = 5
    noise = np.random.default_rng(72).normal(size=(steps, 2 * Nc, 2))
    b.brownian_run(steps, dt=0.005, mu=1.0, T=1e-3,
                   noise=torch.tensor(noise.reshape(steps, -1), device="cuda:0"))
    F, AP, nt1 = oracle.vertex_brownian_run(vpos, box, vn, vcn, cvn, cv, pref, noise, dt=0.005, T=1e-3,
                                           t1_threshold=0.04)
    gvn, gvcn, gcvn, gcv = b.vertex_topology()
    assert nt1 > 1000
    assert b.counters()["t1_flips"] == nt1
    assert np.abs(b.positions() - vpos).max() < 1e-10
    assert np.array_equal(gvn, vn) and np.array_equal(gvcn, vcn) and np.array_equal(gcvn, cvn)
    for c in range(Nc):
        assert np.array_equal(gcv[c, :gcvn[c]], cv[c, :cvn[c]])


def test_t1_flip_into_a_full_row_grows_rows(cglib, oracle, torch):
    """Cell rows created exactly as wide as the largest cell (vmax = 10): a T1 flip in the first
    step's sweep adds an 11th vertex to such a cell. The sweep stops before that flip, the rows
    grow and the sweep resumes where it stopped, as the reference grows vertexMax mid-sweep
    (src/models/vertexModelBase.cpp:474-500,674-684). The hot Brownian run (about 300 flips) then
    follows the oracle, whose rows are wide enough from the start: wiring exact, positions 1e-10."""
    from cellgpu_b200 import VertexBatch
    pos, box = monolayer(400, 43)
    Nc = len(pos)
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    vpos, vn, vcn, cvn, cv = oracle.vertex_from_delaunay(pos, box, nn, nbr, vmax=20)
    vmax0 = int(cvn.max())
    assert vmax0 == 10
    b = VertexBatch([Nc], [box], vmax=vmax0)
    b.from_cells(pos)
    pref = np.tile([1.0, 3.85], (Nc, 1))
    b.set_preferences(pref)
    b.set_t1_threshold(0.08)
    rng = np.random.default_rng(5)
    steps = 40
    noise = rng.normal(size=(steps, 2 * Nc, 2))
    b.brownian_run(steps, dt=0.01, mu=1.0, T=0.02, noise=torch.tensor(noise.reshape(steps, -1), device="cuda:0"))
    nt1, widest = 0, 0
    for t in range(steps):
        _, _, k = oracle.vertex_brownian_run(vpos, box, vn, vcn, cvn, cv, pref, noise[t:t + 1], dt=0.01, T=0.02,
                                            t1_threshold=0.08)
        nt1 += k
        widest = max(widest, int(cvn.max()))
    assert widest > vmax0  # the oracle's run needs wider rows at some step
    assert b.row_capacity() > vmax0
    gvn, gvcn, gcvn, gcv = b.vertex_topology()
    assert np.array_equal(gvn, vn) and np.array_equal(gvcn, vcn) and np.array_equal(gcvn, cvn)
    for c in range(Nc):
        assert np.array_equal(gcv[c, :cvn[c]], cv[c, :cvn[c]])
    assert np.abs(b.positions() - vpos).max() < 1e-10
    assert b.counters()["t1_flips"] == nt1
