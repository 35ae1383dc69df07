"""Snapshots and exact resume: a run interrupted by snapshot -> restore (a new system) continues the
same trajectory, Voronoi and vertex model, with several instances (each with its own noise key).

Tolerance (written here): positions within 1e-9 after 20 resumed steps (floating-point atomics are
summed in another order in the new system); topology bit-exact.
"""
import numpy as np
import pytest

from helpers import canonical, jittered_lattice

pytestmark = pytest.mark.gpu


def test_voronoi_resume_is_exact(cglib):
    from cellgpu_b200 import VoronoiBatch, restore
    (p1, b1), (p2, b2) = jittered_lattice(16, 18, 0.25, 21), jittered_lattice(12, 14, 0.25, 22)
    N = [len(p1), len(p2)]
    b = VoronoiBatch(N, [b1, b2])
    b.set_positions(np.concatenate([p1, p2]))
    rng = np.random.default_rng(3)
    b.set_directors(rng.uniform(0, 2 * np.pi, sum(N)))
    b.set_motility(np.tile([0.1, 1.0], (sum(N), 1)))
    b.set_preferences(np.tile([1.0, 3.85], (sum(N), 1)))
    b.set_moduli(1.0, 0.8)
    b.set_instance_seeds([7, 8])
    b.triangulate()
    b.spp_run(20, dt=0.01)
    snap = b.snapshot()
    b.spp_run(20, dt=0.01)
    r = restore(snap)
    assert r.N == N and np.allclose(r.boxes, [b1, b2])
    r.spp_run(20, dt=0.01)
    assert np.abs(r.positions() - b.positions()).max() < 1e-9
    assert np.abs(r.directors() - b.directors()).max() < 1e-9
    b.enforce_topology()
    r.enforce_topology()
    nn, nbr = b.topology()
    rn, rnbr = r.topology()
    assert np.array_equal(canonical(nn, nbr), canonical(rn, rnbr))
    b.compute_forces()
    r.compute_forces()
    assert np.abs(r.energies() - b.energies()).max() < 1e-9 * max(1.0, np.abs(b.energies()).max())


def test_vertex_resume_is_exact(cglib):
    from cellgpu_b200 import VertexBatch, restore
    (p1, b1), (p2, b2) = jittered_lattice(12, 14, 0.3, 23), jittered_lattice(10, 12, 0.3, 24)
    N = [len(p1), len(p2)]
    b = VertexBatch(N, [b1, b2], vmax=20)
    b.from_cells(np.concatenate([p1, p2]))
    b.set_preferences(np.tile([1.0, 3.8], (sum(N), 1)))
    b.set_t1_threshold(0.06)
    b.set_instance_seeds([5, 6])
    b.brownian_run(20, dt=0.005, mu=1.0, T=0.01)
    snap = b.snapshot()
    b.brownian_run(20, dt=0.005, mu=1.0, T=0.01)
    r = restore(snap)
    assert isinstance(r, VertexBatch) and r.vmax == 20
    r.brownian_run(20, dt=0.005, mu=1.0, T=0.01)
    assert np.abs(r.positions() - b.positions()).max() < 1e-9
    for x, y in zip(r.vertex_topology(), b.vertex_topology()):
        assert np.array_equal(x, y)
