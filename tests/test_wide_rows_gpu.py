"""Rows wider than 16 neighbours. A cell ringed by 18 cells has 18 Delaunay neighbours: a system
created with the default capacity of 16 widens its rows to 32 (as the reference grows neighMax)
and then runs its group kernels in their 32-slot form; topology, forces and SPP steps follow the
oracle. A system created with K = 32 agrees with a K = 16 one on an ordinary monolayer.

Tolerances (written here): topology bit-exact (canonical rotation); forces force_error <= 1e-10;
positions after each re-synchronised step within 1e-12; K = 16 against K = 32 within 1e-12 / 1e-9
(trajectories: floating-point atomics order).
"""
import ctypes as C

import numpy as np
import pytest

from helpers import canonical, force_error, jittered_lattice

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def _flower(n_ring=18, L=20.0, seed=5):
    rng = np.random.default_rng(seed)
    c = np.array([L / 2, L / 2])
    ang = np.arange(n_ring) * 2 * np.pi / n_ring + 0.01
    ring = c + np.stack([np.cos(ang), np.sin(ang)], 1)
    g = np.arange(0.5, L, 1.0)
    lat = np.array([(x, y) for y in g for x in g]) + rng.uniform(-0.15, 0.15, (len(g) ** 2, 2))
    lat = lat[np.linalg.norm(lat - c, axis=1) > 1.8]
    return np.concatenate([[c], ring, lat]) % L, (L, L)


def _canon(nn, nbr):
    return canonical(nn, nbr)[:, :int(nn.max())]


def test_flower_widens_rows_and_follows_the_oracle(cglib, oracle, torch):
    from cellgpu_b200 import VoronoiBatch
    pos, box = _flower()
    N = len(pos)
    rng = np.random.default_rng(6)
    theta = rng.uniform(0, 2 * np.pi, N)
    mot = np.tile([0.05, 1.0], (N, 1))
    pref = np.tile([1.0, 3.8], (N, 1))
    b = VoronoiBatch([N], [box])  # capacity 16
    b.set_positions(pos)
    b.set_directors(theta)
    b.set_motility(mot)
    b.set_preferences(pref)
    b.triangulate()
    assert b._lib.cg_neighbor_capacity(b.handle) == 32
    nn, nbr = b.topology()
    onn, onbr = oracle.periodic_delaunay(pos, box, 32)
    assert nn[0] == 18
    assert np.array_equal(_canon(nn, nbr), _canon(onn, onbr))
    b.compute_forces()
    AP = oracle.voronoi_geometry(pos, box, onn, onbr)
    assert force_error(b.forces(), oracle.voronoi_forces(pos, box, onn, onbr, AP, pref)) < 1e-10
    # SPP steps (local repairs in the 32-slot kernels), each against the oracle's step
    noise = rng.normal(size=(8, N))
    opos, oth = pos.copy(), theta.copy()
    for s in range(8):
        b.spp_run(1, dt=0.01, mu=1.0, noise=torch.tensor(noise[s:s + 1], device="cuda:0"))
        F, _ = oracle.voronoi_spp_run(opos, box, onn, onbr, oth, mot, pref, noise[s:s + 1], dt=0.01)
        assert np.abs(b.positions() - opos).max() < 1e-12
        assert force_error(b.forces(), F) < 1e-10
        b.enforce_topology()
        nn, nbr = b.topology()
        assert np.array_equal(_canon(nn, nbr), _canon(onn, onbr))
        b.set_positions(opos)
        b.set_directors(oth)
        b.set_topology(onn, onbr)


def test_wide_rows_agree_with_narrow(cglib, torch):
    from cellgpu_b200 import VoronoiBatch
    pos, box = jittered_lattice(40, 46, 0.25, 41)  # well conditioned: free runs stay comparable
    N = len(pos)
    rng = np.random.default_rng(42)
    theta = rng.uniform(0, 2 * np.pi, N)
    out = []
    for K in (16, 32):
        b = VoronoiBatch([N], [box], K=K)
        b.set_positions(pos)
        b.set_directors(theta)
        b.set_motility(np.tile([0.3, 1.0], (N, 1)))
        b.set_preferences(np.tile([1.0, 3.8], (N, 1)))
        b.set_seed(7)
        b.triangulate()
        b.compute_forces()
        F0 = b.forces()
        b.spp_run(20, dt=0.02)
        b.enforce_topology()
        nn, nbr = b.topology()
        out.append((F0, b.positions(), _canon(nn, nbr), b.counters()["rows_changed"]))
    assert force_error(out[1][0], out[0][0]) < 1e-12
    assert np.abs(out[1][1] - out[0][1]).max() < 1e-9
    assert np.array_equal(out[1][2], out[0][2])
    assert out[0][3] > 0 and out[1][3] > 0  # the repair ran in both forms


def test_rows_grow_during_steps(cglib, oracle):
    """The rows overflow inside a step: the system starts from rows that fit 16 (the Delaunay rows
    of the same cells with the ringed cell elsewhere), the step's repair or rebuild meets the
    18-neighbour cell, the system widens to 32 and the run continues to a Delaunay state (the
    strong forces on the ringed cell soon pull its coordination back down)."""
    from cellgpu_b200 import VoronoiBatch
    pos, box = _flower()
    N = len(pos)
    p1 = pos.copy()
    p1[0] = [1.3, 1.7]
    nn1, nbr1 = oracle.periodic_delaunay(p1, box, 16)
    b = VoronoiBatch([N], [box])
    b.set_positions(pos)
    b.set_directors(np.zeros(N))
    b.set_motility(np.tile([0.02, 1.0], (N, 1)))
    b.set_preferences(np.tile([1.0, 3.8], (N, 1)))
    b.set_topology(nn1, nbr1)
    b.spp_run(3, dt=0.01)
    assert b._lib.cg_neighbor_capacity(b.handle) == 32
    b.enforce_topology()
    nn, nbr = b.topology()
    onn, onbr = oracle.periodic_delaunay(b.positions(), box, 32)
    assert np.array_equal(_canon(nn, nbr), _canon(onn, onbr))


def test_raw_triangulation_reports_capacity_instead_of_widening(cglib, torch):
    """cg_voronoi_triangulate writes into the caller's rows of capacity K. A cell with 18 Delaunay
    neighbours and K = 16 must give CG_ERR_CAPACITY (the internal system may widen to 32, but the
    caller's buffers cannot hold those rows), and K = 32 must succeed."""
    pos, box = _flower()
    N = len(pos)
    dev = torch.device("cuda:0")
    tpos = torch.tensor(pos, device=dev)
    p = lambda t: C.c_void_p(t.data_ptr())
    for K, want in ((16, -3), (32, 0)):
        nn = torch.full((N,), -1, dtype=torch.int32, device=dev)
        nbr = torch.full((N, K), -1, dtype=torch.int32, device=dev)
        rc = cglib.cg_voronoi_triangulate(p(tpos), N, box[0], box[1], K, p(nn), p(nbr), None)
        torch.cuda.synchronize()
        assert rc == want, (K, rc, cglib.cg_last_error_string())
        if rc == 0:
            assert int(nn[0].item()) == 18
            assert int(nn.sum().item()) == 6 * N
