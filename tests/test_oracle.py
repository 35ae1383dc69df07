"""CPU tests of the oracle itself: exact predicates, Delaunay invariants, analytic known answers,
and finite-difference checks of the reference force formulas it restates."""
import numpy as np
import pytest

from helpers import monolayer


def _hex_lattice(nx=12, ny=14, shift=(0.1, 0.05)):
    a = 1.0
    pts = []
    for j in range(ny):
        for i in range(nx):
            pts.append(((i + 0.5 * (j % 2)) * a + shift[0], j * a * np.sqrt(3) / 2 + shift[1]))
    pts = np.array(pts)
    s = np.sqrt(2 / np.sqrt(3))  # unit-area hexagons
    return pts * s, (nx * a * s, ny * a * np.sqrt(3) / 2 * s)


def test_star_gift_wrap_matches_bruteforce(oracle):
    rng = np.random.default_rng(3)
    for _ in range(50):
        m = rng.integers(8, 40)
        rel = rng.normal(size=(m, 2))
        a = oracle.local_star(rel)
        b = oracle.local_star(rel, brute=True)
        assert np.array_equal(a, b)


def test_exact_predicates_on_degenerate_inputs(oracle):
    # cocircular points on the unit circle through the origin's circle: the star must still close
    t = np.linspace(0, 2 * np.pi, 13)[:-1]
    rel = np.stack([np.cos(t), np.sin(t)], axis=1)
    star = oracle.local_star(rel)
    assert len(star) == 12


@pytest.mark.parametrize("N,seed", [(64, 0), (300, 1), (1000, 2)])
def test_delaunay_euler_invariants(oracle, N, seed):
    pos, box = monolayer(N, seed)
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    assert nn.sum() == 6 * N  # src/models/voronoiModelBase.cpp:263,342
    # symmetry of the adjacency
    for i in range(N):
        for j in nbr[i, : nn[i]]:
            assert i in nbr[j, : nn[j]]
    assert oracle.topology_mismatch(pos, box, nn, nbr) == 0


def test_hexagonal_known_answer(oracle):
    pts, box = _hex_lattice()
    nn, nbr = oracle.periodic_delaunay(pts, box, 16)
    assert set(nn.tolist()) == {6}
    AP = oracle.voronoi_geometry(pts, box, nn, nbr)
    np.testing.assert_allclose(AP[:, 0], 1.0, rtol=1e-12)
    np.testing.assert_allclose(AP[:, 1], np.sqrt(8 * np.sqrt(3)), rtol=1e-12)
    F = oracle.voronoi_forces(pts, box, nn, nbr, AP, np.tile([1.0, 3.8], (len(pts), 1)))
    assert np.abs(F).max() < 1e-12
    E = oracle.voronoi_energy(AP, np.tile([1.0, 3.8], (len(pts), 1)))
    assert abs(E - len(pts) * (np.sqrt(8 * np.sqrt(3)) - 3.8) ** 2) < 1e-10


def test_area_sums_to_box(oracle):
    pos, box = monolayer(500, 7)
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    AP = oracle.voronoi_geometry(pos, box, nn, nbr)
    assert abs(AP[:, 0].sum() - box[0] * box[1]) < 1e-9


def test_voronoi_forces_finite_difference(oracle):
    pos, box = monolayer(200, 11)
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    pref = np.tile([1.0, 3.8], (200, 1))
    AP = oracle.voronoi_geometry(pos, box, nn, nbr)
    F = oracle.voronoi_forces(pos, box, nn, nbr, AP, pref)
    assert np.abs(F.sum(axis=0)).max() < 1e-9  # Newton III
    h = 1e-6
    for i in (0, 17, 123):
        for d in range(2):
            p = pos.copy()
            p[i, d] += h
            Ep = oracle.voronoi_energy(oracle.voronoi_geometry(p, box, nn, nbr), pref)
            p[i, d] -= 2 * h
            Em = oracle.voronoi_energy(oracle.voronoi_geometry(p, box, nn, nbr), pref)
            assert abs(-(Ep - Em) / (2 * h) - F[i, d]) < 1e-5 * max(1.0, abs(F[i, d]))


def test_spp_run_keeps_delaunay(oracle):
    N = 300
    pos, box = monolayer(N, 5)
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    rng = np.random.default_rng(9)
    theta = rng.uniform(0, 2 * np.pi, N)
    mot = np.tile([0.05, 1.0], (N, 1))
    pref = np.tile([1.0, 3.8], (N, 1))
    noise = rng.normal(size=(20, N))
    F, AP = oracle.voronoi_spp_run(pos, box, nn, nbr, theta, mot, pref, noise)
    assert nn.sum() == 6 * N
    assert oracle.topology_mismatch(pos, box, nn, nbr) == 0
    assert np.all((pos >= 0) & (pos < box[0]))
