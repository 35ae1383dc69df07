"""Degenerate and near-degenerate point sets: every cell must reach the same in-circle decision for
the same four points, so the rows stay mutually consistent.

* A perfect square lattice makes every unit square's four corners exactly cocircular; the tie is
  broken by simulation of simplicity on global indices (indices permuted at random, so ties meet
  every index pattern).
* Offsets and spacings that are not representable make the squares cocircular only up to the
  rounding of the relative positions, which differs from cell to cell (and across the periodic
  wrap); the decision is taken in one canonical frame for all cells.
* FIRE in the fluid regime (p0 = 3.95) drives Voronoi edges towards zero length, i.e. quadruples of
  cells towards cocircularity.
Checks: the triangulation is built (the library validates triangle consistency and sum z = 6 N),
the rows are mutually consistent here too, the local Delaunay test passes on the result (nothing
to repair), and stepping from the degenerate state keeps the topology equal to a fresh global
triangulation.
"""
import numpy as np
import pytest

from helpers import canonical

pytestmark = pytest.mark.gpu


def _square_lattice(n, spacing, offset, seed):
    g = (np.arange(n) + offset) * spacing
    pts = np.array([(x, y) for y in g for x in g])
    perm = np.random.default_rng(seed).permutation(n * n)
    return pts[perm], (n * spacing, n * spacing)


def _rows_consistent(nn, nbr):
    for c in range(len(nn)):
        z = nn[c]
        for k in range(z):
            u, v = nbr[c, k], nbr[c, (k + 1) % z]
            ru, rv = list(nbr[u, :nn[u]]), list(nbr[v, :nn[v]])
            if not any(ru[i] == v and ru[(i + 1) % len(ru)] == c for i in range(len(ru))):
                return False
            if not any(rv[i] == c and rv[(i + 1) % len(rv)] == u for i in range(len(rv))):
                return False
    return True


def _batch(pos, box, p0=3.8):
    from cellgpu_b200 import VoronoiBatch
    b = VoronoiBatch([len(pos)], [box])
    b.set_positions(pos)
    b.set_preferences(np.tile([1.0, p0], (len(pos), 1)))
    return b


@pytest.mark.parametrize("spacing,offset", [(1.0, 0.5), (1.0, 0.1), (1.0, 0.0), (0.7, 0.3), (1.1, 0.05)])
def test_square_lattice_triangulation_is_consistent(cglib, oracle, spacing, offset):
    n = 24
    pos, box = _square_lattice(n, spacing, offset, seed=3)
    b = _batch(pos, box)
    b.triangulate()
    nn, nbr = b.topology()
    assert nn.sum() == 6 * n * n
    assert _rows_consistent(nn, nbr)
    before = b.counters()
    b.enforce_topology()  # the local test agrees with the global star: nothing to repair
    after = b.counters()
    assert after["rows_changed"] == before["rows_changed"]
    assert after["global_rebuilds"] == before["global_rebuilds"]
    b.compute_forces()
    np.testing.assert_allclose(b.area_perimeter()[:, 0], spacing ** 2, rtol=1e-12)
    # The energy is not differentiable here (zero-length Voronoi edges, whose unit vector the
    # reference clamps to zero), so the force depends on the chosen diagonals; on the same rows it
    # is the reference's formula. With a spacing that is not representable the edges are rounding
    # noise long instead of zero and their unit vectors are noise: no force comparison then.
    if spacing != 1.0:
        return
    AP = oracle.voronoi_geometry(pos, box, nn, nbr)
    F = oracle.voronoi_forces(pos, box, nn, nbr, AP, np.tile([1.0, 3.8], (n * n, 1)))
    assert np.abs(b.forces() - F).max() < 1e-10


def test_stepping_from_a_square_lattice(cglib):
    n = 20
    pos, box = _square_lattice(n, 1.0, 0.1, seed=4)
    b = _batch(pos, box)
    rng = np.random.default_rng(5)
    b.set_directors(rng.uniform(0, 2 * np.pi, n * n))
    b.set_motility(np.tile([0.02, 1.0], (n * n, 1)))
    b.triangulate()
    b.spp_run(30, dt=0.01)
    b.enforce_topology()
    nn, nbr = b.topology()
    fresh = _batch(b.positions(), box)
    fresh.triangulate()
    fnn, fnbr = fresh.topology()
    assert np.array_equal(canonical(nn, nbr), canonical(fnn, fnbr))


def test_fluid_fire_minimum_stays_consistent(cglib):
    """FIRE far into the fluid regime, then a global triangulation and the local test of the
    result; the state is checked at two points of the minimisation."""
    from cellgpu_b200 import FireParams
    N = 900
    L = np.sqrt(N)
    pos = np.random.default_rng(6).random((N, 2)) * L
    b = _batch(pos, (L, L), p0=3.95)
    b.triangulate()
    for its in (3000, 12000):
        b.fire_minimize(FireParams.defaults(force_cutoff=1e-14, max_iterations=its))
        b.triangulate()
        nn, nbr = b.topology()
        assert nn.sum() == 6 * N and _rows_consistent(nn, nbr)
        before = b.counters()
        b.enforce_topology()
        assert b.counters()["rows_changed"] == before["rows_changed"]
