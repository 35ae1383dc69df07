"""Spatial re-sorting of a Voronoi batch: state and topology move with the cells (forces, areas and
Delaunay rows are the same up to the permutation; tolerance 1e-12 on forces), cells stay within
their instance, neighbours end up closer in memory, and the batch keeps stepping."""
import numpy as np
import pytest

from helpers import canonical, force_error, monolayer

pytestmark = pytest.mark.gpu


def test_spatial_sort_permutes_state_and_topology(cglib):
    from cellgpu_b200 import VoronoiBatch
    (p1, b1), (p2, b2) = monolayer(1500, 61), monolayer(700, 62)
    N = [len(p1), len(p2)]
    b = VoronoiBatch(N, [b1, b2])
    pos0 = np.concatenate([p1, p2])
    b.set_positions(pos0)
    b.set_preferences(np.column_stack([np.ones(sum(N)), np.linspace(3.7, 3.9, sum(N))]))
    b.triangulate()
    b.compute_forces()
    F0, AP0 = b.forces(), b.area_perimeter()
    nn0, nbr0 = b.topology()
    b.spatial_sort()
    tags = b.tags()
    assert sorted(tags[:N[0]]) == list(range(N[0]))  # cells stay in their instance
    assert sorted(tags[N[0]:]) == list(range(N[0], sum(N)))
    assert np.array_equal(b.positions(), pos0[tags])
    assert np.array_equal(b.area_perimeter(), AP0[tags])
    # rows: relabelled back to tags they equal the original rows
    nn, nbr = b.topology()
    back = np.where(nbr >= 0, tags[np.maximum(nbr, 0)], -1)
    inv = np.empty_like(tags)
    inv[tags] = np.arange(len(tags))
    assert np.array_equal(canonical(nn[inv], back[inv]), canonical(nn0, nbr0))
    b.compute_forces()
    assert force_error(b.forces(), F0[tags]) < 1e-12
    # locality: consecutive cells are much closer after sorting
    d_before = np.linalg.norm(np.diff(pos0[:N[0]], axis=0), axis=1).mean()
    d_after = np.linalg.norm(np.diff(b.positions()[:N[0]], axis=0), axis=1).mean()
    assert d_after < 0.25 * d_before
    b.set_motility(np.tile([0.1, 1.0], (sum(N), 1)))
    b.spp_run(20, dt=0.01)
    b.enforce_topology()
    assert np.isfinite(b.energies()).all()


def test_sorted_trajectory_follows_the_oracle(cglib, oracle):
    """Sorting changes the memory order only: a sorted system run with the supplied noise of each cell
    (noise[:, tags]) follows the oracle's trajectory of the unsorted input, mapped back through the
    tags. Free run of 30 SPP steps from a jittered lattice; positions and directors within 1e-9,
    topology bit-exact, forces force_error <= 1e-8 (the free-run tolerances of the unsorted runs)."""
    import torch

    from cellgpu_b200 import VoronoiBatch
    from helpers import jittered_lattice
    pos, box = jittered_lattice(24, 28, 0.25, 63)
    N, steps, dt = len(pos), 30, 0.01
    rng = np.random.default_rng(64)
    theta = rng.uniform(0, 2 * np.pi, N)
    mot = np.tile([0.3, 1.0], (N, 1))
    pref = np.tile([1.0, 3.8], (N, 1))
    noise = rng.normal(size=(steps, N))
    b = VoronoiBatch([N], [box])
    b.set_positions(pos)
    b.set_directors(theta)
    b.set_motility(mot)
    b.set_preferences(pref)
    b.triangulate()
    b.spatial_sort()
    tags = b.tags()
    assert not np.array_equal(tags, np.arange(N))
    b.spp_run(steps, dt=dt, mu=1.0, noise=torch.tensor(noise[:, tags], device="cuda:0"))
    b.enforce_topology()
    onn, onbr = oracle.periodic_delaunay(pos, box, 16)
    opos, oth = pos.copy(), theta.copy()
    F, _ = oracle.voronoi_spp_run(opos, box, onn, onbr, oth, mot, pref, noise, dt=dt)
    inv = np.empty_like(tags)
    inv[tags] = np.arange(N)
    P, TH = b.positions()[inv], b.directors()[inv]
    d = P - opos
    d -= np.asarray(box) * np.round(d / np.asarray(box))  # a cell at the box edge may wrap either way
    assert np.abs(d).max() < 1e-9
    assert np.abs(np.angle(np.exp(1j * (TH - oth)))).max() < 1e-9
    nn, nbr = b.topology()
    back = np.where(nbr >= 0, tags[np.maximum(nbr, 0)], -1)
    assert np.array_equal(canonical(nn[inv], back[inv]), canonical(onn, onbr))
    assert force_error(b.forces()[inv], F) < 1e-8
