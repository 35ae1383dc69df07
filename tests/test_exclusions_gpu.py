"""Particle exclusions (voronoiModelBase::setExclusions; the force summation with exclusions,
src/models/voronoiQuadraticEnergy.cpp:119-135,368-377) on the GPU, through the C ABI, against the
reference's own outputs (tests/golden/exclusions_N400_s9.npz) and the oracle.

Tolerances (written here): forces and external forces force_error <= 1e-10 (FP64, summation order
only); excluded cells' forces exactly 0; positions after 5 supplied-noise SPP steps within 1e-9;
topology bit-exact (canonical rotation).
"""
import glob
import os

import numpy as np
import pytest

from helpers import canonical, force_error

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def g():
    return dict(np.load(sorted(glob.glob(os.path.join(GOLD, "exclusions_N*.npz")))[0]))


def _system(g):
    from cellgpu_b200 import VoronoiBatch
    N, box = int(g["N"]), tuple(g["box"])
    b = VoronoiBatch([N], [box])
    b.set_positions(g["pos"])
    b.set_directors(g["theta"])
    b.set_motility(np.tile([float(g["v0"]), float(g["Dr"])], (N, 1)))
    b.set_preferences(np.tile([1.0, 3.8], (N, 1)))
    b.triangulate()
    b.set_exclusions(g["exes"])
    return b


def test_exclusion_forces_match_reference(cglib, g):
    b = _system(g)
    ex = g["exes"] != 0
    b.compute_forces()
    F, ext = b.forces(), b.external_forces()
    assert np.all(F[ex] == 0.0)
    assert np.all(ext[~ex] == 0.0)
    assert force_error(F, g["F0"]) < 1e-10
    assert force_error(ext[ex], g["ext0"][ex]) < 1e-10


def test_exclusion_spp_run_matches_reference(cglib, oracle, g):
    import torch
    b = _system(g)
    ex = g["exes"] != 0
    N, box = int(g["N"]), tuple(g["box"])
    noise = g["noise"]
    b.spp_run(int(g["steps"]), dt=float(g["dt"]), mu=1.0, noise=torch.tensor(noise, device="cuda:0"))
    # the last force evaluation of the run, against the oracle's
    pos = g["pos"].copy()
    theta = g["theta"].copy()
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    mot = np.tile([float(g["v0"]), float(g["Dr"])], (N, 1))
    mot[ex] = 0.0
    pref = np.tile([1.0, 3.8], (N, 1))
    F, ext, _ = oracle.voronoi_spp_run_exclusions(pos, box, nn, nbr, theta, mot, pref, noise, ex, dt=float(g["dt"]))
    assert force_error(b.forces(), F) < 1e-10
    assert force_error(b.external_forces()[ex], ext[ex]) < 1e-10
    # the state after the run, against the reference's
    assert np.abs(b.positions() - g["pos1"]).max() < 1e-9
    assert np.abs(b.positions()[ex] - g["pos"][ex]).max() < 1e-12  # excluded cells do not move
    b.enforce_topology()
    bnn, bnbr = b.topology()
    assert np.array_equal(canonical(bnn, bnbr), canonical(g["nn1"], g["nbr1"]))
    b.compute_forces()
    assert force_error(b.forces(), g["F1"]) < 1e-9
    assert force_error(b.external_forces()[ex], g["ext1"][ex]) < 1e-9


def test_exclusions_follow_sorting_and_snapshots(cglib, g):
    """The flags move with their cells under spatial sorting and survive a snapshot; clearing them
    restores plain forces."""
    from cellgpu_b200 import models
    b = _system(g)
    ex = g["exes"] != 0
    b.spatial_sort()
    tags = b.tags()
    b.compute_forces()
    F = b.forces()
    assert np.all(F[ex[tags]] == 0.0) and np.any(F[~ex[tags]] != 0.0)
    r = models.restore(b.snapshot())
    r.compute_forces()
    assert np.all(r.forces()[ex[tags]] == 0.0)
    assert force_error(r.external_forces(), b.external_forces()) < 1e-12
    b.set_exclusions(None)
    b.compute_forces()
    assert np.all(b.external_forces() == 0.0)
    assert np.all(np.linalg.norm(b.forces()[ex[tags]], axis=1) > 0.0)
