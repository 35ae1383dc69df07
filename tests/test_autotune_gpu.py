"""Autotuner: it picks among the runtime launch choices without changing results (forces within
1e-12 of max(|F|, RMS F), Delaunay rows bit-exact) and the batch keeps stepping with its choice."""
import numpy as np
import pytest

from helpers import canonical, force_error, monolayer

pytestmark = pytest.mark.gpu


def test_autotune_keeps_results(cglib):
    from cellgpu_b200 import VoronoiBatch
    (p1, b1), (p2, b2) = monolayer(3000, 71), monolayer(900, 72)
    N = [len(p1), len(p2)]
    b = VoronoiBatch(N, [b1, b2])
    b.set_positions(np.concatenate([p1, p2]))
    b.triangulate()
    b.compute_forces()
    F0 = b.forces()
    nn0, nbr0 = b.topology()
    r = b.autotune()
    assert r["force_shape"] in ("2 warps/block", "4 warps/block") and r["bin_side"] in (0.8, 1.0, 1.25)
    assert all(t > 0 for t in r["force_pass_ms"] + r["triangulation_ms"])
    b.triangulate()  # with the chosen bin side
    nn, nbr = b.topology()
    assert np.array_equal(canonical(nn, nbr), canonical(nn0, nbr0))
    b.compute_forces()
    assert force_error(b.forces(), F0) < 1e-12
    b.set_motility(np.tile([0.1, 1.0], (sum(N), 1)))
    b.spp_run(30, dt=0.01)
    b.enforce_topology()
    assert np.isfinite(b.energies()).all()
