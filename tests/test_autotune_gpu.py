"""Autotuner: it picks among the runtime launch choices without changing results (forces within
1e-12 of max(|F|, RMS F), Delaunay rows bit-exact) and the batch keeps stepping with its choice."""
import numpy as np
import pytest

from helpers import canonical, force_error, jittered_lattice, monolayer

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
    assert r["force_shape"] in ("2 warps/block", "4 warps/block", "thread per cell")
    assert r["bin_side"] in (0.8, 1.0, 1.25)
    assert all(t > 0 for t in r["force_pass_ms"] + r["triangulation_ms"])  # FP64: all three shapes
    b.triangulate()  # with the chosen bin side
    nn, nbr = b.topology()
    assert np.array_equal(canonical(nn, nbr), canonical(nn0, nbr0))
    b.compute_forces()
    assert force_error(b.forces(), F0) < 1e-12
    b.set_motility(np.tile([0.1, 1.0], (sum(N), 1)))
    b.spp_run(30, dt=0.01)
    b.enforce_topology()
    assert np.isfinite(b.energies()).all()


def test_autotune_repair_steps_are_real_steps(cglib):
    """cg_autotune_repair runs 12 x steps real SPP steps while it times the repair grids: in the
    deterministic mode the tuned system is bit-identical to one that ran as many steps with the
    default grids, and stays so when both continue (the grids change no result)."""
    from cellgpu_b200 import VoronoiBatch
    pos, box = jittered_lattice(30, 34, 0.3, 73)
    N = len(pos)

    def make():
        b = VoronoiBatch([N], [box])
        b.set_positions(pos)
        b.set_motility(np.tile([0.5, 1.0], (N, 1)))
        b.set_instance_seeds([5])
        b.set_deterministic(True)
        b.triangulate()
        return b

    a, b = make(), make()
    r = a.autotune_repair(steps=4, dt=0.02)
    assert r["star_grid"] in (148 * 5, 148 * 2) and r["commit_grid"] in (148 * 4, 148 * 8, 148 * 16)
    assert all(t > 0 for t in r["ms_per_step"])
    b.spp_run(48, dt=0.02)
    assert a.counters()["rows_changed"] > 0
    assert np.array_equal(a.positions(), b.positions())
    a.spp_run(20, dt=0.02)
    b.spp_run(20, dt=0.02)
    assert np.array_equal(a.positions(), b.positions())
    assert np.array_equal(a.forces(), b.forces())
