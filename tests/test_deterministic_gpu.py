"""Deterministic force sums (cg_set_deterministic; Simulation.setReproducible maps to it).

With the mode on, forces are summed in 64-bit fixed point with integer atomics, which commute
exactly, so:
  * two runs from the same inputs are bit-identical (positions, directors, forces, topology), for
    the Voronoi model in FP64 and mixed precision and for the vertex model with T1 flips;
  * forces keep parity with the oracle (force_error <= 1e-10, the FP64 tolerance of the suite);
  * a repair's retraction cancels the force pass's addition exactly, so the forces at the end of a
    step that repaired rows equal, bit for bit, a fresh force pass on the repaired rows.
"""
import numpy as np
import pytest

from helpers import force_error, jittered_lattice, monolayer

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-10


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def _spp_batch(pos, box, seed, precision=0, v0=0.1, det=True):
    from cellgpu_b200 import VoronoiBatch
    N = len(pos)
    rng = np.random.default_rng(seed)
    b = VoronoiBatch([N], [box], precision=precision)
    b.set_positions(pos)
    b.set_directors(rng.uniform(0, 2 * np.pi, N))
    b.set_motility(np.tile([v0, 1.0], (N, 1)))
    b.set_preferences(np.tile([1.0, 3.8], (N, 1)))
    b.set_seed(seed)
    b.set_deterministic(det)
    b.triangulate()
    return b


@pytest.mark.parametrize("precision", [0, 1])
def test_voronoi_reruns_bit_identical(cglib, precision):
    pos, box = monolayer(4096, 21)
    runs = []
    for _ in range(2):
        b = _spp_batch(pos, box, 22, precision=precision)
        assert b.deterministic
        b.spp_run(200, dt=0.01, mu=1.0)  # device noise, graph steps with repair rounds
        runs.append((b.positions(), b.directors(), b.forces(), b.topology(), b.counters()["rows_changed"],
                     b.energies()))
        b.close()
    (p0, t0, f0, (nn0, nb0), rc0, e0), (p1, t1, f1, (nn1, nb1), rc1, e1) = runs
    assert rc0 > 0 and rc0 == rc1
    assert np.array_equal(p0, p1) and np.array_equal(t0, t1) and np.array_equal(f0, f1)
    assert np.array_equal(nn0, nn1) and np.array_equal(nb0, nb1)
    assert np.array_equal(e0, e1)


def test_enqueue_host_energies_bit_identical(cglib, torch):
    """The host-buffer step's in-graph energy reduction (into page-locked memory) in the
    deterministic mode: reruns give the same bits, and they agree with cg_get_energies."""
    import ctypes as C
    from cellgpu_b200 import VoronoiBatch
    (p1, b1), (p2, b2) = jittered_lattice(40, 46, 0.25, 31), jittered_lattice(30, 36, 0.25, 32)
    Ns = [len(p1), len(p2)]
    N = sum(Ns)
    rng = np.random.default_rng(33)
    theta = rng.uniform(0, 2 * np.pi, N)
    noise = torch.from_numpy(rng.normal(size=(6, N))).pin_memory()
    out = []
    for _ in range(2):
        b = VoronoiBatch(Ns, [b1, b2])
        b.set_positions(np.concatenate([p1, p2]))
        b.set_directors(theta)
        b.set_motility(np.tile([0.3, 1.0], (N, 1)))
        b.set_preferences(np.column_stack([np.ones(N), np.linspace(3.7, 3.9, N)]))
        b.set_deterministic(True)
        b.triangulate()
        pinned = torch.zeros((6, 2), dtype=torch.float64).pin_memory()
        for k in range(6):
            assert b._lib.cg_spp_enqueue_host(b.handle, C.c_void_p(noise[k].data_ptr()), 0.02, 1.0,
                                              C.c_void_p(pinned[k].data_ptr())) == 0
            assert b._lib.cg_poll(b.handle, None, None, 1) == 0
        np.testing.assert_allclose(pinned[5].numpy(), b.energies(), rtol=1e-14)
        out.append(pinned.numpy().copy())
        b.close()
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("N,seed", [(300, 5), (2000, 6)])
def test_deterministic_forces_match_oracle(cglib, oracle, N, seed):
    pos, box = monolayer(N, seed)
    b = _spp_batch(pos, box, seed)
    b.compute_forces()
    nn, nbr = b.topology()
    pref = np.tile([1.0, 3.8], (N, 1))
    AP = oracle.voronoi_geometry(pos, box, nn, nbr)
    F = oracle.voronoi_forces(pos, box, nn, nbr, AP, pref)
    assert force_error(b.forces(), F) < TOL_F64
    b.set_deterministic(False)  # the atomic sums agree to rounding
    b.compute_forces()
    assert force_error(b.forces(), F) < TOL_F64


def test_spp_steps_match_oracle_deterministic(cglib, oracle, torch):
    """Free-running steps with supplied noise, the deterministic mode on: each step's force pass
    meets the rows its previous move left stale and repairs them on the device; positions, forces
    and topology follow the oracle's steps."""
    pos, box = jittered_lattice(32, 36, 0.25, 12)
    N = len(pos)
    b = _spp_batch(pos, box, 112, v0=1.0)
    theta = b.directors()
    mot = np.tile([1.0, 1.0], (N, 1))
    pref = np.tile([1.0, 3.8], (N, 1))
    rng = np.random.default_rng(13)
    onn, onbr = oracle.periodic_delaunay(pos, box, 16)
    opos, oth = pos.copy(), theta.copy()
    for s in range(8):
        noise = rng.normal(size=(1, N))
        b.spp_run(1, dt=0.05, mu=1.0, noise=torch.tensor(noise, device="cuda:0"))
        F, _ = oracle.voronoi_spp_run(opos, box, onn, onbr, oth, mot, pref, noise, dt=0.05)
        assert np.abs(b.positions() - opos).max() < 1e-10
        assert force_error(b.forces(), F) < 1e-9
    assert b.counters()["rows_changed"] > 0


def test_repair_retraction_is_exact(cglib, torch):
    """Rows of a slightly earlier state, repaired inside a step that does not move (dt = 0): the
    step's forces (force pass on the stale rows, then retract/add of every changed row) equal a
    fresh force pass on the repaired rows bit for bit."""
    pos0, box = monolayer(4096, 31)
    b = _spp_batch(pos0, box, 31)
    nn0, nbr0 = b.topology()
    rng = np.random.default_rng(32)
    pos1 = (pos0 + rng.normal(scale=0.01, size=pos0.shape)) % box[0]
    b.set_positions(pos1)
    b.set_topology(nn0, nbr0)
    rc = b.counters()["rows_changed"]
    b.spp_run(1, dt=0.0, mu=1.0, noise=torch.zeros((1, len(pos0)), dtype=torch.float64, device="cuda:0"))
    assert b.counters()["rows_changed"] > rc
    assert np.array_equal(b.positions(), pos1)
    F_step = b.forces()
    b.compute_forces()
    assert np.array_equal(F_step, b.forces())


def test_vertex_reruns_bit_identical(cglib, torch):
    from cellgpu_b200 import VertexBatch
    pos, box = jittered_lattice(16, 18, 0.3, 3)
    Nc = len(pos)
    runs = []
    for _ in range(2):
        b = VertexBatch([Nc], [box], vmax=16)
        b.from_cells(pos)
        b.set_preferences(np.tile([1.0, 3.85], (Nc, 1)))
        b.set_t1_threshold(0.08)
        b.set_seed(4)
        b.set_deterministic(True)
        b.brownian_run(40, dt=0.01, mu=1.0, T=0.02)
        runs.append((b.positions(), b.forces(), b.vertex_topology(), b.counters()["t1_flips"]))
        b.close()
    (p0, f0, top0, n0), (p1, f1, top1, n1) = runs
    assert n0 > 10 and n0 == n1
    assert np.array_equal(p0, p1) and np.array_equal(f0, f1)
    for a, c in zip(top0, top1):
        assert np.array_equal(a, c)


def test_vertex_deterministic_forces_agree(cglib):
    from cellgpu_b200 import VertexBatch
    pos, box = jittered_lattice(16, 18, 0.3, 3)
    Nc = len(pos)
    b = VertexBatch([Nc], [box], vmax=16)
    b.from_cells(pos)
    b.set_preferences(np.tile([1.0, 3.85], (Nc, 1)))
    b.compute_forces()
    F_atomic = b.forces()
    b.set_deterministic(True)
    b.compute_forces()
    assert force_error(b.forces(), F_atomic) < 1e-13


def test_set_reproducible_turns_deterministic_on(cglib):
    from cellgpu_b200.models import Simulation, VoronoiQuadraticEnergy, selfPropelledParticleDynamics
    spv = VoronoiQuadraticEnergy(300, 1.0, 3.8, True)
    sim = Simulation()
    sim.setConfiguration(spv)
    sim.addUpdater(selfPropelledParticleDynamics(300), spv)
    assert not spv.batch.deterministic
    sim.setReproducible(True)
    assert spv.batch.deterministic
    sim.setReproducible(False)
    assert not spv.batch.deterministic


def _fire_batch(Ns, seed):
    from cellgpu_b200 import VoronoiBatch
    rng = np.random.default_rng(seed)
    boxes = [(np.sqrt(n), np.sqrt(n)) for n in Ns]
    pos = np.concatenate([rng.random((n, 2)) * np.sqrt(n) for n in Ns])
    b = VoronoiBatch(Ns, boxes)
    b.set_positions(pos)
    b.set_deterministic(True)
    b.triangulate()
    return b


def test_fire_batch_reruns_bit_identical(cglib):
    """FIRE on a batch whose instance boundaries fall inside 256-dof blocks (and one instance spanning
    whole blocks): the power and norm sums are taken in a fixed order, so reruns are bit-identical."""
    from cellgpu_b200 import FireParams
    Ns = [300, 1000, 257, 4096, 70]
    runs = []
    for _ in range(2):
        b = _fire_batch(Ns, 41)
        b.fire_minimize(FireParams.defaults(force_cutoff=1e-10, max_iterations=3000))
        it, fmax, fnorm = b.fire_state()
        runs.append((b.positions(), it, fmax, fnorm, b.energies()))
        b.close()
    for x, y in zip(*runs):
        assert np.array_equal(x, y)
    assert len(set(runs[0][1].tolist())) > 1


def test_fire_deterministic_reaches_same_minimum(cglib):
    """The fixed-order sums change only rounding: each instance reaches the threshold and the same
    energy as with atomic sums."""
    from cellgpu_b200 import FireParams
    Ns = [120, 300, 64]
    b = _fire_batch(Ns, 4)
    b.fire_minimize(FireParams.defaults(force_cutoff=1e-10, max_iterations=4000))
    _, fmax, _ = b.fire_state()
    assert np.all(fmax <= 1e-10)
    E_det = b.energies()
    a = _fire_batch(Ns, 4)
    a.set_deterministic(False)
    a.fire_minimize(FireParams.defaults(force_cutoff=1e-10, max_iterations=4000))
    E_atomic = a.energies()
    assert np.all(np.abs(E_det - E_atomic) < 1e-8 * np.maximum(1.0, E_atomic))


def test_fire_batch_equals_singles_bit_for_bit(cglib):
    """In the deterministic mode a FIRE minimisation does not depend on where the instance sits in a
    batch: the power and norm sums run over chunks counted from the instance's first dof, so an
    instance gets the same iterations, positions and stopping point alone and at any offset."""
    from cellgpu_b200 import FireParams, VoronoiBatch
    Ns = [300, 1000, 257]
    rng = np.random.default_rng(43)
    poss = [rng.random((n, 2)) * np.sqrt(n) for n in Ns]

    def run(sel):
        b = VoronoiBatch([Ns[i] for i in sel], [(np.sqrt(Ns[i]), np.sqrt(Ns[i])) for i in sel])
        b.set_positions(np.concatenate([poss[i] for i in sel]))
        b.set_deterministic(True)
        b.triangulate()
        b.fire_minimize(FireParams.defaults(force_cutoff=1e-10, max_iterations=3000))
        it, fmax, _ = b.fire_state()
        out = b.positions(), it, fmax
        b.close()
        return out

    order = [2, 0, 1]
    P, it, fmax = run(order)
    off = 0
    for j, i in enumerate(order):
        Ps, its, fms = run([i])
        assert np.array_equal(P[off:off + Ns[i]], Ps)
        assert it[j] == its[0] and fmax[j] == fms[0]
        off += Ns[i]


def test_fire_vertex_reruns_bit_identical(cglib):
    from cellgpu_b200 import FireParams, VertexBatch
    pos, box = jittered_lattice(16, 18, 0.3, 3)
    Nc = len(pos)
    runs = []
    for _ in range(2):
        b = VertexBatch([Nc], [box], vmax=16)
        b.from_cells(pos)
        b.set_preferences(np.tile([1.0, 3.85], (Nc, 1)))
        b.set_deterministic(True)
        b.fire_minimize(FireParams.defaults(force_cutoff=1e-10, max_iterations=2000))
        it, fmax, _ = b.fire_state()
        runs.append((b.positions(), it, fmax, b.energies()))
        b.close()
    for x, y in zip(*runs):
        assert np.array_equal(x, y)


def _typed_batch(pos, box, mode, det, K=16):
    from cellgpu_b200 import VoronoiBatch
    N = len(pos)
    rng = np.random.default_rng(51)
    b = VoronoiBatch([N], [box], K=K)
    b.set_positions(pos)
    b.set_directors(rng.uniform(0, 2 * np.pi, N))
    b.set_motility(np.tile([0.2, 1.0], (N, 1)))
    b.set_preferences(np.tile([1.0, 3.8], (N, 1)))
    b.set_seed(52)
    if mode is not None:
        b.set_cell_types(rng.integers(0, 3, N))
        if mode == "simple":
            b.set_tension(0.2)
        else:
            b.set_tension_matrix(np.array([[0.0, 0.1, 0.3], [0.1, 0.0, 0.2], [0.3, 0.2, 0.0]]))
    b.set_deterministic(det)
    b.triangulate()
    return b


@pytest.mark.parametrize("mode", ["simple", "matrix"])
def test_tension_deterministic(cglib, mode):
    """Line tension (one gamma, or a matrix over three types) with fixed-point sums: forces agree with
    the atomic sums to rounding, and reruns are bit-identical."""
    pos, box = monolayer(2000, 53)
    a = _typed_batch(pos, box, mode, False)
    a.compute_forces()
    runs = []
    for _ in range(2):
        b = _typed_batch(pos, box, mode, True)
        b.compute_forces()
        assert force_error(b.forces(), a.forces()) < 1e-13
        b.spp_run(100, dt=0.01)
        runs.append((b.positions(), b.forces(), b.energies()))
        b.close()
    for x, y in zip(*runs):
        assert np.array_equal(x, y)


def test_wide_rows_deterministic(cglib):
    """The 32-slot form of the force pass with fixed-point sums: it agrees with the 16-slot form, and
    its reruns are bit-identical."""
    pos, box = jittered_lattice(40, 46, 0.25, 41)
    narrow = _typed_batch(pos, box, None, True, K=16)
    narrow.compute_forces()
    runs = []
    for _ in range(2):
        b = _typed_batch(pos, box, None, True, K=32)
        b.compute_forces()
        assert force_error(b.forces(), narrow.forces()) < 1e-13
        b.spp_run(30, dt=0.02)
        runs.append((b.positions(), b.forces(), b.counters()["rows_changed"]))
        b.close()
    for x, y in zip(*runs):
        assert np.array_equal(x, y)
    assert runs[0][2] > 0


def test_resume_is_bit_exact(cglib):
    """A snapshot records the deterministic mode and the restored system switches it on: the run
    resumed in a new system equals the uninterrupted one bit for bit (Voronoi, two instances)."""
    from cellgpu_b200 import VoronoiBatch, restore
    (p1, b1), (p2, b2) = jittered_lattice(16, 18, 0.25, 21), jittered_lattice(12, 14, 0.25, 22)
    N = [len(p1), len(p2)]
    b = VoronoiBatch(N, [b1, b2])
    b.set_positions(np.concatenate([p1, p2]))
    rng = np.random.default_rng(3)
    b.set_directors(rng.uniform(0, 2 * np.pi, sum(N)))
    b.set_motility(np.tile([0.3, 1.0], (sum(N), 1)))
    b.set_preferences(np.tile([1.0, 3.85], (sum(N), 1)))
    b.set_instance_seeds([7, 8])
    b.set_deterministic(True)
    b.triangulate()
    b.spp_run(20, dt=0.02)
    snap = b.snapshot()
    b.spp_run(40, dt=0.02)
    r = restore(snap)
    assert r.deterministic
    r.spp_run(40, dt=0.02)
    assert np.array_equal(r.positions(), b.positions())
    assert np.array_equal(r.directors(), b.directors())
    assert np.array_equal(r.forces(), b.forces())
    assert b.counters()["rows_changed"] > 0


def test_batch_equals_singles_bit_for_bit(cglib):
    """In the deterministic mode an instance's SPP trajectory does not depend on where it sits in a
    batch, bit for bit: forces are sums of instance-local contributions in exact fixed point, the
    topology is exact, and the device noise is keyed by the instance seed and local cell index.
    (Energies agree to rounding: their per-block partial sums follow the batch's block boundaries.)"""
    from cellgpu_b200 import VoronoiBatch
    shapes = [(10, 12), (16, 16), (20, 22)]
    lat = [jittered_lattice(nx, ny, 0.25, 40 + i) for i, (nx, ny) in enumerate(shapes)]
    poss = [p for p, _ in lat]
    boxes = [bx for _, bx in lat]
    Ns = [len(p) for p in poss]
    seeds = [11, 22, 33]
    rng = np.random.default_rng(5)
    ths = [rng.uniform(0, 2 * np.pi, n) for n in Ns]

    def make(sel):
        b = VoronoiBatch([Ns[i] for i in sel], [boxes[i] for i in sel])
        b.set_positions(np.concatenate([poss[i] for i in sel]))
        b.set_directors(np.concatenate([ths[i] for i in sel]))
        b.set_motility(np.tile([0.3, 1.0], (sum(Ns[i] for i in sel), 1)))
        b.set_instance_seeds([seeds[i] for i in sel])
        b.set_deterministic(True)
        b.triangulate()
        b.spp_run(30, dt=0.02)
        return b

    order = [2, 0, 1]  # another placement of the same instances
    b = make(order)
    Pb, Fb, Eb = b.positions(), b.forces(), b.energies()
    assert b.counters()["rows_changed"] > 0
    off = 0
    for j, i in enumerate(order):
        s = make([i])
        n = Ns[i]
        assert np.array_equal(Pb[off:off + n], s.positions())
        assert np.array_equal(Fb[off:off + n], s.forces())
        # energies: per-block partial sums depend on where block boundaries fall in the batch
        assert abs(Eb[j] - s.energies()[0]) <= 1e-13 * abs(Eb[j])
        off += n


def test_random_start_large_contributions(cglib):
    """From uniform random positions (how the bench's monolayer starts) near-degenerate triangles give force
    contributions far above O(1); the deterministic mode sums them exactly (third word of the
    fixed-point form) and the run stays finite, repeatable and equal in force to the atomic sums."""
    pos, box = monolayer(65536, 61)
    runs = []
    for det in (True, True, False):
        b = _spp_batch(pos, box, 62, det=det)
        b.compute_forces()
        F0 = b.forces()
        b.spp_run(20, dt=0.01)
        runs.append((F0, b.positions()))
        b.close()
    assert np.all(np.isfinite(runs[0][0])) and np.all(np.isfinite(runs[0][1]))
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])
    assert force_error(runs[0][0], runs[2][0]) < 1e-12
