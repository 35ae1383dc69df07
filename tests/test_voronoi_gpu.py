"""GPU parity of the Voronoi (SPV) hot path against the CPU oracle, through the C ABI.

Tolerances (written here, used below):
  * topology (Delaunay neighbour rows, canonical rotation): bit-exact;
  * FP64 forces: force_error <= 1e-10 (max |dF| / max(|F|, RMS F); summation order differs);
  * FP64 areas/perimeters: relative 1e-12;
  * mixed precision forces vs FP64 on a relaxed monolayer: norm-wise max |dF| / max |F| <= 1e-6,
    RMS error <= 1e-6 and per-cell max (the force_error normalisation) <= 1e-5. The per-cell
    maximum does not reach 1e-6: near force balance a cell's force is the sum of ~18 terms about ten
    times its size, and FP32 rounding of those terms alone leaves ~1e-6 to 5e-6 per cell
    (tests/test_precision_study.py shows it on the oracle's own arithmetic). FP64 is the mode that
    meets 1e-6 per cell; the mixed mode is measured and stated, not tuned to pass.
"""
import ctypes as C

import numpy as np
import pytest

from helpers import canonical, force_error, jittered_lattice, monolayer

pytestmark = pytest.mark.gpu

TOL_F64 = 1e-10
TOL_AP = 1e-12
TOL_MIXED_NORMWISE = 1e-6
TOL_MIXED_RMS = 1e-6
TOL_MIXED_MAX = 5e-6


@pytest.fixture(scope="module")
def torch():
    import torch
    return torch


def _batch(pos, box, precision=0, K=16):
    from cellgpu_b200 import VoronoiBatch
    b = VoronoiBatch([len(pos)], [box], K=K, precision=precision)
    b.set_positions(pos)
    return b


@pytest.mark.parametrize("N,seed", [(64, 1), (300, 2), (1000, 3), (4096, 4)])
def test_triangulation_matches_oracle(cglib, oracle, N, seed):
    pos, box = monolayer(N, seed)
    b = _batch(pos, box)
    b.triangulate()
    nn, nbr = b.topology()
    onn, onbr = oracle.periodic_delaunay(pos, box, 16)
    assert np.array_equal(nn, onn)
    assert np.array_equal(canonical(nn, nbr), canonical(onn, onbr))


def test_hexagonal_lattice_known_answer(cglib):
    from test_oracle import _hex_lattice
    pts, box = _hex_lattice()
    b = _batch(pts, box)
    b.triangulate()
    b.compute_forces()
    AP = b.area_perimeter()
    np.testing.assert_allclose(AP[:, 0], 1.0, rtol=1e-12)
    np.testing.assert_allclose(AP[:, 1], np.sqrt(8 * np.sqrt(3)), rtol=1e-12)
    assert np.abs(b.forces()).max() < 1e-11


@pytest.mark.parametrize("N,seed", [(300, 5), (2000, 6)])
def test_forces_match_oracle(cglib, oracle, N, seed):
    pos, box = monolayer(N, seed)
    b = _batch(pos, box)
    b.triangulate()
    pref = np.tile([1.0, 3.8], (N, 1))
    b.compute_forces()
    nn, nbr = b.topology()
    AP = oracle.voronoi_geometry(pos, box, nn, nbr)
    F = oracle.voronoi_forces(pos, box, nn, nbr, AP, pref)
    np.testing.assert_allclose(b.area_perimeter(), AP, rtol=TOL_AP, atol=1e-12)
    assert force_error(b.forces(), F) < TOL_F64
    E = b.energies()[0]
    assert abs(E - oracle.voronoi_energy(AP, pref)) < 1e-12 * max(1.0, E)


def test_raw_kernel_callers(cglib, oracle, torch):
    """The L1 drop-in entry points on caller-owned device memory."""
    N = 500
    pos, box = monolayer(N, 8)
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    dev = torch.device("cuda:0")
    tpos = torch.tensor(pos, device=dev)
    tnn = torch.tensor(nn, device=dev)
    tnbr = torch.tensor(nbr, device=dev)
    pref = np.tile([1.0, 3.9], (N, 1))
    tpref = torch.tensor(pref, device=dev)
    tAP = torch.zeros((N, 2), dtype=torch.float64, device=dev)
    tF = torch.zeros((N, 2), dtype=torch.float64, device=dev)
    p = lambda t: C.c_void_p(t.data_ptr())
    assert cglib.cg_voronoi_forces(p(tpos), p(tnn), p(tnbr), 16, N, box[0], box[1], p(tpref), 1.0, 1.0,
                                   p(tAP), p(tF), None) == 0
    torch.cuda.synchronize()
    AP = oracle.voronoi_geometry(pos, box, nn, nbr)
    F = oracle.voronoi_forces(pos, box, nn, nbr, AP, pref)
    assert force_error(tF.cpu().numpy(), F) < TOL_F64
    tAP2 = torch.zeros_like(tAP)
    assert cglib.cg_voronoi_geometry(p(tpos), p(tnn), p(tnbr), 16, N, box[0], box[1], p(tAP2), None) == 0
    torch.cuda.synchronize()
    np.testing.assert_allclose(tAP2.cpu().numpy(), AP, rtol=TOL_AP)
    # triangulate on the device into caller memory
    tnn2 = torch.zeros(N, dtype=torch.int32, device=dev)
    tnbr2 = torch.zeros((N, 16), dtype=torch.int32, device=dev)
    assert cglib.cg_voronoi_triangulate(p(tpos), N, box[0], box[1], 16, p(tnn2), p(tnbr2), None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(canonical(tnn2.cpu().numpy(), tnbr2.cpu().numpy()), canonical(nn, nbr))
    # exact test: the Delaunay triangulation passes; a perturbed point makes it fail
    flag = torch.zeros(N, dtype=torch.int32, device=dev)
    anyf = torch.zeros(1, dtype=torch.int32, device=dev)
    assert cglib.cg_voronoi_test_triangulation(p(tpos), p(tnn), p(tnbr), 16, N, box[0], box[1], p(flag),
                                               p(anyf), None) == 0
    torch.cuda.synchronize()
    assert int(anyf.item()) == 0
    pos2 = pos.copy()
    j = int(nbr[0, 0])
    pos2[0] = pos[j] + 0.02 * (pos[0] - pos[j])  # move cell 0 right next to a neighbour
    tpos2 = torch.tensor(pos2, device=dev)
    assert cglib.cg_voronoi_test_triangulation(p(tpos2), p(tnn), p(tnbr), 16, N, box[0], box[1], p(flag),
                                               p(anyf), None) == 0
    torch.cuda.synchronize()
    assert oracle.topology_mismatch(pos2, box, nn, nbr) > 0
    assert int(anyf.item()) == 1 and int(flag.sum().item()) > 0


def _spp_setup(pos, box, seed, v0=0.05):
    N = len(pos)
    rng = np.random.default_rng(seed + 100)
    theta = rng.uniform(0, 2 * np.pi, N)
    mot = np.tile([v0, 1.0], (N, 1))
    pref = np.tile([1.0, 3.8], (N, 1))
    b = _batch(pos, box)
    b.set_directors(theta)
    b.set_motility(mot)
    b.set_preferences(pref)
    b.triangulate()
    return b, theta, mot, pref, rng


def test_enqueue_host_energy_buffers(cglib, torch):
    """Energies of the asynchronous host-buffer step, per instance of a batch: into page-locked host
    memory (written by the reduction kernel itself) and into ordinary memory (copied), over
    repeated calls (the kernel's accumulators return to zero); each equals cg_get_energies."""
    from cellgpu_b200 import VoronoiBatch
    (p1, b1), (p2, b2) = jittered_lattice(12, 14, 0.25, 31), jittered_lattice(10, 12, 0.25, 32)
    Ns = [len(p1), len(p2)]
    N = sum(Ns)
    rng = np.random.default_rng(33)
    b = VoronoiBatch(Ns, [b1, b2])
    b.set_positions(np.concatenate([p1, p2]))
    b.set_directors(rng.uniform(0, 2 * np.pi, N))
    b.set_motility(np.tile([0.1, 1.0], (N, 1)))
    b.set_preferences(np.column_stack([np.ones(N), np.linspace(3.7, 3.9, N)]))
    b.triangulate()
    lib = b._lib
    noise = torch.from_numpy(rng.normal(size=(8, N))).pin_memory()
    pinned = torch.zeros((4, 2), dtype=torch.float64).pin_memory()
    plain = np.zeros((4, 2))
    for i in range(4):
        for buf, dst in ((pinned, C.c_void_p(pinned[i].data_ptr())), (plain, plain[i].ctypes.data_as(C.c_void_p))):
            k = 2 * i + (buf is plain)
            assert lib.cg_spp_enqueue_host(b.handle, C.c_void_p(noise[k].data_ptr()), 0.01, 1.0, dst) == 0
            assert lib.cg_poll(b.handle, None, None, 1) == 0
            got = np.asarray(buf[i])
            E = b.energies()
            np.testing.assert_allclose(got, E, rtol=1e-12)
            assert np.all(got > 0)


@pytest.mark.parametrize("N,steps,seed,v0,dt", [(300, 20, 10, 0.05, 0.01), (1500, 15, 11, 0.05, 0.01),
                                               (1152, 12, 12, 1.0, 0.05)])
def test_spp_each_step_matches_oracle(cglib, oracle, torch, N, steps, seed, v0, dt):
    """Per-step parity from a common state: each GPU step (forces on the repaired topology,
    integrate, move) against the oracle's CPU step with the same supplied noise; the state is then
    re-synchronised to the oracle's so that chaotic amplification of 1e-16 differences in random
    initial states (near-coincident points) cannot mask a real error."""
    if v0 >= 1.0:  # fast cells on a jittered lattice: many repairs every step
        pos, box = jittered_lattice(32, 36, 0.25, seed)
    else:
        pos, box = monolayer(N, seed)
    b, theta, mot, pref, rng = _spp_setup(pos, box, seed, v0=v0)
    noise = rng.normal(size=(steps, N))
    onn, onbr = oracle.periodic_delaunay(pos, box, 16)
    opos, oth = pos.copy(), theta.copy()
    changed = 0
    for s in range(steps):
        b.spp_run(1, dt=dt, mu=1.0, noise=torch.tensor(noise[s:s + 1], device="cuda:0"))
        F, _ = oracle.voronoi_spp_run(opos, box, onn, onbr, oth, mot, pref, noise[s:s + 1], dt=dt)
        assert np.abs(b.positions() - opos).max() < 1e-12
        assert force_error(b.forces(), F) < TOL_F64
        b.enforce_topology()
        nn, nbr = b.topology()
        assert np.array_equal(canonical(nn, nbr), canonical(onn, onbr))
        b.set_positions(opos)
        b.set_directors(oth)
        b.set_topology(onn, onbr)
    if v0 >= 1.0:
        assert b.counters()["rows_changed"] > 0


@pytest.mark.parametrize("nx,ny,steps,v0,dt", [(20, 24, 40, 0.05, 0.01), (24, 28, 20, 0.3, 0.02)])
def test_spp_free_run_matches_oracle(cglib, oracle, torch, nx, ny, steps, v0, dt):
    """Free-running trajectories (no re-synchronisation) from a well-conditioned jittered lattice;
    the fast case (v0 = 1, dt = 0.05) exercises many repairs per step."""
    pos, box = jittered_lattice(nx, ny, 0.25, 7)
    N = len(pos)
    b, theta, mot, pref, rng = _spp_setup(pos, box, 12, v0=v0)
    noise = rng.normal(size=(steps, N))
    b.spp_run(steps, dt=dt, mu=1.0, noise=torch.tensor(noise, device="cuda:0"))
    b.enforce_topology()
    onn, onbr = oracle.periodic_delaunay(pos, box, 16)
    opos, oth = pos.copy(), theta.copy()
    F, _ = oracle.voronoi_spp_run(opos, box, onn, onbr, oth, mot, pref, noise, dt=dt)
    assert np.abs(b.positions() - opos).max() < 1e-9
    assert np.abs(np.angle(np.exp(1j * (b.directors() - oth)))).max() < 1e-9
    nn, nbr = b.topology()
    assert np.array_equal(canonical(nn, nbr), canonical(onn, onbr))
    assert force_error(b.forces(), F) < 1e-8
    if v0 >= 1.0:
        assert b.counters()["rows_changed"] > 0


def test_enqueue_host_matches_oracle(cglib, oracle, torch):
    """The asynchronous host-buffer step (noise copied from pinned host memory on a copy stream,
    double-buffered; energy copied back every step) follows the oracle like the device-noise run."""
    pos, box = jittered_lattice(20, 24, 0.25, 9)
    N = len(pos)
    steps = 12
    b, theta, mot, pref, rng = _spp_setup(pos, box, 12, v0=0.1)
    noise = torch.from_numpy(rng.normal(size=(steps, N))).pin_memory()
    energy = torch.zeros((steps, 1), dtype=torch.float64).pin_memory()
    lib = b._lib
    for i in range(steps):
        assert lib.cg_spp_enqueue_host(b.handle, C.c_void_p(noise[i].data_ptr()), 0.01, 1.0,
                                       C.c_void_p(energy[i].data_ptr())) == 0
    done, halted = C.c_int(0), C.c_int(0)
    assert lib.cg_poll(b.handle, C.byref(done), C.byref(halted), 1) == 0
    assert not halted.value
    # each step reports the energy of the configuration its forces were computed on
    E_last = b.energies()[0]
    assert abs(energy[-1, 0].item() - E_last) <= 1e-12 * max(1.0, abs(E_last))
    assert np.all(np.diff(energy.numpy()[:, 0]) != 0)
    b.enforce_topology()
    onn, onbr = oracle.periodic_delaunay(pos, box, 16)
    opos, oth = pos.copy(), theta.copy()
    F, _ = oracle.voronoi_spp_run(opos, box, onn, onbr, oth, mot, pref, noise.numpy(), dt=0.01)
    assert np.abs(b.positions() - opos).max() < 1e-9


def test_mixed_precision_force_error(cglib, oracle):
    """Mixed precision (FP32 energy derivatives and contractions relative to each cell, FP64 vertex
    geometry, positions and predicates) against FP64 on the same state: on raw random points and
    on a relaxed monolayer (the dynamics the benchmarks run)."""
    N = 4096
    pos, box = monolayer(N, 31)
    b64 = _batch(pos, box, precision=0)
    b32 = _batch(pos, box, precision=1)
    b64.triangulate()
    b32.triangulate()
    b64.compute_forces()
    b32.compute_forces()
    err_random = force_error(b32.forces(), b64.forces())
    # relax with SPP (FP64, order-independent sums, so that the relaxed state is the same in every
    # run: the trajectory is chaotic, and the error depends on the state), then compare there
    b64.set_motility(np.tile([0.1, 1.0], (N, 1)))
    b64.set_deterministic(True)
    b64.spp_run(400, dt=0.01)
    b64.set_deterministic(False)
    # a run leaves the triangulation of the positions before its last move; mixed precision's
    # perimeter tangent is exact on Delaunay triangulations only, so repair it first
    b64.enforce_topology()
    rel = b64.positions()
    nn, nbr = b64.topology()
    b32.set_positions(rel)
    b32.set_topology(nn, nbr)
    b64.compute_forces()
    b32.compute_forces()
    F64 = b64.forces()
    err_relaxed = force_error(b32.forces(), F64)
    scale = np.sqrt(np.mean(np.sum(F64 ** 2, axis=1)))
    rms = np.sqrt(np.mean(np.sum((b32.forces() - F64) ** 2, axis=1))) / scale
    normwise = np.linalg.norm(b32.forces() - F64, axis=1).max() / np.linalg.norm(F64, axis=1).max()
    print(f"mixed force error: random {err_random:.2e}, relaxed max {err_relaxed:.2e} rms {rms:.2e} "
          f"norm-wise {normwise:.2e}")
    assert normwise < TOL_MIXED_NORMWISE
    assert rms < TOL_MIXED_RMS
    assert err_relaxed < TOL_MIXED_MAX
    assert err_random < TOL_MIXED_MAX


def test_batch_equals_singles(cglib):
    """Instances of a batch evolve as they do alone: forces per instance, and device-noise SPP runs
    (each instance's noise is keyed by its own seed and local cell index, so where it sits in the
    batch does not matter). Tolerance 1e-10 on positions after 20 steps (atomic summation order)."""
    from cellgpu_b200 import VoronoiBatch
    shapes = [(10, 12), (16, 16), (20, 22)]
    lat = [jittered_lattice(nx, ny, 0.25, 40 + i) for i, (nx, ny) in enumerate(shapes)]
    poss = [p for p, _ in lat]
    boxes = [bx for _, bx in lat]
    Ns = [len(p) for p in poss]
    seeds = [11, 22, 33]
    rng = np.random.default_rng(5)
    ths = [rng.uniform(0, 2 * np.pi, n) for n in Ns]
    b = VoronoiBatch(Ns, boxes)
    b.set_positions(np.concatenate(poss))
    b.set_directors(np.concatenate(ths))
    b.set_motility(np.tile([0.1, 1.0], (sum(Ns), 1)))
    b.set_instance_seeds(seeds)
    b.triangulate()
    b.compute_forces()
    Fb = b.forces()
    b.spp_run(20, dt=0.01)
    Pb = b.positions()
    off = 0
    for i, n in enumerate(Ns):
        s = VoronoiBatch([n], [boxes[i]])
        s.set_positions(poss[i])
        s.set_directors(ths[i])
        s.set_motility(np.tile([0.1, 1.0], (n, 1)))
        s.set_instance_seeds([seeds[i]])
        s.triangulate()
        s.compute_forces()
        assert force_error(Fb[off:off + n], s.forces()) < 1e-12
        s.spp_run(20, dt=0.01)
        assert np.abs(Pb[off:off + n] - s.positions()).max() < 1e-10
        off += n


@pytest.mark.parametrize("N", [262144])
def test_large_monolayer_invariants(cglib, N):
    pos, box = monolayer(N, 50)
    b = _batch(pos, box)
    b.triangulate()
    nn, _ = b.topology()
    assert nn.sum() == 6 * N
    b.spp_run(20, dt=0.01)
    b.enforce_topology()
    nn, _ = b.topology()
    assert nn.sum() == 6 * N
    b.compute_forces()
    F = b.forces()
    AP = b.area_perimeter()
    assert abs(AP[:, 0].sum() - box[0] * box[1]) < 1e-6
    assert np.abs(F.sum(axis=0)).max() < 1e-8 * N


@pytest.mark.parametrize("N", [262144])
def test_large_monolayer_matches_oracle(cglib, oracle, N):
    """The full-size monolayer (N = 262144, L = 512) against the oracle directly, after 20 SPP steps
    from uniform positions (the repair's busiest regime): Delaunay rows bit-exact, A/P within
    1e-12 relative and forces within the FP64 tolerance."""
    pos, box = monolayer(N, 50)
    b = _batch(pos, box)
    pref = np.tile([1.0, 3.8], (N, 1))
    b.set_preferences(pref)
    b.triangulate()
    b.spp_run(20, dt=0.01)
    b.enforce_topology()
    P = b.positions()
    nn, nbr = b.topology()
    onn, onbr = oracle.periodic_delaunay(P, box, 32)
    m = int(max(nn.max(), onn.max()))
    assert np.array_equal(nn, onn)
    assert np.array_equal(canonical(nn, nbr)[:, :m], canonical(onn, onbr)[:, :m])
    b.compute_forces()
    AP = oracle.voronoi_geometry(P, box, onn, onbr)
    F = oracle.voronoi_forces(P, box, onn, onbr, AP, pref)
    np.testing.assert_allclose(b.area_perimeter(), AP, rtol=TOL_AP, atol=1e-12)
    assert force_error(b.forces(), F) < TOL_F64
