"""Serving (continuous batching): each request gives the same result alone and in a mix with other
requests of every kind and size, and admission respects the memory budget.

Tolerances (written here): SPP runs -- positions within 1e-9 (periodic minimum image), energies
within 1e-10 relative (floating-point atomics are summed in another order in a larger batch);
FIRE -- both runs reach the force threshold, energies within 1e-9 relative, positions within 1e-6.
"""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests():
    from cellgpu_b200.serve import Request
    # the FIRE cases converge to 1e-10 on the oracle in 468 (Voronoi) and 1401 (vertex) iterations
    return [Request("voronoi", "spp", 150, p0=3.75, seed=1, steps=60),
            Request("voronoi", "fire", 130, p0=3.70, seed=2, fire_tol=1e-10, fire_max_iterations=8000),
            Request("vertex", "spp", 110, p0=3.80, seed=3, steps=40),
            Request("vertex", "fire", 130, p0=3.80, seed=2, fire_tol=1e-10, fire_max_iterations=8000)]


def _fillers():
    from cellgpu_b200.serve import Request
    out = []
    for i in range(3):
        out.append(Request("voronoi", "spp", 90 + 40 * i, p0=3.85, seed=100 + i, steps=60))
        out.append(Request("voronoi", "fire", 100 + 20 * i, p0=3.65, seed=200 + i, fire_tol=1e-10,
                           fire_max_iterations=8000))
        out.append(Request("vertex", "spp", 80 + 30 * i, p0=3.75, seed=300 + i, steps=40))
        out.append(Request("vertex", "fire", 90 + 25 * i, p0=3.85, seed=400 + i, fire_tol=1e-10,
                           fire_max_iterations=8000))
    return out


def _pdist(a, b, n):
    L = np.sqrt(n)
    d = a - b
    d -= L * np.round(d / L)
    return np.abs(d).max()


def test_same_result_alone_and_in_mix(cglib):
    from cellgpu_b200.serve import Server
    reqs = _requests()
    alone = []
    for r in reqs:
        with Server(lanes=1) as srv:
            alone.append(srv.submit(copy.deepcopy(r)).result())
    mix_in, where = [], []
    fill = _fillers()
    for i, r in enumerate(reqs):  # interleave: every batch kind holds several instances
        mix_in.extend(fill[3 * i:3 * i + 3])
        where.append(len(mix_in))
        mix_in.append(copy.deepcopy(r))
    with Server(lanes=3) as srv:
        futs = srv.submit_many(mix_in)
        mix = [f.result() for f in futs]
    for r, a, k in zip(reqs, alone, where):
        m = mix[k]
        assert m.batch_requests > 1  # it really shared a batch
        if r.task == "spp":
            assert _pdist(a.positions, m.positions, r.n) < 1e-9
            assert abs(a.energy - m.energy) <= 1e-10 * max(1.0, abs(a.energy))
        else:
            assert a.fmax <= r.fire_tol and m.fmax <= r.fire_tol
            assert abs(a.energy - m.energy) <= 1e-9 * max(1.0, abs(a.energy))
            assert _pdist(a.positions, m.positions, r.n) < 1e-6


def test_admission_by_footprint(cglib):
    """A budget that fits about one batch at a time: every request still completes, and the
    resident footprint never exceeds the budget."""
    from cellgpu_b200.serve import Request, Server, footprint
    reqs = [Request("voronoi", "spp", 400 + 50 * i, seed=i, steps=20) for i in range(8)]
    budget = footprint("voronoi", [max(r.n for r in reqs)]) * 2
    with Server(lanes=4, memory_budget=budget) as srv:
        res = [f.result() for f in srv.submit_many(reqs)]
        peak = srv.peak_resident
    assert len(res) == 8 and all(np.isfinite(r.energy) for r in res)
    assert peak <= budget
    with Server(lanes=1, memory_budget=1000) as srv:
        fut = srv.submit(Request("voronoi", "spp", 500, seed=1, steps=5))
        with pytest.raises(MemoryError):
            fut.result()


def test_deterministic_server_same_bits_alone_and_in_mix(cglib):
    """Server(deterministic=True): an SPP request's positions are the same bits alone and in a
    mixed batch, for both models (fixed-point force sums; noise keyed per instance)."""
    from cellgpu_b200.serve import Server
    reqs = [r for r in _requests() if r.task == "spp"]
    alone = []
    for r in reqs:
        with Server(lanes=1, deterministic=True) as srv:
            alone.append(srv.submit(copy.deepcopy(r)).result())
    fill = [r for r in _fillers() if r.task == "spp"]
    mix_in = fill[:2] + [copy.deepcopy(reqs[0])] + fill[2:4] + [copy.deepcopy(reqs[1])] + fill[4:]
    where = [2, 5]
    with Server(lanes=2, deterministic=True) as srv:
        mix = [f.result() for f in srv.submit_many(mix_in)]
    for a, k in zip(alone, where):
        m = mix[k]
        assert m.batch_requests > 1
        assert np.array_equal(a.positions, m.positions)


def _join(reqs, deterministic):
    """Run reqs[0] on a one-lane server and submit the others once its batch is running: they join
    it at a chunk end (the batch is rebuilt around the running request)."""
    import time

    from cellgpu_b200.serve import Server
    with Server(lanes=1, deterministic=deterministic) as srv:
        first = srv.submit(copy.deepcopy(reqs[0]))
        t0 = time.perf_counter()
        while srv.batches == 0 and time.perf_counter() - t0 < 60:
            time.sleep(0.001)
        rest = [srv.submit(copy.deepcopy(r)) for r in reqs[1:]]
        out = [first.result()] + [f.result() for f in rest]
        joined = srv.joined
    return out, joined


@pytest.mark.parametrize("model", ["voronoi", "vertex"])
def test_spp_request_joining_a_running_batch_same_bits(cglib, model):
    """Deterministic mode: an SPP request admitted into a running batch, and the request whose state
    moved into the rebuilt batch, both end with the positions they have alone, bit for bit."""
    from cellgpu_b200.serve import Request, Server
    reqs = [Request(model, "spp", 1200, p0=3.8, seed=21, steps=3000, v0=0.1),
            Request(model, "spp", 500, p0=3.7, seed=22, steps=3000, v0=0.1)]
    alone = []
    for r in reqs:
        with Server(lanes=1, deterministic=True) as srv:
            alone.append(srv.submit(copy.deepcopy(r)).result())
    mix, joined = _join(reqs, True)
    assert joined >= 1 and mix[1].joined
    for a, m in zip(alone, mix):
        assert np.array_equal(a.positions, m.positions)
        assert a.energy == m.energy


@pytest.mark.parametrize("deterministic", [True, False])
def test_fire_request_joining_a_running_batch(cglib, deterministic):
    """FIRE requests admitted into a running minimisation batch (the running request's velocities and
    FIRE state move with it into the rebuilt batch). Deterministic mode: both end bit for bit where
    they end alone, with the same iteration counts (forces in fixed point, FIRE sums in an order
    fixed by the instance alone). Default mode: the sums are atomic, so the paths differ from the
    lone runs by rounding, and FIRE from a random start may then settle in another local minimum;
    both requests still converge to the tolerance."""
    from cellgpu_b200.serve import Request, Server
    reqs = [Request("voronoi", "fire", 900, p0=3.7, seed=31, fire_tol=1e-10, fire_max_iterations=20000),
            Request("voronoi", "fire", 700, p0=3.7, seed=32, fire_tol=1e-10, fire_max_iterations=20000)]
    alone = []
    for r in reqs:
        with Server(lanes=1, deterministic=deterministic) as srv:
            alone.append(srv.submit(copy.deepcopy(r)).result())
    mix, joined = _join(reqs, deterministic)
    assert joined >= 1 and mix[1].joined
    for r, a, m in zip(reqs, alone, mix):
        assert a.fmax <= r.fire_tol and m.fmax <= r.fire_tol
        if deterministic:
            assert np.array_equal(a.positions, m.positions)
            assert a.energy == m.energy and a.iterations == m.iterations


def test_fire_in_pieces_equals_one_call(cglib):
    """cg_fire_begin + cg_fire_advance in pieces of 48 iterations give the same minimisation as one
    cg_fire_minimize call (same iteration count, energies within 1e-12 relative)."""
    from cellgpu_b200 import FireParams, VoronoiBatch
    from helpers import monolayer
    pos, box = monolayer(400, 71)
    out = []
    for pieces in (False, True):
        b = VoronoiBatch([400], [box])
        b.set_positions(pos)
        b.set_preferences(np.tile([1.0, 3.7], (400, 1)))
        b.set_deterministic(True)
        b.triangulate()
        prm = FireParams.defaults(force_cutoff=1e-10, max_iterations=4000)
        if pieces:
            b.fire_begin(prm)
            while b.fire_advance(prm, 48) < 1:
                pass
        else:
            b.fire_minimize(prm)
        its, fmax, _ = b.fire_state()
        out.append((int(its[0]), float(b.energies()[0]), b.positions()))
    assert out[0][0] == out[1][0]
    assert abs(out[0][1] - out[1][1]) <= 1e-12 * abs(out[0][1])
    assert np.array_equal(out[0][2], out[1][2])
