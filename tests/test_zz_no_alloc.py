"""The allocation-free triangulation entry point (cg_voronoi_triangulate_noalloc) against the
allocating one (cg_voronoi_triangulate), through the C ABI.

The no-alloc variant is for callers that cannot allocate device memory: applications that give the
library a fixed memory budget owned by another allocator, latency-critical loops that cannot absorb
cudaFree's implicit device synchronisation, and host threads that run while another thread captures
a CUDA graph in global mode (cudaMalloc is illegal for every thread then). Its scratch is a
file-scope device array shared by all calls, so this test also makes two calls in a row on
different inputs: the second must not see anything left over from the first. Topology is integer
data, so the tolerance is exact equality of the neighbour counts and rows.

This file is collected last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _tri(cglib, torch, fn, pos, box, K=16):
    dev = torch.device("cuda:0")
    N = len(pos)
    tpos = torch.tensor(pos, device=dev)
    nn = torch.full((N,), -1, dtype=torch.int32, device=dev)
    nbr = torch.full((N, K), -1, dtype=torch.int32, device=dev)
    p = lambda t: C.c_void_p(t.data_ptr())
    rc = fn(p(tpos), N, box[0], box[1], K, p(nn), p(nbr), None)
    torch.cuda.synchronize()
    assert rc == 0, cglib.cg_last_error_string()
    return nn.cpu().numpy(), nbr.cpu().numpy()


def test_noalloc_triangulation_matches_allocating_entry_point(cglib):
    import torch

    rng = np.random.default_rng(77)
    cases = []
    for N in (3000, 1200):  # two calls in a row: larger first, then smaller
        L = float(np.sqrt(N))
        cases.append((rng.random((N, 2)) * L, (L, L)))
    for pos, box in cases:
        nn0, nbr0 = _tri(cglib, torch, cglib.cg_voronoi_triangulate, pos, box)
        nn1, nbr1 = _tri(cglib, torch, cglib.cg_voronoi_triangulate_noalloc, pos, box)
        assert np.array_equal(nn0, nn1)
        for i in range(len(pos)):
            assert np.array_equal(nbr0[i, : nn0[i]], nbr1[i, : nn1[i]])
        assert nn1.sum() == 6 * len(pos)


def test_noalloc_rejects_sizes_beyond_its_limit(cglib):
    import torch

    N = 65537  # CG_NOALLOC_MAX_CELLS + 1: rejected before any device work
    dev = torch.device("cuda:0")
    tpos = torch.zeros((N, 2), dtype=torch.float64, device=dev)
    nn = torch.zeros(N, dtype=torch.int32, device=dev)
    nbr = torch.zeros((N, 16), dtype=torch.int32, device=dev)
    p = lambda t: C.c_void_p(t.data_ptr())
    rc = cglib.cg_voronoi_triangulate_noalloc(p(tpos), N, 256.0, 256.0, 16, p(nn), p(nbr), None)
    assert rc == -3  # CG_ERR_CAPACITY
    assert b"CG_NOALLOC_MAX_CELLS" in cglib.cg_last_error_string()


def _flower(n_ring=18, L=20.0, seed=5):
    """A cell ringed by n_ring cells (n_ring Delaunay neighbours) in a jittered unit lattice."""
    rng = np.random.default_rng(seed)
    c = np.array([L / 2, L / 2])
    ang = np.arange(n_ring) * 2 * np.pi / n_ring + 0.01
    ring = c + np.stack([np.cos(ang), np.sin(ang)], 1)
    g = np.arange(0.5, L, 1.0)
    lat = np.array([(x, y) for y in g for x in g]) + rng.uniform(-0.15, 0.15, (len(g) ** 2, 2))
    lat = lat[np.linalg.norm(lat - c, axis=1) > 1.8]
    return np.concatenate([[c], ring, lat]) % L, (L, L)


def test_noalloc_capacity_failure_leaves_no_stale_reads(cglib):
    """A star that overflows K = 8 (the ringed cell has 18 neighbours, random cells reach 9-10) makes
    the star kernel stop with rows half written. The rows and counts are prefilled with -1, so the
    consistency pass would read far outside the buffers if it ran on them: the call must report
    CG_ERR_CAPACITY, and a following good call on the same shared scratch must still succeed."""
    import torch

    pos, box = _flower()
    N = len(pos)
    dev = torch.device("cuda:0")
    tpos = torch.tensor(pos, device=dev)
    p = lambda t: C.c_void_p(t.data_ptr())
    K = 8
    nn = torch.full((N,), -1, dtype=torch.int32, device=dev)
    nbr = torch.full((N, K), -1, dtype=torch.int32, device=dev)
    rc = cglib.cg_voronoi_triangulate_noalloc(p(tpos), N, box[0], box[1], K, p(nn), p(nbr), None)
    torch.cuda.synchronize()
    assert rc == -3, (rc, cglib.cg_last_error_string())  # CG_ERR_CAPACITY
    nn0, nbr0 = _tri(cglib, torch, cglib.cg_voronoi_triangulate, pos, box, K=32)
    nn1, nbr1 = _tri(cglib, torch, cglib.cg_voronoi_triangulate_noalloc, pos, box, K=32)
    assert nn1[0] == 18
    assert np.array_equal(nn0, nn1) and np.array_equal(nbr0, nbr1)


def test_noalloc_beside_a_global_mode_capture(cglib):
    """The use the entry point exists for: while another thread holds a global-mode stream capture
    open (cudaMalloc would be an illegal call for every thread then), a call on a non-blocking stream
    succeeds, and the capture still ends cleanly and replays."""
    import threading

    import torch

    rng = np.random.default_rng(78)
    N = 2000
    L = float(np.sqrt(N))
    pos = rng.random((N, 2)) * L
    dev = torch.device("cuda:0")
    tpos = torch.tensor(pos, device=dev)
    nn = torch.full((N,), -1, dtype=torch.int32, device=dev)
    nbr = torch.full((N, 16), -1, dtype=torch.int32, device=dev)
    nn_ref, nbr_ref = _tri(cglib, torch, cglib.cg_voronoi_triangulate_noalloc, pos, (L, L))
    x = torch.ones(1024, device=dev)
    y = torch.empty_like(x)
    torch.cuda.synchronize()
    started, release = threading.Event(), threading.Event()
    graph = torch.cuda.CUDAGraph()
    err = []

    def capture():
        try:
            s = torch.cuda.Stream()
            with torch.cuda.stream(s):
                graph.capture_begin(capture_error_mode="global")
                y.copy_(x * 2)
                started.set()
                release.wait(60)
                graph.capture_end()
        except Exception as e:  # reported by the main thread
            err.append(e)
            started.set()

    t = threading.Thread(target=capture)
    t.start()
    started.wait(60)
    s2 = torch.cuda.Stream()  # torch streams are created non-blocking
    p = lambda v: C.c_void_p(v.data_ptr())
    try:
        rc = cglib.cg_voronoi_triangulate_noalloc(p(tpos), N, L, L, 16, p(nn), p(nbr), C.c_void_p(s2.cuda_stream))
        msg = cglib.cg_last_error_string()
    finally:
        release.set()
        t.join(60)
    assert not err, err
    assert rc == 0, msg
    graph.replay()
    torch.cuda.synchronize()
    assert torch.equal(y, x * 2)
    assert np.array_equal(nn.cpu().numpy(), nn_ref) and np.array_equal(nbr.cpu().numpy(), nbr_ref)
