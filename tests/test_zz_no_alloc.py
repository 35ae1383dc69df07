"""The allocation-free triangulation entry point (cg_voronoi_triangulate_noalloc) against the
allocating one (cg_voronoi_triangulate), through the C ABI.

The no-alloc variant is for callers that cannot allocate device memory: enqueueing while a CUDA
graph is captured in global mode, latency-critical loops that cannot absorb cudaFree's implicit
device synchronisation, and applications that give the library a fixed memory budget. Its scratch
is a file-scope device array shared by all calls, so this test also makes two calls in a row on
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
