"""On-device observables per instance against the same quantities computed on the host from the
state the library returns (tolerance 1e-12 relative for the shape statistics, 1e-12 absolute for
MSD; overlap exact), for a two-instance Voronoi batch and a vertex batch."""
import numpy as np
import pytest

from helpers import jittered_lattice

pytestmark = pytest.mark.gpu


def _host_obs(AP, P, P0, box, cutoff):
    q = AP[:, 1] / np.sqrt(AP[:, 0])
    d = P - P0
    d -= np.asarray(box) * np.round(d / np.asarray(box))
    r2 = np.sum(d * d, axis=1)
    return {"mean_q": q.mean(), "var_q": np.mean((q - q.mean()) ** 2), "mean_A": AP[:, 0].mean(),
            "mean_P": AP[:, 1].mean(), "var_A": np.mean((AP[:, 0] - AP[:, 0].mean()) ** 2),
            "var_P": np.mean((AP[:, 1] - AP[:, 1].mean()) ** 2), "msd": r2.mean(),
            "overlap": np.mean(np.sqrt(r2) < cutoff)}


def _check(obs, i, ref):
    for k in ("mean_q", "var_q", "mean_A", "mean_P", "var_A", "var_P"):
        assert abs(obs[k][i] - ref[k]) <= 1e-12 * max(1.0, abs(ref[k])), k
    assert abs(obs["msd"][i] - ref["msd"]) < 1e-12
    assert obs["overlap"][i] == pytest.approx(ref["overlap"], abs=1e-15)


def test_voronoi_observables(cglib):
    from cellgpu_b200 import VoronoiBatch
    (p1, b1), (p2, b2) = jittered_lattice(20, 22, 0.25, 31), jittered_lattice(14, 16, 0.25, 32)
    N = [len(p1), len(p2)]
    b = VoronoiBatch(N, [b1, b2])
    b.set_positions(np.concatenate([p1, p2]))
    b.set_motility(np.tile([0.3, 1.0], (sum(N), 1)))
    b.triangulate()
    obs = b.observables()
    assert np.all(np.isnan(obs["msd"]))
    b.set_reference_positions()
    P0 = b.positions()
    b.spp_run(60, dt=0.01)
    b.compute_forces()
    obs = b.observables(cutoff=0.05)
    AP, P = b.area_perimeter(), b.positions()
    off = 0
    for i, (n, box) in enumerate(zip(N, [b1, b2])):
        _check(obs, i, _host_obs(AP[off:off + n], P[off:off + n], P0[off:off + n], box, 0.05))
        off += n
    assert 0 < obs["overlap"][0] < 1


def test_vertex_observables(cglib):
    from cellgpu_b200 import VertexBatch
    p, box = jittered_lattice(12, 14, 0.3, 33)
    n = len(p)
    b = VertexBatch([n], [box], vmax=20)
    b.from_cells(p)
    b.set_reference_positions()
    V0 = b.positions()
    b.brownian_run(30, dt=0.005, mu=1.0, T=0.01)
    b.compute_forces()
    obs = b.observables(cutoff=0.02)
    _check(obs, 0, _host_obs(b.area_perimeter(), b.positions(), V0, box, 0.02))


def _golden():
    import glob
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    return dict(np.load(sorted(glob.glob(os.path.join(here, "observables_N*.npz")))[0]))


def test_voronoi_observables_match_reference(cglib):
    """Against the reference's own Simple2DCell::reportq / reportVarq / reportVarAP and
    dynamicalFeatures::computeMSD / computeOverlapFunction (tests/golden/observables_N500_s11.npz):
    the reference's state after 40 SPP steps, with its starting positions as the MSD reference.
    Tolerance 1e-12 relative (summation order); overlap exact."""
    from cellgpu_b200 import VoronoiBatch
    g = _golden()
    N, box = int(g["N"]), tuple(g["box"])
    b = VoronoiBatch([N], [box])
    b.set_positions(g["pos0"])
    b.set_reference_positions()
    b.set_positions(g["pos1"])
    b.triangulate()
    b.compute_forces()
    obs = b.observables(cutoff=float(g["cutoff"]))
    assert np.abs(b.area_perimeter() - g["AP1"]).max() < 1e-12
    for k in ("mean_q", "var_q", "var_A", "var_P", "msd"):
        assert abs(obs[k][0] - float(g[k])) <= 1e-12 * max(1.0, abs(float(g[k]))), k
    assert obs["overlap"][0] == float(g["overlap"])
