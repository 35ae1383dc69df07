"""Pins the CPU oracle against the reference's own CPU path.

tests/golden/*.npz are outputs of the reference's sources (compiled in place by
oracle/Makefile.ref, see tests/golden/make_golden.py). The oracle must reproduce them: Voronoi and
vertex geometry, forces and energies, SPP and Brownian trajectories with the reference's own
reproducible noise (topology and T1 rewiring bit-exact), and FIRE minimisations to the same
force threshold. When the reference build is present, the same checks run live against it too.
"""
import glob
import os

import numpy as np
import pytest

from helpers import canonical, force_error

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


def _load(pattern):
    files = sorted(glob.glob(os.path.join(GOLD, pattern)))
    assert files, f"missing golden fixtures {pattern}"
    return [dict(np.load(f, allow_pickle=False)) for f in files]


@pytest.mark.parametrize("g", _load("voronoi_N*.npz"), ids=lambda g: f"N{int(g['N'])}")
def test_voronoi_golden(oracle, g):
    N, box = int(g["N"]), tuple(g["box"])
    pos = g["pos"].copy()
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    assert np.array_equal(canonical(nn, nbr), canonical(g["nn0"], g["nbr0"]))
    pref = np.tile([1.0, 3.8], (N, 1))
    AP = oracle.voronoi_geometry(pos, box, nn, nbr)
    F = oracle.voronoi_forces(pos, box, nn, nbr, AP, pref)
    assert np.abs(AP - g["AP0"]).max() < 1e-12
    assert force_error(F, g["F0"]) < 1e-12
    assert abs(oracle.voronoi_energy(AP, pref) - float(g["E0"])) < 1e-10
    # SPP with the reference's reproducible deviates
    theta = g["theta"].copy()
    mot = np.tile([float(g["v0"]), float(g["Dr"])], (N, 1))
    oracle.voronoi_spp_run(pos, box, nn, nbr, theta, mot, pref, g["noise"], dt=float(g["dt"]))
    assert np.abs(pos - g["pos1"]).max() < 1e-11
    assert np.abs(theta - g["theta1"]).max() < 1e-11
    assert np.array_equal(canonical(nn, nbr), canonical(g["nn1"], g["nbr1"]))


def test_vertex_golden(oracle):
    g = _load("vertex_Nc*.npz")[0]
    box, vmax = tuple(g["box"]), int(g["vmax"])
    cp = g["cellpos"]
    nn, nbr = oracle.periodic_delaunay(cp, box, 16)
    vpos, vn, vcn, cvn, cv = oracle.vertex_from_delaunay(cp, box, nn, nbr, vmax=vmax)
    assert np.abs(vpos - g["vpos"]).max() == 0.0
    assert np.array_equal(vn, g["vn"]) and np.array_equal(vcn, g["vcn"]) and np.array_equal(cvn, g["cvn"])
    for c in range(len(cvn)):
        assert np.array_equal(cv[c, :cvn[c]], g["cv"][c, :cvn[c]])
    AP = oracle.vertex_geometry(vpos, box, cvn, cv)
    F = oracle.vertex_forces(vpos, box, cvn, cv, vcn, AP, g["pref"])
    assert np.abs(AP - g["AP0"]).max() < 1e-12
    assert force_error(F, g["F0"]) < 1e-12
    oracle.vertex_brownian_run(vpos, box, vn, vcn, cvn, cv, g["pref"], g["noise"], dt=float(g["dt"]),
                               T=float(g["T"]), t1_threshold=float(g["t1"]))
    assert np.abs(vpos - g["vpos1"]).max() < 1e-12
    assert np.array_equal(vn, g["vn1"]) and np.array_equal(vcn, g["vcn1"]) and np.array_equal(cvn, g["cvn1"])
    for c in range(len(cvn)):
        assert np.array_equal(cv[c, :cvn[c]], g["cv1"][c, :cvn[c]])


def test_fire_voronoi_golden(oracle):
    g = _load("fire_voronoi_*.npz")[0]
    N, box = int(g["N"]), tuple(g["box"])
    pos = g["pos"].copy()
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    prm = oracle.FireParams.defaults(force_cutoff=float(g["cutoff"]), max_iterations=int(g["max_iterations"]))
    F, AP, _ = oracle.fire_voronoi(pos, box, nn, nbr, np.tile([1.0, 3.8], (N, 1)), prm)
    assert np.sqrt(np.max(np.sum(F ** 2, axis=1))) <= float(g["cutoff"])
    assert np.abs(pos - g["pos1"]).max() < 1e-8
    E = oracle.voronoi_energy(AP, np.tile([1.0, 3.8], (N, 1)))
    assert abs(E - float(g["E1"])) < 1e-10 * max(1.0, abs(E))


def test_fire_vertex_golden(oracle):
    g = _load("fire_vertex_*.npz")[0]
    box, vmax, Nc = tuple(g["box"]), int(g["vmax"]), int(g["Nc"])
    vpos, vn, vcn, cvn, cv = (g["vpos"].copy(), g["vn"].copy(), g["vcn"].copy(), g["cvn"].copy(),
                              np.ascontiguousarray(g["cv"]).copy())
    prm = oracle.FireParams.defaults(force_cutoff=float(g["cutoff"]), max_iterations=int(g["max_iterations"]))
    # the reference's VertexQuadraticEnergy(n, A0=1, P0=3.8) and its T1 threshold default 0.01
    F, AP, _ = oracle.fire_vertex(vpos, box, vn, vcn, cvn, cv, np.tile([1.0, 3.8], (Nc, 1)), prm, t1_threshold=0.01)
    assert np.abs(vpos - g["vpos1"]).max() < 1e-8
    assert abs(oracle.voronoi_energy(AP, np.tile([1.0, 3.8], (Nc, 1))) - float(g["E1"])) < 1e-9


@pytest.mark.parametrize("mode", ["simple", "matrix"])
def test_tension_golden(oracle, mode):
    """VoronoiQuadraticEnergyWithTension: forces and energy with one gamma for unlike types and
    with a symmetric tension matrix."""
    g = _load("tension_N*.npz")[0]
    pos, box = g["pos"], tuple(g["box"])
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    AP = oracle.voronoi_geometry(pos, box, nn, nbr)
    kw = dict(gamma=float(g["gamma"])) if mode == "simple" else dict(gammas=g["gammas"])
    F = oracle.voronoi_tension_forces(pos, box, nn, nbr, AP, g["pref"], g["types"], **kw)
    E = oracle.voronoi_tension_energy(pos, box, nn, nbr, AP, g["pref"], g["types"], **kw)
    assert np.abs(AP - g["AP_" + mode]).max() < 1e-12
    assert force_error(F, g["F_" + mode]) < 1e-12
    assert abs(E - float(g["E_" + mode])) < 1e-10 * abs(E)


def test_tension_forces_are_a_gradient(oracle):
    """The tension forces are minus the gradient of the quadratic energy plus every unlike edge's
    gamma l counted from both of its cells (central differences, topology held fixed)."""
    from helpers import monolayer
    pos, box = monolayer(80, 11)
    N = len(pos)
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    rng = np.random.default_rng(3)
    types = rng.integers(0, 2, N)
    pref = np.tile([1.0, 3.8], (N, 1))

    def energy(p):
        AP = oracle.voronoi_geometry(p, box, nn, nbr)
        quad = oracle.voronoi_energy(AP, pref)
        return quad + 2.0 * (oracle.voronoi_tension_energy(p, box, nn, nbr, AP, pref, types, gamma=0.2) - quad)

    AP = oracle.voronoi_geometry(pos, box, nn, nbr)
    F = oracle.voronoi_tension_forces(pos, box, nn, nbr, AP, pref, types, gamma=0.2)
    h = 1e-6
    for c in rng.choice(N, 12, replace=False):
        for d in range(2):
            p1, p2 = pos.copy(), pos.copy()
            p1[c, d] += h
            p2[c, d] -= h
            assert abs(-(energy(p1) - energy(p2)) / (2 * h) - F[c, d]) < 1e-6 * max(1.0, np.abs(F).max())


@pytest.mark.parametrize("mode", ["simple", "matrix"])
def test_vertex_tension_golden(oracle, mode):
    """VertexQuadraticEnergyWithTension (CPU branch): forces with one gamma and with a symmetric
    matrix on the reference's Delaunay-dual state; the tension energy (not implemented by the
    reference) has these forces as its negative gradient."""
    g = _load("vertex_tension_Nc*.npz")[0]
    box = tuple(g["box"])
    AP = oracle.vertex_geometry(g["vpos"], box, g["cvn"], g["cv"])
    kw = dict(gamma=float(g["gamma"])) if mode == "simple" else dict(gammas=g["gammas"])
    F = oracle.vertex_tension_forces(g["vpos"], box, g["cvn"], g["cv"], g["vcn"], AP, g["pref"], g["types"], **kw)
    assert np.abs(AP - g["AP_" + mode]).max() < 1e-12
    assert force_error(F, g["F_" + mode]) < 1e-12
    assert abs(oracle.voronoi_energy(AP, g["pref"]) - float(g["E_" + mode])) < 1e-10

    def energy(vp):
        A = oracle.vertex_geometry(vp, box, g["cvn"], g["cv"])
        return oracle.vertex_tension_energy(vp, box, g["cvn"], g["cv"], g["vcn"], A, g["pref"], g["types"], **kw)

    h = 1e-6
    for v in np.random.default_rng(2).choice(len(g["vpos"]), 12, replace=False):
        for d in range(2):
            p1, p2 = g["vpos"].copy(), g["vpos"].copy()
            p1[v, d] += h
            p2[v, d] -= h
            assert abs(-(energy(p1) - energy(p2)) / (2 * h) - F[v, d]) < 1e-6 * max(1.0, np.abs(F).max())


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libcgref.so")),
                    reason="reference build not present")
def test_live_reference_spp_matches_oracle(oracle):
    import contextlib
    import io

    from oracle import ref_harness as R
    N, steps = 500, 15
    L = float(np.sqrt(N))
    rng = np.random.default_rng(99)
    pos = rng.random((N, 2)) * L
    theta = rng.uniform(0, 2 * np.pi, N)
    with contextlib.redirect_stdout(io.StringIO()):
        r = R.RefVoronoi(N)
        r.set_state(pos, theta)
        r.set_motility(0.1, 1.0)
        r.spp_run(steps, 0.01, True)
        p1, t1, nn1, nbr1 = r.state()
    noise = R.reproducible_normals(steps * N).reshape(steps, N)
    nn, nbr = oracle.periodic_delaunay(pos, (L, L), 16)
    oracle.voronoi_spp_run(pos, (L, L), nn, nbr, theta, np.tile([0.1, 1.0], (N, 1)), np.tile([1.0, 3.8], (N, 1)),
                           noise)
    assert np.abs(pos - p1).max() < 1e-11
    assert np.array_equal(canonical(nn, nbr), canonical(nn1, nbr1))


def test_exclusions_golden(oracle):
    """Particle exclusions (voronoiModelBase::setExclusions) against the reference's own outputs:
    forces and external forces on the initial state, then SPP steps with the reference's deviates."""
    g = _load("exclusions_N*.npz")[0]
    N, box = int(g["N"]), tuple(g["box"])
    ex = g["exes"]
    pos = g["pos"].copy()
    nn, nbr = oracle.periodic_delaunay(pos, box, 16)
    pref = np.tile([1.0, 3.8], (N, 1))
    AP = oracle.voronoi_geometry(pos, box, nn, nbr)
    F, ext = oracle.apply_exclusions(oracle.voronoi_forces(pos, box, nn, nbr, AP, pref), ex)
    assert np.all(F[ex != 0] == 0.0)
    assert force_error(F, g["F0"]) < 1e-12
    assert force_error(ext[ex != 0], g["ext0"][ex != 0]) < 1e-12 and np.all(g["ext0"][ex == 0] == 0.0)
    theta = g["theta"].copy()
    mot = np.tile([float(g["v0"]), float(g["Dr"])], (N, 1))
    mot[ex != 0] = 0.0
    F1, ext1, _ = oracle.voronoi_spp_run_exclusions(pos, box, nn, nbr, theta, mot, pref, g["noise"], ex,
                                                    dt=float(g["dt"]))
    assert np.abs(pos - g["pos1"]).max() < 1e-11
    assert np.array_equal(canonical(nn, nbr), canonical(g["nn1"], g["nbr1"]))
    AP = oracle.voronoi_geometry(pos, box, nn, nbr)
    F, ext = oracle.apply_exclusions(oracle.voronoi_forces(pos, box, nn, nbr, AP, pref), ex)
    assert force_error(F, g["F1"]) < 1e-10
    assert force_error(ext[ex != 0], g["ext1"][ex != 0]) < 1e-10


def test_observables_golden():
    """The host formulas the observables tests use (mean and variance of q = P/sqrt(A), variances of
    A and P, minimum-image MSD and overlap) reproduce the reference's own reportq / reportVarq /
    reportVarAP and dynamicalFeatures outputs on the fixture."""
    g = _load("observables_N*.npz")[0]
    AP, box = g["AP1"], np.asarray(g["box"])
    q = AP[:, 1] / np.sqrt(AP[:, 0])
    d = g["pos1"] - g["pos0"]
    d -= box * np.round(d / box)
    r2 = np.sum(d * d, axis=1)
    ref = {"mean_q": q.mean(), "var_q": np.mean((q - q.mean()) ** 2),
           "var_A": np.mean((AP[:, 0] - AP[:, 0].mean()) ** 2), "var_P": np.mean((AP[:, 1] - AP[:, 1].mean()) ** 2),
           "msd": r2.mean(), "overlap": np.mean(np.sqrt(r2) < float(g["cutoff"]))}
    for k, v in ref.items():
        assert abs(v - float(g[k])) <= 1e-12 * max(1.0, abs(v)), k
