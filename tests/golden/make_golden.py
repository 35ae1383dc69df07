"""Generate the golden fixtures in this folder from the reference's own CPU code.

The reference (abaso/cellGPU) ships no test vectors, so the fixtures are outputs of its CPU path,
compiled in place from its sources by oracle/Makefile.ref (with the DelaunayCGAL stand-in,
oracle/shim) into oracle/_ref/libcgref.so. Run from the repository root, where the reference
sources are available:

    make -C oracle -f Makefile.ref && python tests/golden/make_golden.py [voronoi vertex fire tension exclusions observables]

Each .npz holds the inputs and the reference's outputs of one case (small sizes, seeded).
"""
import contextlib
import io
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref_harness as R  # noqa: E402


def quiet():
    return contextlib.redirect_stdout(io.StringIO())


def voronoi_case(N, seed, steps, v0=0.05, dt=0.01):
    L = float(np.sqrt(N))
    rng = np.random.default_rng(seed)
    pos = rng.random((N, 2)) * L
    theta = rng.uniform(0, 2 * np.pi, N)
    with quiet():
        r = R.RefVoronoi(N)
        r.set_state(pos, theta)
        r.set_motility(v0, 1.0)
        F0, AP0, E0 = r.forces()
        _, _, nn0, nbr0 = r.state()
        r.spp_run(steps, dt, True)
        pos1, th1, nn1, nbr1 = r.state()
        F1, AP1, E1 = r.forces()
    noise = R.reproducible_normals(steps * N).reshape(steps, N)
    np.savez_compressed(os.path.join(HERE, f"voronoi_N{N}_s{seed}.npz"), N=N, box=np.array([L, L]), pos=pos,
                        theta=theta, v0=v0, Dr=1.0, dt=dt, steps=steps, noise=noise, F0=F0, AP0=AP0, E0=E0,
                        nn0=nn0, nbr0=nbr0, pos1=pos1, theta1=th1, nn1=nn1, nbr1=nbr1, F1=F1, AP1=AP1, E1=E1)


def exclusions_case(N=400, seed=9, steps=5, v0=0.05, dt=0.01, every=7):
    """Particle exclusions (voronoiModelBase::setExclusions): every `every`-th cell excluded; forces and
    external forces on the initial state, then `steps` SPP steps (local repair) and the same again."""
    L = float(np.sqrt(N))
    rng = np.random.default_rng(seed)
    pos = rng.random((N, 2)) * L
    theta = rng.uniform(0, 2 * np.pi, N)
    exes = (np.arange(N) % every == 3).astype(np.int32)
    with quiet():
        r = R.RefVoronoi(N)
        r.set_state(pos, theta)
        r.set_motility(v0, 1.0)
        r.set_exclusions(exes)
        F0, AP0, E0 = r.forces()
        ext0 = r.external_forces()
        r.spp_run(steps, dt, True)
        pos1, th1, nn1, nbr1 = r.state()
        F1, AP1, E1 = r.forces()
        ext1 = r.external_forces()
    noise = R.reproducible_normals(steps * N).reshape(steps, N)
    np.savez_compressed(os.path.join(HERE, f"exclusions_N{N}_s{seed}.npz"), N=N, box=np.array([L, L]), pos=pos,
                        theta=theta, v0=v0, Dr=1.0, dt=dt, steps=steps, noise=noise, exes=exes, F0=F0, ext0=ext0,
                        AP0=AP0, E0=E0, pos1=pos1, theta1=th1, nn1=nn1, nbr1=nbr1, F1=F1, ext1=ext1)


def observables_case(N=500, seed=11, steps=40, v0=0.3, dt=0.01):
    """The reference's observables (Simple2DCell::reportq / reportVarq / reportVarAP and
    dynamicalFeatures::computeMSD / computeOverlapFunction with cutoff 0.5) after `steps` SPP steps
    from seeded uniform positions, with the positions before and after and the reference's A/P."""
    L = float(np.sqrt(N))
    rng = np.random.default_rng(seed)
    pos = rng.random((N, 2)) * L
    theta = rng.uniform(0, 2 * np.pi, N)
    with quiet():
        r = R.RefVoronoi(N)
        r.set_state(pos, theta)
        r.set_motility(v0, 1.0)
        pos0, _, _, _ = r.state()
        r.spp_run(steps, dt, True)
        obs = r.observables(pos0, 0.5)
        pos1, th1, nn1, nbr1 = r.state()
        F1, AP1, E1 = r.forces()
    np.savez_compressed(os.path.join(HERE, f"observables_N{N}_s{seed}.npz"), N=N, box=np.array([L, L]), pos0=pos0,
                        pos1=pos1, nn1=nn1, nbr1=nbr1, AP1=AP1, cutoff=0.5,
                        **{k: np.float64(v) for k, v in obs.items()})


def vertex_case(Nc, steps, dt=0.005, T=1e-3, t1=0.04, seed=2):
    with quiet():
        rv = R.RefVertex(Nc)
    cp, vp, vn, vcn, cvn, cv = rv.state()
    rng = np.random.default_rng(seed)
    pref = np.stack([np.ones(Nc), rng.uniform(3.7, 3.9, Nc)], 1)
    with quiet():
        rv.set_preferences(pref)
        rv.set_t1(t1)
        F0, AP0, E0 = rv.forces()
        rv.brownian_run(steps, dt, T, 1.0)
        _, vp1, vn1, vcn1, cvn1, cv1 = rv.state()
        F1, AP1, E1 = rv.forces()
    noise = R.reproducible_normals(steps * 2 * rv.Nv).reshape(steps, rv.Nv, 2)
    L = float(np.sqrt(Nc))
    np.savez_compressed(os.path.join(HERE, f"vertex_Nc{Nc}.npz"), Nc=Nc, box=np.array([L, L]), vmax=rv.vmax,
                        cellpos=cp, vpos=vp, vn=vn, vcn=vcn, cvn=cvn, cv=cv, pref=pref, F0=F0, AP0=AP0, E0=E0,
                        dt=dt, T=T, t1=t1, steps=steps, noise=noise, vpos1=vp1, vn1=vn1, vcn1=vcn1, cvn1=cvn1,
                        cv1=cv1, F1=F1, AP1=AP1, E1=E1)


def fire_case(N, seed, vertex=False):
    L = float(np.sqrt(N))
    rng = np.random.default_rng(seed)
    if vertex:
        with quiet():
            rv = R.RefVertex(N)
            cp, vp, vn, vcn, cvn, cv = rv.state()
            rv.fire(force_cutoff=1e-10, max_iterations=3000)
            _, vp1, vn1, vcn1, cvn1, cv1 = rv.state()
            F1, AP1, E1 = rv.forces()
        np.savez_compressed(os.path.join(HERE, f"fire_vertex_Nc{N}.npz"), Nc=N, box=np.array([L, L]),
                            vmax=rv.vmax, vpos=vp, vn=vn, vcn=vcn, cvn=cvn, cv=cv, vpos1=vp1, F1=F1, AP1=AP1,
                            E1=E1, cutoff=1e-10, max_iterations=3000)
        return
    pos = rng.random((N, 2)) * L
    with quiet():
        r = R.RefVoronoi(N)
        r.set_state(pos, np.zeros(N))
        r.fire(force_cutoff=1e-10, max_iterations=3000)
        pos1, _, nn1, nbr1 = r.state()
        F1, AP1, E1 = r.forces()
    np.savez_compressed(os.path.join(HERE, f"fire_voronoi_N{N}_s{seed}.npz"), N=N, box=np.array([L, L]), pos=pos,
                        pos1=pos1, nn1=nn1, nbr1=nbr1, F1=F1, AP1=AP1, E1=E1, cutoff=1e-10, max_iterations=3000)


def tension_case(N, seed):
    """VoronoiQuadraticEnergyWithTension: three cell types, one gamma for unlike types and a
    symmetric tension matrix."""
    L = float(np.sqrt(N))
    rng = np.random.default_rng(seed)
    pos = rng.random((N, 2)) * L
    types = rng.integers(0, 3, N).astype(np.int32)
    pref = np.stack([np.ones(N), rng.uniform(3.7, 3.9, N)], 1)
    gammas = np.array([[0.0, 0.1, 0.3], [0.1, 0.0, 0.2], [0.3, 0.2, 0.0]])
    Fs, APs, Es = R.voronoi_tension_forces(pos, types, pref, gamma=0.15)
    Fm, APm, Em = R.voronoi_tension_forces(pos, types, pref, gammas=gammas)
    np.savez_compressed(os.path.join(HERE, f"tension_N{N}_s{seed}.npz"), N=N, box=np.array([L, L]), pos=pos,
                        types=types, pref=pref, gamma=0.15, gammas=gammas, F_simple=Fs, AP_simple=APs,
                        E_simple=Es, F_matrix=Fm, AP_matrix=APm, E_matrix=Em)


def vertex_tension_case(Nc, seed):
    """VertexQuadraticEnergyWithTension (CPU branch): three cell types, one gamma for unlike types
    and a symmetric tension matrix, on the reference's reproducible Delaunay-dual state. E is the
    quadratic part (the reference does not implement the tension energy)."""
    with quiet():
        rv = R.RefVertex(Nc)
    cp, vp, vn, vcn, cvn, cv = rv.state()
    rng = np.random.default_rng(seed)
    types = rng.integers(0, 3, Nc).astype(np.int32)
    pref = np.stack([np.ones(Nc), rng.uniform(3.7, 3.9, Nc)], 1)
    gammas = np.array([[0.0, 0.1, 0.3], [0.1, 0.0, 0.2], [0.3, 0.2, 0.0]])
    with quiet():
        rv.set_preferences(pref)
        rv.set_tension(types, gamma=0.15)
        Fs, APs, Es = rv.forces()
        rv.set_tension(types, gammas=gammas)
        Fm, APm, Em = rv.forces()
    L = float(np.sqrt(Nc))
    np.savez_compressed(os.path.join(HERE, f"vertex_tension_Nc{Nc}_s{seed}.npz"), Nc=Nc, box=np.array([L, L]),
                        vmax=rv.vmax, vpos=vp, vn=vn, vcn=vcn, cvn=cvn, cv=cv, types=types, pref=pref, gamma=0.15,
                        gammas=gammas, F_simple=Fs, AP_simple=APs, E_simple=Es, F_matrix=Fm, AP_matrix=APm,
                        E_matrix=Em)


if __name__ == "__main__":
    if not R.available():
        raise SystemExit("oracle/_ref/libcgref.so missing: make -C oracle -f Makefile.ref")
    cases = {
        "voronoi": lambda: (voronoi_case(300, 1, 20), voronoi_case(1000, 2, 10, v0=0.3)),
        "vertex": lambda: vertex_case(400, 15),
        "fire": lambda: (fire_case(200, 3), fire_case(200, 4, vertex=True)),
        "tension": lambda: (tension_case(400, 5), vertex_tension_case(300, 7)),
        "exclusions": lambda: exclusions_case(),
        "observables": lambda: observables_case(),
    }
    for name in sys.argv[1:] or list(cases):  # python make_golden.py [case ...]
        cases[name]()
    print("golden fixtures written to", HERE)
