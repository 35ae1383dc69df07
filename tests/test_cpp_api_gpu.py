"""The C++ class API (cellgpu_b200/cpp/cellgpu.hpp: Simulation, VoronoiQuadraticEnergy,
VoronoiQuadraticEnergyWithTension, VertexQuadraticEnergy, selfPropelledParticleDynamics,
brownianParticleDynamics, EnergyMinimizerFIRE) against the Python API on the same deterministic states.

Tolerances (written here): energies and forces of one state 1e-12 relative / absolute (same
kernels); trajectories after 50 steps with device noise 1e-9 (floating-point atomics order);
FIRE energies 1e-9 relative; T1 flip counts equal.
"""
import json
import math
import os
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
EXE = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "cellgpu_b200", "cpp", "api_check")


def _r2(n, L):
    a1, a2 = 0.7548776662466927, 0.5698402909980532
    i = np.arange(1, n + 1, dtype=np.float64)
    x, y = 0.5 + a1 * i, 0.5 + a2 * i
    return np.stack([(x - np.floor(x)) * L, (y - np.floor(y)) * L], axis=1)


def _golden(n):
    x = 0.5 + 0.6180339887498949 * np.arange(n, dtype=np.float64)
    return 2.0 * math.pi * (x - np.floor(x))


def _rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


def test_cpp_class_api_matches_python(cglib):
    from cellgpu_b200 import FireParams, VertexBatch, VoronoiBatch
    assert os.path.exists(EXE), "build the C++ programs (cellgpu_b200.build.build_cpp)"
    run = subprocess.run([EXE, "400", "240"], capture_output=True, text=True, timeout=600)
    assert run.returncode == 0, run.stderr
    d = json.loads(run.stdout.strip().splitlines()[-1])

    n = 400
    L = math.sqrt(n)
    b = VoronoiBatch([n], [(L, L)])
    b.set_seed(13377)
    b.set_positions(_r2(n, L))
    b.set_directors(_golden(n))
    b.set_preferences(np.tile([1.0, 3.8], (n, 1)))
    b.triangulate()
    b.compute_forces()
    v = d["voronoi"]
    assert _rel(b.energies()[0], v["E0"]) < 1e-12
    assert np.abs(b.forces()[:4].ravel() - np.array(v["F0"])).max() < 1e-12
    b.set_motility(np.tile([0.1, 1.0], (n, 1)))
    b.spp_run(50, dt=0.01)
    assert np.abs(b.positions()[:4].ravel() - np.array(v["P_spp"])).max() < 1e-9
    b.fire_minimize(FireParams.defaults(force_cutoff=1e-10, max_iterations=10000))
    b.compute_forces()
    assert _rel(b.energies()[0], v["E_fire"]) < 1e-9

    # VoronoiQuadraticEnergyWithTension through both APIs
    from cellgpu_b200 import VoronoiQuadraticEnergyWithTension
    t = VoronoiQuadraticEnergyWithTension(n, 1.0, 3.8, True)
    t.setCellPositions(_r2(n, L))
    t.setCellType(np.arange(n) % 2)
    t.setSurfaceTension(0.2)
    t.setUseSurfaceTension(True)
    assert _rel(t.computeEnergy(), d["tension"]["E_simple"]) < 1e-12
    assert np.abs(t.returnForces()[:4].ravel() - np.array(d["tension"]["F_simple"])).max() < 1e-12
    t.setSurfaceTension([0.0, 0.35, 0.35, 0.0])
    assert _rel(t.computeEnergy(), d["tension"]["E_matrix"]) < 1e-12
    assert d["tension"]["E_matrix"] > d["tension"]["E_simple"] > v["E0"]

    nc = 240
    Lv = math.sqrt(nc)
    vb = VertexBatch([nc], [(Lv, Lv)])
    vb.set_seed(13377)
    vb.from_cells(_r2(nc, Lv))
    vb.set_t1_threshold(0.04)
    vb.set_preferences(np.tile([1.0, 3.8], (nc, 1)))
    vb.compute_forces()
    x = d["vertex"]
    assert _rel(vb.energies()[0], x["E0"]) < 1e-12
    vb.brownian_run(50, dt=0.005, mu=1.0, T=1e-3)
    assert np.abs(vb.positions()[:4].ravel() - np.array(x["P_brownian"])).max() < 1e-9
    assert vb.counters()["t1_flips"] == x["t1_flips"]
    vb.fire_minimize(FireParams.defaults(force_cutoff=1e-10, max_iterations=10000))
    vb.compute_forces()
    assert _rel(vb.energies()[0], x["E_fire"]) < 1e-9
