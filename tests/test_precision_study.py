"""Why the mixed-precision mode cannot meet a 1e-6 per-cell force error (CPU only).

A numpy restatement of the scatter-form force pass (every Voronoi vertex h_k of cell c contributes
g . dh_k/dr to c and to the two neighbours that define h_k, g = -dE_c/dh_k) is first pinned to the
oracle in FP64 (1e-12). Rounding one quantity of it to FP32 then shows where the error comes from
on a relaxed SPP state (p0 = 3.8, 300 steps from uniform positions), with the normalisation every
force tolerance of this suite uses, |dF_i| / max(|F_i|, RMS |F|):
  * the per-vertex derivative g rounded to FP32 (everything else FP64), or FP32 accumulation of
    FP64 terms, each leave a maximum near 1e-6 on 4096 cells and about 4e-6 on 16384 (the largest
    of more cells): near force balance a cell's force is the sum of ~18 terms about ten times larger
    than the RMS force, and FP32's unit roundoff of 6e-8 on each term leaves ~1e-6 and more;
  * a mode with FP32 in the force arithmetic therefore sits at a few 1e-6 per cell (the library's
    mixed mode, FP32 derivatives and contractions, is measured at about 5e-6 on the GPU), while its
    norm-wise error max|dF| / max|F| stays below 1e-6.
"""
import numpy as np
import pytest


def _relaxed(oracle, N=4096, steps=300, seed=1):
    L = float(np.sqrt(N))
    rng = np.random.default_rng(seed)
    pos = rng.random((N, 2)) * L
    th = rng.uniform(0, 2 * np.pi, N)
    nn, nbr = oracle.periodic_delaunay(pos, (L, L), 16)
    mot, pref = np.tile([0.1, 1.0], (N, 1)), np.tile([1.0, 3.8], (N, 1))
    noise = np.random.default_rng(seed + 1).standard_normal((steps, N))
    oracle.voronoi_spp_run(pos, (L, L), nn, nbr, th, mot, pref, noise)
    nn, nbr = oracle.periodic_delaunay(pos, (L, L), 16)
    return pos, (L, L), nn, nbr, pref


def _forces(pos, box, nn, nbr, pref, g32=False, acc32=False):
    """Scatter-form forces; g32 rounds g = -dE_c/dh_k to FP32, acc32 accumulates in FP32."""
    L = np.asarray(box)
    N = len(nn)
    c = np.repeat(np.arange(N), nn)
    k = np.concatenate([np.arange(z) for z in nn])
    z = nn[c]
    off = np.concatenate([[0], np.cumsum(nn)])
    ip, im = off[c] + (k + 1) % z, off[c] + (k - 1) % z
    nb, nbm = nbr[c, k], nbr[c, (k - 1) % z]
    md = lambda d: d - L * np.round(d / L)
    rb, ra = md(pos[nb] - pos[c]), md(pos[nbm] - pos[c])
    an, bn = (ra ** 2).sum(1), (rb ** 2).sum(1)
    den = 0.5 / (ra[:, 0] * rb[:, 1] - ra[:, 1] * rb[:, 0])
    h = np.stack([den * (an * rb[:, 1] - ra[:, 1] * bn), den * (ra[:, 0] * bn - an * rb[:, 0])], 1)
    hp, hm = h[ip], h[im]
    A, P = np.zeros(N), np.zeros(N)
    np.add.at(A, c, np.abs(0.5 * (h[:, 0] * hp[:, 1] - h[:, 1] * hp[:, 0])))
    np.add.at(P, c, np.sqrt(((hp - h) ** 2).sum(1)))
    Ad, Pd = (A - pref[:, 0])[c], (P - pref[:, 1])[c]
    u = hp - h
    u = u / np.maximum(np.sqrt((u ** 2).sum(1)), 1e-18)[:, None]
    dA = 0.5 * np.stack([hp[:, 1] - hm[:, 1], hm[:, 0] - hp[:, 0]], 1)
    g = -2.0 * (Ad[:, None] * dA + Pd[:, None] * (u[im] - u))
    if g32:
        g = g.astype(np.float32).astype(np.float64)
    hi = 2 * den * den
    t1, t2 = rb[:, 1] * an - ra[:, 1] * bn, rb[:, 0] * an - ra[:, 0] * bn
    d = [hi * (rb[:, 1] - ra[:, 1]) * t1, hi * (ra[:, 1] - rb[:, 1]) * t2, hi * (ra[:, 0] - rb[:, 0]) * t1,
         hi * (rb[:, 0] - ra[:, 0]) * t2]
    p, q = -ra, rb - ra
    q2 = (q ** 2).sum(1)
    u1, u2 = q[:, 1] * an - p[:, 1] * q2, q[:, 0] * an - p[:, 0] * q2
    e = [hi * (q[:, 1] - p[:, 1]) * u1, hi * (p[:, 1] - q[:, 1]) * u2, hi * (p[:, 0] - q[:, 0]) * u1,
         hi * (q[:, 0] - p[:, 0]) * u2]
    b = [1 - d[0] - e[0], -d[1] - e[1], -d[2] - e[2], 1 - d[3] - e[3]]
    con = lambda m: np.stack([g[:, 0] * m[0] + g[:, 1] * m[2], g[:, 0] * m[1] + g[:, 1] * m[3]], 1)
    tgt = np.concatenate([c, nbm, nb])
    vec = np.concatenate([con(d), con(e), con(b)])
    F = np.zeros((N, 2), np.float32 if acc32 else np.float64)
    perm = np.random.default_rng(0).permutation(len(tgt))  # an arbitrary arrival order
    np.add.at(F, tgt[perm], vec[perm].astype(F.dtype))
    return F.astype(np.float64)


def _err(F, Fr):
    s = np.sqrt(np.mean((Fr ** 2).sum(1)))
    dd = np.linalg.norm(F - Fr, axis=1)
    return float(np.max(dd / np.maximum(np.linalg.norm(Fr, axis=1), s))), float(dd.max() / np.linalg.norm(Fr, axis=1).max())


@pytest.fixture(scope="module")
def state(oracle):
    return _relaxed(oracle)


def test_restatement_matches_the_oracle(oracle, state):
    pos, box, nn, nbr, pref = state
    AP = oracle.voronoi_geometry(pos, box, nn, nbr)
    Fo = oracle.voronoi_forces(pos, box, nn, nbr, AP, pref)
    assert _err(_forces(pos, box, nn, nbr, pref), Fo)[0] < 1e-12


def test_fp32_force_terms_exceed_1e6_per_cell(state):
    pos, box, nn, nbr, pref = state
    F64 = _forces(pos, box, nn, nbr, pref)
    out = {}
    for name, kw in (("g", dict(g32=True)), ("accumulation", dict(acc32=True)), ("both", dict(g32=True, acc32=True))):
        out[name] = _err(_forces(pos, box, nn, nbr, pref, **kw), F64)
        print(f"FP32 {name}: per cell {out[name][0]:.2e}, norm-wise {out[name][1]:.2e}")
    # each source alone is within a factor of a few of 1e-6 on 4096 cells (the maximum grows with
    # N: 3.9e-6 and 4.2e-6 on 16384 cells); together they exceed it
    assert out["both"][0] > 1e-6
    assert min(out["g"][0], out["accumulation"][0]) > 3e-7
    assert all(v[1] < 1e-6 for v in out.values())
