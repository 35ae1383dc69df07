"""Shared test helpers: seeded monolayers and tolerance checks."""
import numpy as np


def monolayer(N, seed, L=None):
    L = float(np.sqrt(N)) if L is None else L
    rng = np.random.default_rng(seed)
    return rng.random((N, 2)) * L, (L, L)


def force_error(F, Fref):
    """max_i |F_i - Fref_i| / max(|Fref_i|, F_scale), F_scale = RMS |Fref| (the normalisation used for
    every force tolerance in this suite)."""
    F = np.asarray(F)
    Fref = np.asarray(Fref)
    scale = np.sqrt(np.mean(np.sum(Fref ** 2, axis=1)))
    den = np.maximum(np.linalg.norm(Fref, axis=1), scale)
    return float(np.max(np.linalg.norm(F - Fref, axis=1) / den))


def canonical(nn, nbr):
    out = np.full_like(nbr, -1)
    for i in range(len(nn)):
        z = int(nn[i])
        r = nbr[i, :z]
        s = int(np.argmin(r))
        out[i, :z] = np.roll(r, -s)
    return out


def jittered_lattice(nx, ny, jitter, seed):
    """Triangular lattice of unit-area cells in a rectangular periodic box, each point displaced by
    a uniform jitter (a well-conditioned state: no near-coincident points)."""
    rng = np.random.default_rng(seed)
    s = np.sqrt(2 / np.sqrt(3))
    pts = []
    for j in range(ny):
        for i in range(nx):
            pts.append(((i + 0.5 * (j % 2)) * s, j * s * np.sqrt(3) / 2))
    pts = np.array(pts) + rng.uniform(-jitter, jitter, (nx * ny, 2))
    box = (nx * s, ny * s * np.sqrt(3) / 2)
    pts[:, 0] %= box[0]
    pts[:, 1] %= box[1]
    return pts, box
