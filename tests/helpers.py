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
