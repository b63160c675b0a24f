"""Shared helpers for the parity tests."""
import numpy as np


def degree_begin(width, depth):
    db = [0]
    for _ in range(depth + 1):
        db.append(1 + width * db[-1])
    return db


def level_rel_err(got, want, width, depth):
    """max over rows and levels of ||got_k - want_k||_inf / ||want_k||_inf.

    Per-level normwise relative error; levels whose reference is exactly zero
    fall back to the absolute error.
    """
    got = np.asarray(got, dtype=np.float64).reshape(-1, np.shape(got)[-1])
    want = np.asarray(want, dtype=np.float64).reshape(-1, np.shape(want)[-1])
    db = degree_begin(width, depth)
    worst = 0.0
    for k in range(depth + 1):
        g = got[:, db[k]:db[k + 1]]
        w = want[:, db[k]:db[k + 1]]
        num = np.max(np.abs(g - w), axis=1)
        den = np.max(np.abs(w), axis=1)
        rel = np.where(den > 0, num / np.where(den > 0, den, 1.0), num)
        worst = max(worst, float(np.max(rel)) if rel.size else 0.0)
    return worst


def level_scaled(rng, width, depth, batch, unit=True, dtype=np.float64):
    """Level-0 coefficient 1, level-k coefficients N(0,1)/k! (the FMA sweep inputs)."""
    db = degree_begin(width, depth)
    x = np.zeros((batch, db[depth + 1]))
    fact = 1.0
    for k in range(depth + 1):
        if k > 0:
            fact *= k
        x[:, db[k]:db[k + 1]] = rng.standard_normal((batch, db[k + 1] - db[k])) / fact
    if unit:
        x[:, 0] = 1.0
    return x.astype(dtype)
