"""Seeded synthetic seed sets for the tests (reference frame [0,1000]^3)."""
import numpy as np


def uniform(n, seed=1):
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 4), np.float32)
    x[:, :3] = (rng.random((n, 3), dtype=np.float32) * np.float32(1000.0)).astype(np.float32)
    return x


def jittered(m, seed=2, weights=False):
    """m^3 points on a jittered lattice (spacing h = 1000/m, +-0.25h), with
    optional weights U[0, 0.1 h^2]."""
    rng = np.random.default_rng(seed)
    h = 1000.0 / m
    g = np.stack(np.meshgrid(np.arange(m), np.arange(m), np.arange(m), indexing="ij"), -1).reshape(-1, 3)
    p = (g + 0.5) * h + rng.uniform(-0.25 * h, 0.25 * h, size=g.shape)
    x = np.zeros((len(p), 4), np.float32)
    x[:, :3] = p.astype(np.float32)
    if weights:
        x[:, 3] = rng.uniform(0, 0.1 * h * h, size=len(p)).astype(np.float32)
    return x


def clustered(n, seed=3):
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 4), np.float32)
    centers = rng.random((8, 3)) * 800 + 100
    c = centers[rng.integers(0, 8, n)]
    x[:, :3] = np.clip(c + rng.normal(0, 40, (n, 3)), 0, 999.9).astype(np.float32)
    return x
