"""Seeded synthetic inputs of the benchmark configurations.

Seeds come out in the reference frame: positions in [0,1]^3 scaled x1000,
weights (squared units) scaled x1e6, float32 xyzw rows.
"""
from __future__ import annotations

import numpy as np

SCALE = 1000.0


def uniform(n: int, seed: int = 1) -> np.ndarray:
    """n i.i.d. U[0,1]^3 seeds, weights 0."""
    rng = np.random.default_rng(seed)
    x = np.zeros((n, 4), np.float32)
    x[:, :3] = (rng.random((n, 3)) * SCALE).astype(np.float32)
    return x


def jittered_lattice(m: int, seed: int = 2, jitter: float = 0.25, weights: bool = True,
                     wmax_h2: float = 0.1) -> np.ndarray:
    """m^3 seeds on the lattice of spacing h = 1/m, each coordinate perturbed
    by U[-jitter*h, jitter*h]; weights U[0, wmax_h2 * h^2] as float32."""
    rng = np.random.default_rng(seed)
    h = 1.0 / m
    idx = np.arange(m, dtype=np.float64)
    g = np.stack(np.meshgrid(idx, idx, idx, indexing="ij"), -1).reshape(-1, 3)
    p = (g + 0.5) * h + rng.uniform(-jitter * h, jitter * h, size=g.shape)
    x = np.zeros((len(p), 4), np.float32)
    x[:, :3] = (np.clip(p, 0.0, 1.0) * SCALE).astype(np.float32)
    if weights:
        w = rng.uniform(0.0, wmax_h2 * h * h, size=len(p)).astype(np.float32)
        x[:, 3] = (w.astype(np.float64) * SCALE * SCALE).astype(np.float32)
    return x


def poisson_disk(n: int, seed: int = 3, rfac: float = 0.7, max_tries: int = 60) -> np.ndarray:
    """Dart throwing in [0,1]^3 with minimum distance r = rfac * n^(-1/3),
    accelerated by a background grid of cell r/sqrt(3) (one dart per cell).
    Returns up to n seeds (fewer when the darts saturate)."""
    rng = np.random.default_rng(seed)
    r = rfac * n ** (-1.0 / 3.0)
    cell = r / np.sqrt(3.0)
    G = int(np.ceil(1.0 / cell))
    occ = -np.ones((G, G, G), np.int64)
    pts = np.zeros((n, 3), np.float64)
    count = 0
    r2 = r * r
    batch = max(4096, n // 8)
    tries = 0
    while count < n and tries < max_tries:
        tries += 1
        cand = rng.random((batch, 3))
        ci = np.minimum((cand / cell).astype(np.int64), G - 1)
        # greedy, in order: a candidate is kept if no kept dart lies within r
        for k in range(batch):
            if count >= n:
                break
            i, j, l = ci[k]
            if occ[i, j, l] >= 0:
                continue
            p = cand[k]
            ok = True
            for di in (-2, -1, 0, 1, 2):
                ii = i + di
                if ii < 0 or ii >= G:
                    continue
                for dj in (-2, -1, 0, 1, 2):
                    jj = j + dj
                    if jj < 0 or jj >= G:
                        continue
                    for dl in (-2, -1, 0, 1, 2):
                        ll = l + dl
                        if ll < 0 or ll >= G:
                            continue
                        q = occ[ii, jj, ll]
                        if q >= 0:
                            d = pts[q] - p
                            if d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < r2:
                                ok = False
                                break
                    if not ok:
                        break
                if not ok:
                    break
            if ok:
                occ[i, j, l] = count
                pts[count] = p
                count += 1
    x = np.zeros((count, 4), np.float32)
    x[:, :3] = (pts[:count] * SCALE).astype(np.float32)
    return x


def to_unit(xyzw: np.ndarray) -> np.ndarray:
    """Reference-frame moments (m*x, m*y, m*z, m) back to [0,1]^3 units."""
    out = np.asarray(xyzw, np.float64).copy()
    out[..., :3] *= 1.0 / SCALE ** 4
    out[..., 3] *= 1.0 / SCALE ** 3
    return out
