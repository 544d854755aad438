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


def poisson_disk(n: int, seed: int = 3, rfac: float = 0.7) -> np.ndarray:
    """Up to n seeds of [0,1]^3 (x1000) by seeded dart throwing with minimum
    distance r = rfac * n^(-1/3) (rpd_synth_poisson_disk, weights 0)."""
    import ctypes as C

    from . import lib

    L = lib()
    L.rpd_synth_poisson_disk.argtypes = [C.c_int, C.c_uint64, C.c_double, C.c_void_p]
    out = np.zeros((n, 4), np.float32)
    k = L.rpd_synth_poisson_disk(n, seed, rfac, C.c_void_p(out.ctypes.data))
    if k < 0:
        raise ValueError(f"rpd_synth_poisson_disk failed: {k}")
    return out[:k]


def to_unit(xyzw: np.ndarray) -> np.ndarray:
    """Reference-frame moments (m*x, m*y, m*z, m) back to [0,1]^3 units."""
    out = np.asarray(xyzw, np.float64).copy()
    out[..., :3] *= 1.0 / SCALE ** 4
    out[..., 3] *= 1.0 / SCALE ** 3
    return out


def uneven_batch(count: int, seed: int = 4, nmin: int = 1000, nmax: int = 200_000, gmin: int = 64, gmax: int = 160,
                 ks=(20, 50, 70)):
    """`count` independent diagram specs of the batched workload: seed counts
    log-uniform in [nmin, nmax]; positions uniform or jittered-lattice
    (alternating), weights U[0, 0.1 h^2] with h the diagram's spacing
    n^(-1/3); a seeded ellipsoid-blob domain of gmin..gmax voxels per axis; K
    from `ks`.  Returns dicts {xyzw, grid_size, grid_seed, K}."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(count):
        n = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        s = int(rng.integers(1 << 30))
        if i % 2 == 0:
            x = uniform(n, seed=s)
        else:
            m = max(2, int(round(n ** (1.0 / 3.0))))
            x = jittered_lattice(m, seed=s, weights=False)
        h = len(x) ** (-1.0 / 3.0)
        w = np.random.default_rng(s + 1).uniform(0.0, 0.1 * h * h, size=len(x))
        x[:, 3] = (w * SCALE * SCALE).astype(np.float32)
        specs.append({"xyzw": x, "grid_size": int(rng.integers(gmin, gmax + 1)), "grid_seed": int(rng.integers(1 << 20)),
                      "K": int(ks[int(rng.integers(len(ks)))])})
    return specs
