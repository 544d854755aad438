"""The outside probe's cage bound (csrc/cell.cu, cage_bits and k_probe),
restated in numpy with the kernel's float constants and margins, against
exact power cells from half-space intersections: whatever radius the cage
certifies holds the cell, and for jittered-lattice neighbourhoods it
certifies a radius close to the cell's own.  No GPU."""
import numpy as np
import pytest

scipy_spatial = pytest.importorskip("scipy.spatial")

F = np.float32
COS_C = F(0.882947592858927)    # cos(28 deg), the covering radius 27.57 deg with a margin
SIN2_C = F(0.2204035482646266)  # sin(28 deg)^2


def directions():
    out = []
    for z in (-1, 0, 1):
        for y in (-1, 0, 1):
            for x in (-1, 0, 1):
                if (x, y, z) == (0, 0, 0):
                    continue
                nnz = (x != 0) + (y != 0) + (z != 0)
                out.append((F(x), F(y), F(z), F([1.0, 0.70710678, 0.57735027][nnz - 1])))
    return out


DIRS = directions()


def test_stencil_covers_the_sphere_within_the_cage_angle():
    d = np.array([[x, y, z] for x, y, z, _ in DIRS], float)
    d /= np.linalg.norm(d, axis=1)[:, None]
    rng = np.random.default_rng(0)
    u = rng.normal(size=(400_000, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    worst = np.degrees(np.arccos(np.clip((u @ d.T).max(axis=1), -1, 1))).max()
    assert 27.0 < worst < 27.6 < 28.0


def cage_certifies(nb, w_s, w, r):
    """All 26 stencil directions bounded to r (the kernel's test, in float)."""
    inv_r = F(1.0 / r) * F(1.001)
    mask = 0
    for b, wb in zip(nb, w):
        dx, dy, dz = F(b[0]), F(b[1]), F(b[2])
        d2 = dx * dx + dy * dy + dz * dz
        ln = np.sqrt(d2)
        inv = F(1) / ln
        off = (d2 + (F(wb) - F(w_s))) * (F(0.5) * inv)
        q = off * inv_r
        nx, ny, nz = dx * inv, dy * inv, dz * inv
        for i, (x, y, z, inn) in enumerate(DIRS):
            ct = (x * nx + y * ny + z * nz) * inn - F(1e-3)
            lhs = COS_C * ct - q
            if lhs >= 0 and lhs * lhs >= SIN2_C * (F(1) - ct * ct):
                mask |= 1 << i
    return mask == (1 << 26) - 1


def cell_radius(nb, w_s, w):
    """Largest distance from the seed (at the origin) to a vertex of its
    power cell: x . n_b <= (|b|^2 + w_b - w_s) / (2 |b|), the reference's
    bisector (ConvexCell.cl:321-328), in a large box."""
    hs = []
    for b, wb in zip(nb, w):
        ln = np.linalg.norm(b)
        hs.append(np.r_[b / ln, -(ln * ln + wb - w_s) / (2 * ln)])
    for k in range(3):
        e = np.zeros(3)
        e[k] = 1
        hs.append(np.r_[e, -1e4])
        hs.append(np.r_[-e, -1e4])
    cell = scipy_spatial.HalfspaceIntersection(np.array(hs), np.zeros(3))
    return np.sqrt((cell.intersections ** 2).sum(axis=1)).max()


def neighbourhoods(rng, count):
    lattice = np.array([(x, y, z) for x in (-1, 0, 1) for y in (-1, 0, 1) for z in (-1, 0, 1)
                        if (x, y, z) != (0, 0, 0)], float) * 10
    for t in range(count):
        kind = t % 3
        if kind == 0:  # a jittered lattice around the seed
            nb = lattice + rng.uniform(-2.5, 2.5, lattice.shape) - rng.uniform(-2.5, 2.5, 3)
        elif kind == 1:  # i.i.d. uniform
            nb = rng.uniform(-15, 15, (int(rng.integers(20, 90)), 3))
        else:  # few and flattened: some directions uncovered
            nb = rng.uniform(-15, 15, (int(rng.integers(8, 30)), 3)) * np.array([1, 1, rng.uniform(0.3, 1)])
        nb = nb[np.linalg.norm(nb, axis=1) > 0.5]
        w = rng.uniform(0, 10, len(nb))
        w_s = rng.uniform(0, 10)
        # only cells that cannot be empty, as the probe requires
        if w_s - w.min() < 0.999 * np.linalg.norm(nb, axis=1).min() ** 2:
            yield kind, nb, w_s, w


def test_cage_never_certifies_less_than_the_cell():
    rng = np.random.default_rng(1)
    checked = 0
    for kind, nb, w_s, w in neighbourhoods(rng, 240):
        radius = cell_radius(nb, w_s, w)
        assert not cage_certifies(nb, w_s, w, radius * 0.999), (kind, radius)
        checked += 1
    assert checked > 150


def test_cage_certifies_jittered_lattice_cells():
    rng = np.random.default_rng(2)
    ratios = []
    for kind, nb, w_s, w in neighbourhoods(rng, 120):
        if kind != 0:
            continue
        radius = cell_radius(nb, w_s, w)
        ratios.append(cage_certifies(nb, w_s, w, 1.6 * radius))
    assert np.mean(ratios) > 0.9
