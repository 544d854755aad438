"""Used cells and compaction (voronoi.cpp:513-751, ConvexCell.cl:680-690,
756-809, 1118-1126) in the oracle: the restatement against the reference's
own kernels built with CUSED_CELL, and the structure of the marks (no GPU)."""
import numpy as np
import pytest

import oracle
from seeds_util import jittered


@pytest.fixture(scope="module")
def case():
    import rpd

    g = rpd.Grid.blob(20, 5, 2)
    a = g.arrays()
    grid = oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])
    x = jittered(18, seed=7, weights=True).astype(np.float64)
    return x, grid


@pytest.mark.skipif(not oracle.has_reference_kernels(), reason="reference kernels not built here")
@pytest.mark.parametrize("keep_distance,keep_volume", [(0, 1.0), (1, 1.0), (2, 1.0), (3, 1.0), (0, 0.0), (1, -1.0)])
def test_restatement_bitexact_with_reference_kernels(case, keep_distance, keep_volume):
    x, grid = case
    kw = dict(K=30, P=30, V=40, T=100, knn_mode=0, keep_distance=keep_distance, keep_volume=keep_volume)
    b1, s1, u1 = oracle.solve_used(x, grid, kernels=1, **kw)
    b0, s0, u0 = oracle.solve_used(x, grid, kernels=0, **kw)
    assert np.array_equal(s0, s1)
    assert np.array_equal(b0, b1)
    assert np.array_equal(u0, u1)
    assert u0.max() == max(keep_distance, 1 if (b0[:, 3] >= keep_volume).any() else 0)


def test_rings_grow_with_distance(case):
    x, grid = case
    kw = dict(K=30, P=30, V=40, T=100, keep_volume=1.0)
    us = [oracle.solve_used(x, grid, keep_distance=d, **kw)[2] for d in range(4)]
    b = oracle.solve_used(x, grid, keep_distance=0, **kw)[0]
    used = b[:, 3] >= 1.0
    assert np.array_equal(us[0] != 0, used)
    for d in range(1, 4):
        # every seed kept at distance d-1 is kept at d, with the same mark
        prev = us[d - 1] != 0
        assert np.array_equal(us[d][prev], us[d - 1][prev])
        assert (us[d] != 0).sum() > prev.sum()
        assert set(np.unique(us[d])) <= set(range(d + 1))


def test_compaction_marks_the_outer_ring(case):
    x, grid = case
    b, s, u = oracle.solve_used(x, grid, keep_distance=2, K=30, P=30, V=40, T=100, keep_volume=1.0)
    rows, perm = oracle.compact(b, u, 2, 1.0)
    assert len(rows) == (u != 0).sum() and np.all(np.diff(perm) > 0)
    outer = (u[perm] == 2) & (b[perm, 3] < 1.0)
    assert np.all(rows[outer, 3] == -100000.0)
    assert np.array_equal(rows[~outer], b[perm][~outer])
