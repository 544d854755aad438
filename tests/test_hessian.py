"""--hessian on the CPU (no GPU): the oracle's facet-area rows pinned bit for
bit against the reference's own kernels (ConvexCell.cl:621-678,1133-1150)
compiled for the host, and their geometric invariants."""
import numpy as np
import pytest

import oracle
from seeds_util import jittered

needs_ref = pytest.mark.skipif(not oracle.has_reference_kernels(), reason="reference kernels not built here")


@pytest.fixture(scope="module")
def blob():
    import rpd

    rpd.lib()
    g = rpd.Grid.blob(24, 5, 2)
    a = g.arrays()
    return oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])


@needs_ref
@pytest.mark.parametrize("hc", [1, 4])
@pytest.mark.parametrize("with_grid", [False, True])
def test_hessian_restatement_bitexact_with_reference_kernels(blob, hc, with_grid):
    x = jittered(12, seed=3, weights=True).astype(np.float64)
    g = blob if with_grid else None
    kw = dict(grid=g, H=40, HC=hc, K=30, P=30, V=40, T=60, knn_mode=1)
    b0, s0, h0, i0 = oracle.solve_hessian(x, kernels=0, **kw)
    b1, s1, h1, i1 = oracle.solve_hessian(x, kernels=1, **kw)
    assert np.array_equal(s0, s1)
    assert np.array_equal(b0, b1)
    assert np.array_equal(i0, i1)
    assert np.array_equal(h0, h1)
    assert (i0[:, 0] >= 0).sum() > len(x) // 5  # cells with at least one facet (many lie outside the blob)


@needs_ref
def test_hessian_overflow_matches_reference_kernels(blob):
    x = jittered(10, seed=5, weights=True).astype(np.float64)
    kw = dict(grid=blob, H=6, HC=1, K=30, P=30, V=40, T=60, knn_mode=1)
    _, s0, h0, i0 = oracle.solve_hessian(x, kernels=0, **kw)
    _, s1, h1, i1 = oracle.solve_hessian(x, kernels=1, **kw)
    assert (s0 == 10).sum() > 0  # hessian_overflow
    assert np.array_equal(s0, s1) and np.array_equal(i0, i1) and np.array_equal(h0, h1)


def test_hessian_areas_are_symmetric_and_close_the_cells():
    """Without a domain: a facet's area seen from both of its cells agrees,
    and in the unit box every cell's interior facets plus its box faces
    close it (the divergence theorem on the cell)."""
    x = jittered(8, seed=7, weights=True).astype(np.float64)
    _, st, h, ids = oracle.solve_hessian(x, H=60, HC=1, K=40, P=40, V=60)
    assert (st == oracle.SUCCESS).all()
    area = {}
    for i in range(len(x)):
        for a, j in zip(h[i], ids[i]):
            if j < 0:
                break
            area[(i, int(j))] = a
    for (i, j), a in area.items():
        assert (j, i) in area
        assert abs(area[(j, i)] - a) <= 1e-9 * max(a, 1.0)
