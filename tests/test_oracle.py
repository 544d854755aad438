"""CPU tests of the oracle itself (no GPU)."""
import numpy as np
import pytest

import oracle
from seeds_util import jittered, uniform


def test_exact_knn_matches_reference_order_on_random_input():
    x = uniform(20000, seed=11).astype(np.float64)
    a = oracle.knn(x, 20, knn_mode=0)
    b = oracle.knn(x, 20, knn_mode=1)
    assert np.array_equal(a, b)


@pytest.mark.skipif(not oracle.has_reference_kernels(), reason="reference kernels not built here")
@pytest.mark.parametrize("use_double", [0, 1])
def test_restatement_bitexact_with_reference_kernels_no_grid(use_double):
    x = jittered(22, seed=4, weights=True).astype(np.float64)
    b1, s1 = oracle.solve(x, K=20, P=25, V=30, kernels=1, use_double=use_double)
    b0, s0 = oracle.solve(x, K=20, P=25, V=30, kernels=0, use_double=use_double)
    assert np.array_equal(s0, s1)
    assert np.array_equal(b0, b1)


def test_unit_cube_volume_fp64():
    x = uniform(5000, seed=3).astype(np.float64)
    b, s = oracle.solve(x, K=30, P=40, V=60, use_double=True)
    assert (s == oracle.SUCCESS).all()
    assert abs(b[:, 3].sum() - 1e9) < 1e-3


@pytest.mark.skipif(not oracle.has_reference_kernels(), reason="reference kernels not built here")
def test_restatement_bitexact_with_reference_kernels_empty_cells_in_a_domain():
    """Seeds far outside a blob domain whose weight empties their power cell:
    the restatement gives them the reference kernels' empty_cell status and
    every other cell the same bits (the configuration of the device test of
    the early exits outside the domain)."""
    import rpd

    g = rpd.Grid.blob(40, 5, 2)
    a = g.arrays()
    grid = oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])
    x = jittered(24, seed=11, weights=True)
    h2 = (1000.0 / 24) ** 2
    corner = (x[:, :3] < 150).all(axis=1) | (x[:, :3] > 850).all(axis=1)
    idx = np.where(corner)[0][::3]
    x[idx, 3] = 4 * h2
    x = x.astype(np.float64)
    kw = dict(grid=grid, K=50, P=30, V=40, T=100, use_double=True)
    b1, s1 = oracle.solve(x, kernels=1, **kw)
    b0, s0 = oracle.solve(x, kernels=0, **kw)
    assert np.array_equal(s0, s1)
    assert np.array_equal(b0, b1)
    assert (s0[idx] == 6).sum() > len(idx) // 2


def _margin_cell_case():
    """A weighted seed at x = 999.95 next to a lighter neighbour 0.95 away:
    its power cell (the reference adds the weight to the squared distance)
    lies entirely past x = 1000.05, inside the 0.1 margin the box has with a
    domain (voronoi.cpp:929), so its voxel range is empty and the
    restriction finds no start corner (ConvexCell.cl:924-1055)."""
    import rpd

    from seeds_util import jittered

    g = rpd.Grid.blob(50, 5, 2)
    a = g.arrays()
    ga = oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])
    x = jittered(20, seed=3, weights=True).astype(np.float64)
    i = int(np.argmin(np.abs(x[:, 0] - 975) + np.abs(x[:, 1] - 500) + np.abs(x[:, 2] - 500)))
    x = np.vstack([x, [[999.95, x[i, 1], x[i, 2], 1.0925]]])
    x[i] = [999.0, x[i, 1], x[i, 2], 0.0]
    return g, ga, x


@pytest.mark.skipif(not oracle.has_reference_kernels(), reason="reference kernels not built here")
def test_cell_in_the_box_margin_has_no_start_corner():
    """Known answer of the reference's kernels: find_another_beginning_vertex
    (7) for a cell entirely in the box margin past the grid; the restatement
    agrees bit for bit."""
    _, ga, x = _margin_cell_case()
    kw = dict(grid=ga, K=30, P=30, V=40, T=100, use_double=True)
    b1, s1 = oracle.solve(x, kernels=1, **kw)
    b0, s0 = oracle.solve(x, kernels=0, **kw)
    assert s1[-1] == 7 and (b1[-1] == 0).all()
    assert np.array_equal(s0, s1) and np.array_equal(b0, b1)
