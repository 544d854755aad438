"""--hessian on the device against the FP64 oracle (ConvexCell.cl:621-678,
1133-1150): the same facets per row, in the same order, with the same
neighbours; areas within 1e-5 (relative, floor 1 squared unit) and facet
centroids within 1e-4 reference-frame units.  A facet whose area lies
within that tolerance of the reference's 0.2 cut may be kept by one side
only; nothing else may differ."""
import numpy as np
import pytest

import oracle
from seeds_util import jittered

pytestmark = pytest.mark.gpu

AREA_RTOL = 1e-5
CENTROID_TOL = 1e-4
CUT = 0.2


@pytest.fixture(scope="module")
def rpd():
    import rpd as m

    m.default_context()
    return m


def oracle_grid(g):
    a = g.arrays()
    return oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])


def rows(vals, ids, hc, i):
    out = []
    for k in range(ids.shape[1]):
        j = int(ids[i, k])
        if j < 0:
            break
        out.append((j, vals[i, k] if hc == 1 else vals[i, k, :]))
    return out


def area_of(v, hc):
    return float(v if hc == 1 else v[3])


def near_cut(a):
    return abs(a - CUT) <= AREA_RTOL * max(abs(a), 1.0)


def compare_rows(gv, gi, ov, oi, hc, check):
    bad = []
    for i in check:
        g = rows(gv, gi, hc, i)
        o = rows(ov, oi, hc, i)
        if [j for j, _ in g] != [j for j, _ in o]:
            g = [(j, v) for j, v in g if not near_cut(area_of(v, hc))]
            o = [(j, v) for j, v in o if not near_cut(area_of(v, hc))]
            if [j for j, _ in g] != [j for j, _ in o]:
                bad.append((i, "ids", [j for j, _ in g], [j for j, _ in o]))
                continue
        for (j, a), (_, b) in zip(g, o):
            aa, ab = area_of(a, hc), area_of(b, hc)
            if abs(aa - ab) > AREA_RTOL * max(abs(ab), 1.0):
                bad.append((i, "area", j, aa, ab))
            if hc == 4:
                ca, cb = np.asarray(a[:3]) / aa, np.asarray(b[:3]) / ab
                if np.abs(ca - cb).max() > CENTROID_TOL:
                    bad.append((i, "centroid", j, ca, cb))
    assert not bad, bad[:5]


def solve_both(rpd, x, g, H, hc, flags=0, K=40, P=40, V=60, T=100):
    s = rpd.Solver().set_points(x)
    if g is not None:
        s.set_grid(g)
    s.launch(rpd.Params.default(K=K, P=P, V=V, T=T, hessian_h=H, hessian_hc=hc, flags=flags))
    gv, gi = s.hessian(H, hc)
    ob, ost, ov, oi = oracle.solve_hessian(x.astype(np.float64), grid=oracle_grid(g) if g is not None else None,
                                           H=H, HC=hc, K=K, P=P, V=V, T=T, knn_mode=1)
    return s, gv, gi, ob, ost, ov, oi


@pytest.mark.parametrize("hc", [1, 4])
def test_hessian_no_domain(rpd, hc):
    x = jittered(14, seed=2, weights=True)
    s, gv, gi, _, ost, ov, oi = solve_both(rpd, x, None, 40, hc)
    st = s.status()
    assert np.array_equal(st, ost)
    compare_rows(gv, gi, ov, oi, hc, range(len(x)))
    assert (gi[:, 0] >= 0).all()


@pytest.mark.parametrize("hc", [1, 4])
@pytest.mark.parametrize("ref_apex", [False, True])
def test_hessian_blob_domain(rpd, hc, ref_apex):
    """The restricted facets: inner-apex facet pieces (default) and the
    reference's cone clipping (reference apex)."""
    x = jittered(16, seed=4, weights=True)
    g = rpd.Grid.blob(40, 5, 3)
    flags = rpd.FLAG_REFERENCE_APEX if ref_apex else 0
    s, gv, gi, _, ost, ov, oi = solve_both(rpd, x, g, 40, hc, flags=flags)
    st = s.status()
    assert np.array_equal(st, ost)
    compare_rows(gv, gi, ov, oi, hc, range(len(x)))
    assert (gi[:, 0] >= 0).sum() > len(x) // 10  # most seeds lie outside the blob


def test_hessian_overflow(rpd):
    x = jittered(12, seed=6, weights=True)
    g = rpd.Grid.blob(32, 5, 2)
    s, gv, gi, _, ost, ov, oi = solve_both(rpd, x, g, 6, 1)
    st = s.status()
    assert (ost == 10).sum() > 0
    assert np.array_equal(st, ost)
    compare_rows(gv, gi, ov, oi, 1, range(len(x)))


def test_hessian_facets_are_symmetric_and_sum_to_the_surface(rpd):
    """A facet seen from both of its cells has one area; without a domain
    the facets of all cells plus the box faces cover 2x the interior
    surface and the box once."""
    x = jittered(10, seed=9, weights=True)
    s = rpd.Solver().set_points(x)
    s.launch(rpd.Params.default(K=40, P=40, V=60, hessian_h=50, hessian_hc=1))
    v, ids = s.hessian(50, 1)
    area = {}
    for i in range(len(x)):
        for k in range(50):
            j = int(ids[i, k])
            if j < 0:
                break
            area[(i, j)] = v[i, k]
    for (i, j), a in area.items():
        assert abs(area[(j, i)] - a) <= 1e-9 * max(a, 1.0)


def test_hessian_rows_with_used_cells(rpd):
    """Used cells: the rows of the used cells, neighbours as their compacted
    positions, light cells' rows and light or unused neighbours left out
    (compact_result, voronoi.cpp:594-629)."""
    x = jittered(14, seed=8, weights=True)
    g = rpd.Grid.blob(40, 5, 2)
    H, kv = 40, 0.001
    s = rpd.Solver().set_points(x).set_grid(g)
    s.launch(rpd.Params.default(K=40, P=40, V=60, keep_distance=1, keep_volume=kv, hessian_h=H, hessian_hc=1))
    rows_used, uids = s.used()
    gv, gi = s.hessian(H, 1)
    assert gv.shape[0] == len(uids)
    ob, ost, ov, oi = oracle.solve_hessian(x.astype(np.float64), grid=oracle_grid(g), H=H, HC=1, K=40, P=40, V=60,
                                           knn_mode=1)
    pos = {int(u): p for p, u in enumerate(uids)}
    ev = np.zeros_like(gv)
    ei = np.full_like(gi, -1)
    for p, u in enumerate(uids):
        if ob[u, 3] < kv:
            continue
        w = 0
        for k in range(H):
            j = int(oi[u, k])
            if j < 0:
                break
            if j not in pos or ob[j, 3] < kv:
                continue
            ei[p, w] = pos[j]
            ev[p, w] = ov[u, k]
            w += 1
    compare_rows(gv, gi, ev, ei, 1, range(len(uids)))
