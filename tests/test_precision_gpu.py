"""The FP32 clipping loops (rpd_params.precision) against the FP64 one.

RPD_PRECISION_MIXED keeps the clipping state in float and escalates every
half-space, vertex and radius test that lies within its rigorous error bound
of the decision threshold to FP64, recomputed from the FP64 planes: every
decision is the FP64 clipping's, and the FP64 vertices are rebuilt from the
same planes before the restriction and integration, so statuses, moments,
Hessian rows and used cells are the FP64 mode's bit for bit -- and within
the FP64 oracle's 1e-5 (tests/parity.py).  RPD_PRECISION_FP32 (float planes,
no escalation) is the comparison point: its results are only checked to be
close."""
import numpy as np
import pytest

import oracle
from parity import assert_parity, compare
from seeds_util import clustered, jittered, uniform

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rpd():
    import rpd as m

    m.default_context()
    return m


def oracle_grid(g):
    a = g.arrays()
    return oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])


def solve(rpd, x, grid=None, **kw):
    s = rpd.Solver().set_points(x)
    if grid is not None:
        s.set_grid(grid)
    s.launch(**kw)
    out = (s.moments().copy(), s.status().copy(), s.stats())
    s.close()
    return out


CASES = {
    "weighted_blob40": lambda rpd: (jittered(30, seed=5, weights=True), rpd.Grid.blob(40, 5, 2),
                                    dict(K=50, P=30, V=40, T=100)),
    "uniform_cube": lambda rpd: (uniform(20000, seed=1), None, dict(K=20, P=25, V=30)),
    "voronoi_blob50_k70": lambda rpd: (uniform(30000, seed=3), rpd.Grid.blob(50, 5, 7), dict(K=70, P=30, V=40, T=100)),
    "small_caps_retries": lambda rpd: (jittered(20, seed=9, weights=True), rpd.Grid.blob(30, 5, 3),
                                       dict(K=12, P=10, V=12, T=8)),
    "clustered": lambda rpd: (clustered(20000, seed=4), None, dict(K=30, P=40, V=60)),
}


def _lattice():
    g = np.stack(np.meshgrid(*[np.arange(20) * 50.0 + 25.0] * 3, indexing="ij"), -1).reshape(-1, 3)
    x = np.zeros((len(g), 4), np.float32)
    x[:, :3] = g
    return x


CASES["lattice_ties"] = lambda rpd: (_lattice(), None, dict(K=26, P=30, V=40))


@pytest.mark.parametrize("case", sorted(CASES))
def test_mixed_equals_fp64_bit_for_bit(rpd, case):
    x, g, kw = CASES[case](rpd)
    m0, s0, st0 = solve(rpd, x, g, precision=rpd.PRECISION_FP64, **kw)
    m1, s1, st1 = solve(rpd, x, g, precision=rpd.PRECISION_MIXED, **kw)
    assert np.array_equal(s0, s1), f"{int((s0 != s1).sum())} statuses differ"
    assert np.array_equal(m0, m1), f"{int((m0 != m1).any(1).sum())} cells differ"
    assert [p["cells"] for p in st0["passes"]] == [p["cells"] for p in st1["passes"]]


def test_mixed_parity_with_oracle_and_escalations(rpd):
    g = rpd.Grid.blob(40, 5, 2)
    x = jittered(30, seed=5, weights=True)
    kw = dict(K=50, P=30, V=40, T=100)
    s = rpd.Solver().set_points(x).set_grid(g)
    s.launch(precision=rpd.PRECISION_MIXED, **kw)
    got, gst = s.moments(), s.status()
    ref, rst = oracle.solve(x.astype(np.float64), grid=oracle_grid(g), use_double=True, knn_mode=1, **kw)
    assert_parity(compare(got, gst, ref, rst))
    s.launch(precision=rpd.PRECISION_MIXED, flags=rpd.FLAG_COUNTERS, **kw)
    c = s.stats()["counters"]
    print(c)
    assert c["vertex_tests"] > 0
    # escalation is the exception: the float test decides nearly every vertex
    assert c["escalated_tests"] < 0.01 * c["vertex_tests"]
    assert np.array_equal(s.moments(), got)


def test_mixed_hessian_and_used_cells_equal_fp64(rpd):
    g = rpd.Grid.blob(32, 5, 2)
    x = jittered(20, seed=3, weights=True)
    out = []
    for prec in (rpd.PRECISION_FP64, rpd.PRECISION_MIXED):
        s = rpd.Solver().set_points(x).set_grid(g)
        s.launch(precision=prec, K=40, P=30, V=40, T=100, hessian_h=30, hessian_hc=4)
        h, hid = s.hessian(30, 4)
        s.launch(precision=prec, K=40, P=30, V=40, T=100, keep_distance=2, keep_volume=0.5)
        rows, ids = s.used()
        out.append((h.copy(), hid.copy(), rows.copy(), ids.copy()))
        s.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_plain_fp32_is_close(rpd):
    g = rpd.Grid.blob(40, 5, 2)
    x = jittered(30, seed=5, weights=True)
    kw = dict(K=50, P=30, V=40, T=100)
    m0, s0, _ = solve(rpd, x, g, precision=rpd.PRECISION_FP64, **kw)
    m2, s2, _ = solve(rpd, x, g, precision=rpd.PRECISION_FP32, **kw)
    met = compare(m2, s2, m0, s0)
    print(met)
    assert met["status_mismatch"] <= len(x) // 1000
    assert met["total_rel"] < 1e-5


@pytest.mark.parametrize("workload", ["weighted-1m", "voronoi-100k"])
def test_mixed_bench_workloads_full_size(rpd, workload):
    import os
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    cfg = bench.CONFIGS[workload]
    x = bench.make_seeds(cfg, 0)
    g = bench.make_grid(cfg)
    kw = dict(K=cfg["K"], P=cfg["P"], V=cfg["V"], T=cfg["T"])
    m0, s0, _ = solve(rpd, x, g, precision=rpd.PRECISION_FP64, **kw)
    m1, s1, _ = solve(rpd, x, g, precision=rpd.PRECISION_MIXED, **kw)
    assert np.array_equal(s0, s1)
    assert np.array_equal(m0, m1)
