"""Device restricted power cells against the FP64 oracle (the reference's
USE_DOUBLE algorithm restated), through the C ABI."""
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


def solve_gpu(rpd, x, grid=None, **kw):
    s = rpd.Solver().set_points(x)
    if grid is not None:
        s.set_grid(grid)
    s.launch(**kw)
    return s.moments(), s.status(), s.stats()


def run_case(rpd, x, grid=None, K=20, P=25, V=30, T=100, **kw):
    got, gst, stats = solve_gpu(rpd, x, grid, K=K, P=P, V=V, T=T, **kw)
    ref, rst = oracle.solve(x.astype(np.float64), grid=oracle_grid(grid) if grid is not None else None, K=K, P=P,
                            V=V, T=T, use_double=True, knn_mode=1)
    met = compare(got, gst, ref, rst)
    print(met, stats["passes"])
    rel = np.abs(got[:, 3] - ref[:, 3]) / np.maximum(np.abs(ref[:, 3]), 1e-3)
    for i in np.argsort(rel)[-3:]:
        print("  worst", i, "m_gpu", got[i, 3], "m_ref", ref[i, 3], "rel", rel[i], "status", gst[i], rst[i])
    return met, got, gst, ref, rst, stats


def test_unit_cube_voronoi(rpd):
    met, got, gst, *_ = run_case(rpd, uniform(20000, seed=1), K=20, P=25, V=30)
    assert_parity(met)
    assert abs(got[:, 3].sum() / 1e9 - 1) < 1e-6


def test_weighted_lattice_blob(rpd):
    g = rpd.Grid.blob(40, 5, 2)
    met, *_ = run_case(rpd, jittered(30, seed=5, weights=True), grid=g, K=50, P=30, V=40)
    assert_parity(met)


def test_voronoi_blob_k70(rpd):
    g = rpd.Grid.blob(50, 5, 7)
    met, got, gst, ref, rst, stats = run_case(rpd, uniform(30000, seed=3), grid=g, K=70, P=30, V=40)
    assert_parity(met)
    assert abs(got[:, 3].sum() / g.getVolume() - 1) < 1e-6


def test_inset_cube_domain(rpd):
    g = rpd.Grid.cube(16)
    x = jittered(25, seed=9)
    met, got, gst, ref, rst, _ = run_case(rpd, x, grid=g, K=50, P=30, V=40)
    bad = np.where(~np.isfinite(got[:, 3]) | (gst != rst))[0]
    if len(bad):
        s = rpd.Solver().set_points(x).set_grid(g)
        np.set_printoptions(linewidth=200, precision=6, suppress=False)
        for i in bad[:2]:
            print("cell", i, "seed", x[i], "gpu", got[i], gst[i], "ref", ref[i], rst[i])
            for r in s.trace_cell(int(i), K=50, P=45, V=60, T=150):
                print("  ", rpd.Solver.TRACE_KINDS.get(int(r[0]), r[0]), r[1:].tolist())
    assert_parity(met)
    assert abs(got[:, 3].sum() / g.getVolume() - 1) < 1e-6


def test_retry_passes_small_caps(rpd):
    # caps far too small: overflow statuses drive the x1.5 retries
    met, got, gst, ref, rst, stats = run_case(rpd, uniform(8000, seed=4), K=12, P=12, V=14)
    assert stats["npasses"] > 2
    assert_parity(met)


def test_clustered_seeds(rpd):
    met, *_ = run_case(rpd, clustered(15000), K=30, P=40, V=60)
    assert_parity(met)


def test_wall_seeds(rpd):
    x = uniform(6000, seed=8)
    x[::97, 3] = rpd.NO_CELL_LIMITS
    met, got, gst, ref, rst, _ = run_case(rpd, x, K=20, P=25, V=30)
    assert_parity(met)
    walls = x[:, 3] <= rpd.NO_CELL_LIMITS
    assert np.array_equal(got[walls], x[walls].astype(np.float64))


def test_early_out_and_parking_do_not_change_results(rpd):
    g = rpd.Grid.blob(60, 5, 2)
    x = jittered(40, seed=6, weights=True)
    s = rpd.Solver().set_points(x).set_grid(g)
    res = {}
    ref = rpd.FLAG_REFERENCE_APEX
    for name, flags in [("default", 0), ("no_early", rpd.FLAG_NO_EARLY_OUT), ("no_defer", rpd.FLAG_NO_DEFER),
                        ("inline", rpd.FLAG_NO_EARLY_OUT | rpd.FLAG_NO_DEFER),
                        ("ref_apex", ref), ("ref_apex_no_defer", ref | rpd.FLAG_NO_DEFER),
                        ("plain", rpd.FLAG_NO_EARLY_OUT | rpd.FLAG_NO_DEFER | ref)]:
        s.launch(K=50, P=30, V=40, T=60, flags=flags)
        res[name] = (s.moments(), s.status())
    s.launch(K=50, P=30, V=40, T=60, flags=ref | rpd.FLAG_COUNTERS)
    assert s.stats()["counters"]["cones_skipped"] == 0
    s.launch(K=50, P=30, V=40, T=60, flags=rpd.FLAG_COUNTERS)
    ctr = s.stats()["counters"]
    print("counters", ctr)
    assert 0 < ctr["cones_skipped"] < ctr["triangles"]
    m0, s0 = res["plain"]
    # parking sums a cell's cone pieces per chunk, and another apex gives
    # other pieces, so small restricted pieces that cancel against whole-cell
    # volumes differ in rounding: the scale of every cell is the typical cell
    # volume (moments x1000)
    typ = np.median(np.abs(m0[:, 3][np.abs(m0[:, 3]) > 0]))
    scale = np.maximum(np.abs(m0[:, 3]), typ)[:, None] * np.array([1000.0, 1000.0, 1000.0, 1.0])
    for name, (m, st) in res.items():
        assert np.array_equal(st, s0), name
        err = np.abs(m - m0) / scale
        print(name, "max rel", err.max())
        assert err.max() < 1e-12, name
    assert np.array_equal(res["no_defer"][0], res["inline"][0]), "the early exit must not change any bit"
    assert np.array_equal(res["ref_apex_no_defer"][0], m0), "the early exit must not change any bit"


def test_outside_probe_does_not_change_results(rpd):
    """The outside probe (RPD_FLAG_OUTSIDE_PROBE: cells proven empty outside
    the domain from the seeds of their 3x3x3 bins) changes no bit of the
    moments, nor here of the statuses (every cell it settles is one the
    reference's clipping settles too)."""
    g = rpd.Grid.blob(60, 5, 2)
    x = jittered(40, seed=6, weights=True)
    s = rpd.Solver().set_points(x).set_grid(g)
    probe = rpd.FLAG_OUTSIDE_PROBE
    fresh = rpd.FLAG_FRESH_NEIGHBOURS
    s.launch(K=50, P=30, V=40, T=60, flags=fresh | probe)
    st = s.stats()
    m1, s1 = s.moments(), s.status()
    print("probe", st["probe_outside"], "of", len(x), st["probe_ms"], "ms", st["passes"][0])
    assert st["probe_outside"] > len(x) // 4
    assert st["passes"][0]["cells"] == len(x)
    s.launch(K=50, P=30, V=40, T=60, flags=fresh)
    assert s.stats()["probe_outside"] == 0
    assert np.array_equal(s.status(), s1)
    assert np.array_equal(s.moments(), m1)
    # a weight-only re-solve after a probed first launch builds the whole
    # neighbour table (no probe), which the next one keeps
    t = rpd.Solver().set_points(x).set_grid(g)
    t.launch(K=50, P=30, V=40, T=60, flags=probe)
    assert t.stats()["probe_outside"] > 0
    x2 = x.copy()
    for it in range(2):
        x2[:, 3] = x[:, 3] * (0.5 + 0.25 * it)
        t.set_weights(x2[:, 3])
        t.launch(K=50, P=30, V=40, T=60, flags=probe)
        st = t.stats()
        assert st["probe_outside"] == 0
        f = rpd.Solver().set_points(x2).set_grid(g)
        f.launch(K=50, P=30, V=40, T=60)
        assert np.array_equal(t.status(), f.status())
        assert np.array_equal(t.moments(), f.moments())
    met, *_ = run_case(rpd, x2, grid=g, K=50, P=30, V=40, T=60)
    assert_parity(met)


@pytest.mark.parametrize("T", [20, 40])
def test_triangle_overflows_settled_ahead(rpd, T):
    """Small T: the first pass parks the cells that only overflow T and
    restricts them at once, as the retry passes would; the results are those
    of the retry passes (bit for bit) and of the oracle, with far fewer cells
    retried."""
    g = rpd.Grid.blob(40, 5, 2)
    x = jittered(30, seed=5, weights=True)
    s = rpd.Solver().set_points(x).set_grid(g)
    s.launch(K=50, P=30, V=40, T=T, flags=rpd.FLAG_FRESH_NEIGHBOURS)
    m1, s1, st1 = s.moments(), s.status(), s.stats()
    s.launch(K=50, P=30, V=40, T=T, flags=rpd.FLAG_FRESH_NEIGHBOURS | rpd.FLAG_NO_T_AHEAD)
    m0, s0, st0 = s.moments(), s.status(), s.stats()
    print("passes ahead", [p["cells"] for p in st1["passes"]], "retries", [p["cells"] for p in st0["passes"]])
    retried = lambda st: sum(p["cells"] for p in st["passes"][1:])  # noqa: E731
    assert st0["npasses"] >= 3 and retried(st1) < retried(st0) / 2
    assert np.array_equal(s1, s0)
    assert np.array_equal(m1, m0)
    met, *_ = run_case(rpd, x, grid=g, K=50, P=30, V=40, T=T)
    assert_parity(met)


def test_empty_cells_outside_the_domain(rpd):
    """Seeds far outside the domain whose weight empties their power cell
    keep the status empty_cell: the early exits outside the domain (the cell
    kernel's and the outside probe's) only take cells that cannot be empty."""
    g = rpd.Grid.blob(40, 5, 2)
    x = jittered(24, seed=11, weights=True)
    h2 = (1000.0 / 24) ** 2
    corner = (x[:, :3] < 150).all(axis=1) | (x[:, :3] > 850).all(axis=1)
    idx = np.where(corner)[0][::3]
    x[idx, 3] = 4 * h2
    for flags in (rpd.FLAG_OUTSIDE_PROBE, 0):
        met, got, gst, ref, rst, stats = run_case(rpd, x, grid=g, K=50, P=30, V=40,
                                                  flags=flags | rpd.FLAG_FRESH_NEIGHBOURS)
        assert (rst[idx] == 6).sum() > len(idx) // 2
        assert_parity(met)


def test_blue_noise_cube_domain(rpd):
    # the 5M blue-noise workload in small: Poisson-disk seeds, unit cube domain
    from rpd import synth

    x = synth.poisson_disk(30_000, seed=3)
    g = rpd.Grid.cube(48)
    met, got, gst, ref, rst, _ = run_case(rpd, x, grid=g, K=20, P=25, V=30, T=100)
    assert_parity(met)
    assert abs(got[:, 3].sum() / g.getVolume() - 1) < 1e-9


@pytest.mark.parametrize("workload", ["weighted-1m", "voronoi-100k"])
def test_bench_workloads_full_size(rpd, workload):
    # the benchmark's own inputs at full size against the FP64 oracle
    import os
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    cfg = bench.CONFIGS[workload]
    x = bench.make_seeds(cfg, 0)
    g = bench.make_grid(cfg)
    met, got, gst, *_ = run_case(rpd, x, grid=g, K=cfg["K"], P=cfg["P"], V=cfg["V"], T=cfg["T"])
    assert_parity(met)


def test_cell_in_the_box_margin_has_no_start_corner(rpd):
    """A weighted cell entirely in the box's margin past the grid (x >
    1000.05): the reference's find_another_beginning_vertex, as the oracle
    gives it; every other cell as the oracle."""
    import test_oracle

    g, _, x = test_oracle._margin_cell_case()
    met, got, gst, ref, rst, _ = run_case(rpd, x.astype(np.float32), grid=g, K=30, P=30, V=40, T=100)
    assert gst[-1] == 7 and rst[-1] == 7
    assert_parity(met)


def test_safe_radius_guard(rpd):
    """RPD_FLAG_SAFE_RADIUS: with weights the reference's Voronoi stop test
    (d^2 > 4 R^2) can end a cell before a lighter far neighbour cuts it, so
    the cells overlap and their masses over-count the domain; with the
    weighted guard they partition it to FP64 rounding.  Without weights the
    guard is the reference's test."""
    g = rpd.Grid.blob(40, 5, 2)
    vol = g.getVolume()
    x = jittered(24, seed=12, weights=True)
    h = 1000.0 / 24
    x[:, 3] = np.random.default_rng(3).uniform(0, 0.6 * h * h, len(x)).astype(np.float32)
    kw = dict(K=50, P=40, V=60, T=100)
    m0, s0, _ = solve_gpu(rpd, x, g, **kw)
    m1, s1, _ = solve_gpu(rpd, x, g, flags=rpd.FLAG_SAFE_RADIUS, **kw)
    assert (s0 == 4).all() and (s1 == 4).all()
    err0 = abs(m0[:, 3].sum() / vol - 1)
    err1 = abs(m1[:, 3].sum() / vol - 1)
    differ = int((m0 != m1).any(1).sum())
    print("reference test", err0, "guard", err1, "cells that differ", differ)
    assert err1 < 1e-12 and err0 > 100 * err1 and differ > 0
    # the reference's test equals the oracle (the reference algorithm)
    ref, rst = oracle.solve(x.astype(np.float64), grid=oracle_grid(g), use_double=True, knn_mode=1, **kw)
    assert_parity(compare(m0, s0, ref, rst))
    # equal weights: the same cells
    y = x.copy()
    y[:, 3] = 0
    ma, sa, _ = solve_gpu(rpd, y, g, **kw)
    mb, sb, _ = solve_gpu(rpd, y, g, flags=rpd.FLAG_SAFE_RADIUS, **kw)
    assert np.array_equal(sa, sb)
    assert np.abs(ma - mb).max() <= 1e-9 * np.abs(ma).max()
