"""Batched solves (rpd_batch_*): many diagrams in shared launches and one
CUDA graph give every solver exactly the results of its own launch."""
import numpy as np
import pytest

import oracle
from parity import assert_parity, compare

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rpd():
    import rpd as m

    m.default_context()
    return m


def specs(count, seed, nmin=800, nmax=20_000, gmin=24, gmax=56, ks=(20, 50, 70)):
    from rpd import synth

    return synth.uneven_batch(count, seed=seed, nmin=nmin, nmax=nmax, gmin=gmin, gmax=gmax, ks=ks)


def build(rpd, sp, with_grid):
    grids, solvers = [], []
    for i, s in enumerate(sp):
        g = rpd.Grid.blob(s["grid_size"], 5, s["grid_seed"]) if with_grid(i) else None
        v = rpd.Solver().set_points(s["xyzw"])
        if g is not None:
            v.set_grid(g)
        grids.append(g)
        solvers.append(v)
    return grids, solvers


def alone(rpd, x, g, p):
    """The diagram solved on its own: a first launch after its seeds were
    set, so with the outside probe where its flags ask for it, as in every
    batch replay (the probe settles in the first pass cells outside the
    domain that a full clip may retry, so per-pass cell counts depend on
    it).  Both settle triangle overflows ahead."""
    s = rpd.Solver().set_points(x)
    if g is not None:
        s.set_grid(g)
    s.launch(p)
    return s


def assert_same(got, ref):
    assert np.array_equal(got.status(), ref.status())
    assert np.array_equal(got.moments(), ref.moments())
    a, b = got.stats(), ref.stats()
    assert a["npasses"] == b["npasses"]
    assert a["status"] == b["status"]
    assert a["probe_outside"] == b["probe_outside"]
    for pa, pb in zip(a["passes"], b["passes"]):
        assert (pa["cells"], pa["K"], pa["P"], pa["V"], pa["T"]) == (pb["cells"], pb["K"], pb["P"], pb["V"], pb["T"])


def test_batch_equals_solves_alone(rpd):
    """Uneven diagrams, with and without domains, small caps so that every
    retry kind runs (K, P, V and T growth), a first-pass-only diagram and a
    reference-apex one."""
    sp = specs(12, seed=5)
    grids, solvers = build(rpd, sp, with_grid=lambda i: i % 4 != 3)
    params = []
    for i, s in enumerate(sp):
        p = rpd.Params.default(K=s["K"], P=12 + (i % 3) * 4, V=16 + (i % 2) * 8, T=20 + 10 * (i % 3))
        if i == 5:
            p.flags |= rpd.FLAG_FIRST_PASS_ONLY
        if i == 7:
            p.flags |= rpd.FLAG_REFERENCE_APEX
        if i in (1, 2, 4, 8):
            p.flags |= rpd.FLAG_OUTSIDE_PROBE
        if i == 9:
            p.flags |= rpd.FLAG_OUTSIDE_PROBE | rpd.FLAG_NO_PROBE
        if i == 10:
            p.flags |= rpd.FLAG_SAFE_RADIUS
        params.append(p)
    b = rpd.Batch(solvers, params)
    b.launch()
    st = b.stats()
    assert st["diagrams"] == 12 and st["cells"] == sum(len(s["xyzw"]) for s in sp)
    assert st["max_passes"] >= 3 and st["captures"] == 1
    print("solved alone", st["solved_alone"], [v.stats()["passes"][-1] for v in solvers])
    assert st["probe_outside"] > 0  # the domains leave plainly-outside seeds to prove
    assert solvers[9].stats()["probe_outside"] == 0 and solvers[0].stats()["probe_outside"] == 0
    for i, s in enumerate(sp):
        assert_same(solvers[i], alone(rpd, s["xyzw"], grids[i], params[i]))


def test_batch_replays_and_follows_weights_and_points(rpd):
    sp = specs(6, seed=8)
    grids, solvers = build(rpd, sp, with_grid=lambda i: True)
    params = [rpd.Params.default(K=s["K"], P=30, V=40) for s in sp]
    b = rpd.Batch(solvers, params)
    b.launch()
    first = [(v.status().copy(), v.moments().copy()) for v in solvers]
    b.launch()
    for v, (st0, m0) in zip(solvers, first):
        assert np.array_equal(v.status(), st0) and np.array_equal(v.moments(), m0)
    # weight-only change: the same graph, new results
    rng = np.random.default_rng(1)
    for i in (0, 3):
        x = sp[i]["xyzw"]
        x[:, 3] = rng.uniform(0, x[:, 3].max() * 2, len(x)).astype(np.float32)
        solvers[i].set_weights(x[:, 3])
    b.launch()
    assert b.stats()["captures"] == 1
    for i in range(len(sp)):
        assert_same(solvers[i], alone(rpd, sp[i]["xyzw"], grids[i], params[i]))
    # new seeds for one diagram: captured again
    y = sp[2]["xyzw"][: len(sp[2]["xyzw"]) // 2].copy()
    solvers[2].set_points(y)
    b.launch()
    assert b.stats()["captures"] == 2
    assert_same(solvers[2], alone(rpd, y, grids[2], params[2]))
    assert_same(solvers[1], alone(rpd, sp[1]["xyzw"], grids[1], params[1]))


def test_batch_parity_with_oracle(rpd):
    """Batched diagrams against the FP64 oracle."""
    sp = specs(3, seed=11, nmin=2000, nmax=6000)
    grids, solvers = build(rpd, sp, with_grid=lambda i: True)
    params = [rpd.Params.default(K=s["K"], P=30, V=40, T=100) for s in sp]
    rpd.Batch(solvers, params).launch()
    for i, s in enumerate(sp):
        a = grids[i].arrays()
        ga = oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])
        ref, rst = oracle.solve(s["xyzw"].astype(np.float64), grid=ga, use_double=True, knn_mode=1, K=s["K"], P=30,
                                V=40, T=100)
        assert_parity(compare(solvers[i].moments(), solvers[i].status(), ref, rst))


def test_batch_rejects_unsupported(rpd):
    sp = specs(2, seed=2, nmax=3000)
    grids, solvers = build(rpd, sp, with_grid=lambda i: True)
    with pytest.raises(rpd.RpdError):
        rpd.Batch(solvers, rpd.Params.default(flags=rpd.FLAG_COUNTERS))
    with pytest.raises(rpd.RpdError):
        rpd.Batch(solvers, rpd.Params.default(keep_distance=1)).launch()
    with pytest.raises(rpd.RpdError):
        rpd.Batch(solvers, rpd.Params.default(precision=rpd.PRECISION_MIXED))


def test_batch_parity_with_oracle_larger(rpd):
    """A larger uneven batch (12 diagrams up to 40K seeds, K 20/50/70, own
    blobs at 24^3..56^3, one without a domain) against the FP64 oracle,
    every cell of every diagram."""
    sp = specs(12, seed=21, nmin=5000, nmax=40_000)
    grids, solvers = build(rpd, sp, with_grid=lambda i: i != 4)
    params = [rpd.Params.default(K=s["K"], P=30, V=40, T=100) for s in sp]
    b = rpd.Batch(solvers, params)
    b.launch()
    for i, s in enumerate(sp):
        ga = None
        if grids[i] is not None:
            a = grids[i].arrays()
            ga = oracle.GridArrays(a["size"], a["in_domain"], a["points"], a["triangles"], a["tri_list"], a["offsets"])
        ref, rst = oracle.solve(s["xyzw"].astype(np.float64), grid=ga, use_double=True, knn_mode=1, K=s["K"], P=30,
                                V=40, T=100)
        assert_parity(compare(solvers[i].moments(), solvers[i].status(), ref, rst))


def test_batch_hessian_rows(rpd):
    """Batched diagrams with --hessian rows (rpd_solver_get_hessian on each
    solver): rows, moments and statuses equal those of each diagram solved
    alone, bit for bit; the batch then sums boundary cells in their own warps
    (no parked cells, no triangle overflows settled ahead), so its per-pass
    counts are those of a lone solve with RPD_FLAG_NO_DEFER.  Diagrams with
    rows must share hessian_hc."""
    sp = specs(6, seed=13, nmin=2000, nmax=12_000)
    grids, solvers = build(rpd, sp, with_grid=lambda i: i != 2)
    params = []
    for i, s in enumerate(sp):
        kw = dict(K=s["K"], P=30, V=40, T=60)
        if i % 2 == 0:
            kw.update(hessian_h=40, hessian_hc=1)
        params.append(rpd.Params.default(**kw))
    b = rpd.Batch(solvers, params)
    b.launch()
    for i, s in enumerate(sp):
        p = params[i]
        if p.hessian_h == 0:
            p = rpd.Params.default(K=s["K"], P=30, V=40, T=60, flags=rpd.FLAG_NO_DEFER)
        ref = alone(rpd, s["xyzw"], grids[i], p)
        assert_same(solvers[i], ref)
        if params[i].hessian_h:
            v, ids = solvers[i].hessian(40, 1)
            rv, rids = ref.hessian(40, 1)
            assert np.array_equal(v, rv) and np.array_equal(ids, rids)
            assert (ids[:, 0] >= 0).any()
        ref.close()
    mixed = [rpd.Params.default(K=s["K"], hessian_h=20, hessian_hc=1 + 3 * (i % 2)) for i, s in enumerate(sp)]
    with pytest.raises(rpd.RpdError):
        rpd.Batch(solvers, mixed).launch()
