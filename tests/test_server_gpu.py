"""The serving loop (rpd_server_*): requests admitted onto concurrent streams
give the same results as alone, a session's requests run in order, and the
memory budget serializes requests that do not fit together."""
import numpy as np
import pytest

from seeds_util import jittered, uniform

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rpd():
    import rpd as m

    m.default_context()
    return m


def workload(rpd):
    g1 = rpd.Grid.blob(48, 5, 2)
    g2 = rpd.Grid.blob(32, 5, 9)
    sets = [
        (jittered(30, seed=1, weights=True), g1, dict(K=50, P=30, V=40, T=100)),
        (uniform(20000, seed=2), g2, dict(K=70, P=30, V=40, T=100)),
        (jittered(20, seed=3, weights=True), None, dict(K=20, P=25, V=30)),
        (jittered(26, seed=4, weights=True), g1, dict(K=50, P=30, V=40, T=100)),
    ]
    rng = np.random.default_rng(5)
    reweights = []
    for i, (x, g, kw) in enumerate(sets):
        h = 1000.0 / round(len(x) ** (1 / 3))
        for _ in range(2):
            w = np.clip(x[:, 3] + rng.normal(0, 0.05 * h * h, len(x)), 0, None).astype(np.float32)
            reweights.append((i, w))
    return (g1, g2), sets, reweights


def run(rpd, slots, budget, sets, reweights, submit_all):
    out = {}
    with rpd.Server(slots=slots, mem_budget=budget) as sv:
        tickets = []
        sessions = []
        for i, (x, g, kw) in enumerate(sets):
            t, sess = sv.solve(x, grid=g, **kw)
            sessions.append(sess)
            tickets.append((("solve", i), t))
            if not submit_all:
                out[("solve", i)] = sv.wait(t)
                tickets.pop()
        for j, (i, w) in enumerate(reweights):
            t = sv.reweight(sessions[i], w, **sets[i][2])
            tickets.append((("reweight", j), t))
            if not submit_all:
                out[("reweight", j)] = sv.wait(t)
                tickets.pop()
        for key, t in tickets:
            out[key] = sv.wait(t)
        for s in sessions:
            sv.release(s)
    return out


def test_results_same_alone_and_in_the_mix(rpd):
    grids, sets, reweights = workload(rpd)
    alone = run(rpd, 1, 0, sets, reweights, submit_all=False)
    mix = run(rpd, 4, 0, sets, reweights, submit_all=True)
    assert set(alone) == set(mix)
    slots = set()
    for key in alone:
        a, ia = alone[key]
        m, im = mix[key]
        assert ia["status"] == 0 and im["status"] == 0
        assert np.array_equal(a, m), key
        slots.add(im["slot"])
    assert len(slots) > 1  # the mix ran on several streams
    # and a plain solver agrees with the served results
    for i, (x, g, kw) in enumerate(sets):
        s = rpd.Solver().set_points(x)
        if g is not None:
            s.set_grid(g)
        s.launch(**kw)
        assert np.array_equal(s.moments(), alone[("solve", i)][0])
    # re-solves: the last weights of each session, solved from scratch
    last = {}
    for j, (i, w) in enumerate(reweights):
        last[i] = (j, w)
    for i, (j, w) in last.items():
        x, g, kw = sets[i]
        x2 = x.copy()
        x2[:, 3] = w
        s = rpd.Solver().set_points(x2)
        if g is not None:
            s.set_grid(g)
        s.launch(**kw)
        assert np.array_equal(s.moments(), mix[("reweight", j)][0])


def test_tiny_budget_runs_one_request_at_a_time(rpd):
    grids, sets, reweights = workload(rpd)
    out = run(rpd, 4, 1, sets[:3], [], submit_all=True)
    spans = sorted((i["admitted_at_ms"], i["done_at_ms"]) for _, i in out.values())
    for (a0, d0), (a1, d1) in zip(spans, spans[1:]):
        assert a1 >= d0  # admitted only after the previous one finished


def test_failed_request_reports_error(rpd):
    with rpd.Server(slots=2) as sv:
        t, sess = sv.solve(jittered(10, seed=1), K=0)
        with pytest.raises(rpd.RpdError):
            sv.wait(t)
        with pytest.raises(rpd.RpdError):
            sv.reweight(sess, np.zeros(1000, np.float32))
        t2, s2 = sv.solve(jittered(10, seed=1), K=20)
        m, info = sv.wait(t2)
        assert info["status"] == 0 and abs(m[:, 3].sum() / 1e9 - 1) < 1e-6


def test_hessian_rows_served(rpd):
    """Requests with --hessian rows (rpd_server_submit_*_hessian): the rows a
    served solve and a served weight-only re-solve return equal those of the
    same launches on a solver of their own, bit for bit, while another
    session's plain requests share the slots; the plain submit rejects
    hessian_h > 0."""
    g = rpd.Grid.blob(40, 5, 2)
    x = jittered(24, seed=6, weights=True)
    y = jittered(20, seed=7, weights=True)
    w = np.clip(x[:, 3] * 1.5, 0, None).astype(np.float32)
    kw1 = dict(K=50, P=30, V=40, T=100, hessian_h=40, hessian_hc=1)
    kw4 = dict(K=50, P=30, V=40, T=100, hessian_h=40, hessian_hc=4)
    with rpd.Server(slots=2) as sv:
        t1, s1 = sv.solve(x, grid=g, **kw1)
        t2, s2 = sv.solve(y, grid=g, K=50, P=30, V=40, T=100)
        t3 = sv.reweight(s1, w, **kw4)
        m1, _, rows1 = sv.wait(t1, hessian=True)
        m2, _, rows2 = sv.wait(t2, hessian=True)
        m3, _, rows3 = sv.wait(t3, hessian=True)
        sv.release(s1)
        sv.release(s2)
        p = rpd.Params.default(K=50, hessian_h=8)
        out = np.zeros((len(x), 4), np.float64)
        sess = rpd.C.c_int(-1)
        assert rpd.lib().rpd_server_submit_solve(sv.h, rpd._ptr(x), len(x), None, rpd.C.byref(p), rpd._ptr(out),
                                                 rpd.C.byref(sess)) < 0
    assert rows2 is None
    ref = rpd.Solver().set_points(x).set_grid(g)
    ref.launch(**kw1)
    v1, i1 = ref.hessian(40, 1)
    assert np.array_equal(m1, ref.moments())
    assert np.array_equal(rows1[0], v1) and np.array_equal(rows1[1], i1)
    assert (i1[:, 0] >= 0).sum() > len(x) // 10  # cells inside the domain have rows
    x2 = x.copy()
    x2[:, 3] = w
    ref2 = rpd.Solver().set_points(x2).set_grid(g)
    ref2.launch(**kw4)
    v4, i4 = ref2.hessian(40, 4)
    assert np.array_equal(m3, ref2.moments())
    assert np.array_equal(rows3[0], v4) and np.array_equal(rows3[1], i4)


def test_domains_built_on_the_device(rpd):
    """Sessions whose domains are built on the device (rpd_server_submit_solve_blob
    / _field): a blob request equals a solver on the host-built blob (the same
    triangles voxel by voxel), a field request equals a solver with the same
    field, their weight-only re-solves keep the session's domain, and a
    session on a shared host grid runs beside them; Hessian rows come back
    through the blob form."""
    x = jittered(24, seed=11, weights=True)
    y = uniform(15000, seed=12)
    z = jittered(20, seed=13, weights=True)
    S = 40
    g = np.arange(S + 1) / S
    zz, yy, xx = np.meshgrid(g, g, g, indexing="ij")
    f = (np.sqrt((xx - 0.5) ** 2 + (yy - 0.45) ** 2 + (zz - 0.55) ** 2) - 0.32).astype(np.float32)
    host = rpd.Grid.blob(32, 5, 9)
    kw = dict(K=50, P=30, V=40, T=100)
    kwh = dict(kw, hessian_h=40, hessian_hc=1)
    w = np.clip(x[:, 3] * 1.3, 0, None).astype(np.float32)
    wy = np.full(len(y), 50.0, np.float32)
    with rpd.Server(slots=3) as sv:
        t1, s1 = sv.solve(x, blob=(48, 5, 2), **kwh)
        t2, s2 = sv.solve(y, field=f, **kw)
        t3, s3 = sv.solve(z, grid=host, **kw)
        t4 = sv.reweight(s1, w, **kw)
        t5 = sv.reweight(s2, wy, **kw)
        m1, i1, rows1 = sv.wait(t1, hessian=True)
        m2, i2 = sv.wait(t2)
        m3, i3 = sv.wait(t3)
        m4, i4 = sv.wait(t4)
        m5, i5 = sv.wait(t5)
        for s in (s1, s2, s3):
            sv.release(s)
        with pytest.raises(ValueError):
            sv.solve(x, grid=host, blob=(48, 5, 2))
        p = rpd.Params.default(**kw)
        out = np.zeros((len(x), 4), np.float64)
        sess = rpd.C.c_int(-1)
        assert rpd.lib().rpd_server_submit_solve_blob(sv.h, rpd._ptr(x), len(x), 2000, 5, 2, rpd.C.byref(p),
                                                      rpd._ptr(out), None, None, rpd.C.byref(sess)) < 0
        assert rpd.lib().rpd_server_submit_solve_field(sv.h, rpd._ptr(x), len(x), 16, None, rpd.C.byref(p),
                                                       rpd._ptr(out), None, None, rpd.C.byref(sess)) < 0
    assert all(i["status"] == 0 for i in (i1, i2, i3, i4, i5))
    ref = rpd.Solver().set_points(x).set_grid(rpd.Grid.blob(48, 5, 2))
    ref.launch(**kwh)
    assert np.array_equal(m1, ref.moments())
    v, ids = ref.hessian(40, 1)
    assert np.array_equal(rows1[0], v) and np.array_equal(rows1[1], ids)
    x2 = x.copy()
    x2[:, 3] = w
    ref = rpd.Solver().set_points(x2).set_grid(rpd.Grid.blob(48, 5, 2))
    ref.launch(**kw)
    assert np.array_equal(m4, ref.moments())
    ref = rpd.Solver().set_points(y).set_grid_field(f)
    ref.launch(**kw)
    assert np.array_equal(m2, ref.moments())
    assert (m2[:, 3] > 0).sum() > len(y) // 10  # cells inside the domain
    y2 = y.copy()
    y2[:, 3] = wy
    ref = rpd.Solver().set_points(y2).set_grid_field(f)
    ref.launch(**kw)
    assert np.array_equal(m5, ref.moments())
    ref = rpd.Solver().set_points(z).set_grid(host)
    ref.launch(**kw)
    assert np.array_equal(m3, ref.moments())
