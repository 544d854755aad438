"""One diagram split into parts (rpd_solver_launch_part) against the whole
solve (rpd_solver_launch), bit for bit.  The parts run as host threads on
one GPU, each with its own context (stream) and solver; they meet only in
the reduction callback, a host-side barrier after each pass (no kernel waits
for another), as ranks on several GPUs would meet in an all-reduce."""
import threading

import numpy as np
import pytest

from seeds_util import jittered, uniform

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rpd():
    import rpd as m

    m.default_context()
    return m


class HostAllReduce:
    """Sums / maxima over `parts` threads, one round per call."""

    def __init__(self, parts):
        self.barrier = threading.Barrier(parts)
        self.lock = threading.Lock()
        self.rounds = {}
        self.calls = threading.local()

    def __call__(self, sums, maxes):
        r = getattr(self.calls, "n", 0)
        self.calls.n = r + 1
        with self.lock:
            acc = self.rounds.setdefault(r, [np.zeros_like(sums), np.full_like(maxes, np.iinfo(np.int64).min), 0])
            acc[0] += sums
            acc[1] = np.maximum(acc[1], maxes)
            acc[2] += 1
        self.barrier.wait(timeout=120)
        return acc[0].copy(), acc[1].copy()


def split_solve(rpd, x, g, parts, **kw):
    red = HostAllReduce(parts)
    out = [None] * parts
    errs = []

    def run(part):
        try:
            ctx = rpd.Context(0)
            s = rpd.Solver(ctx).set_points(x)
            if g is not None:
                s.set_grid(g)
            s.launch_part(part, parts, red, **kw)
            first, count = rpd.part_range(len(x), part, parts)
            out[part] = (s.stored(first, count), s.stats())
            s.close()
        except Exception as exc:
            errs.append(exc)
            red.barrier.abort()

    th = [threading.Thread(target=run, args=(p,)) for p in range(parts)]
    for t in th:
        t.start()
    for t in th:
        t.join(timeout=300)
    assert not errs, errs
    m = np.concatenate([o[0][0] for o in out])
    st = np.concatenate([o[0][1] for o in out])
    return m, st, [o[1] for o in out], len(red.rounds)


@pytest.mark.parametrize("parts", [2, 3])
@pytest.mark.parametrize("case", ["weighted_blob", "uniform_cube_tight"])
def test_split_equals_whole(rpd, case, parts):
    if case == "weighted_blob":
        x, g, kw = jittered(30, seed=5, weights=True), rpd.Grid.blob(40, 5, 2), dict(K=50, P=30, V=40, T=40)
    else:
        x, g, kw = uniform(20000, seed=7), None, dict(K=14, P=14, V=18)
    whole = rpd.Solver().set_points(x)
    if g is not None:
        whole.set_grid(g)
    whole.launch(**kw)
    m_all, s_all, st_all = whole.moments(), whole.status(), whole.stats()
    m, st, stats, rounds = split_solve(rpd, x, g, parts, **kw)
    gathered = rpd.Solver().set_points(x)
    gathered.set_stored(m, st)
    assert np.array_equal(gathered.status(), s_all)
    assert np.array_equal(gathered.moments(), m_all)
    # every part ran the whole diagram's schedule: the same passes and caps
    assert rounds == st_all["npasses"]
    for p in stats:
        assert p["npasses"] == st_all["npasses"]
        assert [(q["K"], q["P"], q["V"], q["T"]) for q in p["passes"]] == \
               [(q["K"], q["P"], q["V"], q["T"]) for q in st_all["passes"]]
    # the parts' retry cells add up to the whole's
    for i in range(1, st_all["npasses"]):
        assert sum(p["passes"][i]["cells"] for p in stats) == st_all["passes"][i]["cells"]
