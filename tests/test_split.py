"""One diagram split over world-size-2 gloo ranks (CPU): rpd.split's
protocol -- every part's counts all-reduced after each pass, the parts'
stored-order results all-gathered and installed -- on a stand-in solver
whose part launch is the oracle (no GPU here).  Each rank must end with the
whole diagram's results, in the stored order of the reference's binning,
and the reduction must hand every part the whole diagram's counts."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class OracleParts:
    """The parts of a solver's C ABI that rpd.split uses, over the oracle:
    launch_part runs the whole diagram, keeps its part's stored range and
    reduces the range's failing counts; stored / set_stored / moments as
    rpd.Solver's."""

    def __init__(self, x, K, P, V):
        import oracle

        self.x = x
        self.kw = dict(K=K, P=P, V=V, use_double=True, knn_mode=1, first_pass_only=True)
        _, self.perm, _ = oracle.bin_seeds(x)  # stored index -> user index
        self.n = len(x)
        self.reduced = None

    def launch_part(self, part, parts, reduce, params=None, **kw):
        import oracle
        import rpd

        b, s = oracle.solve(self.x, **self.kw)
        first, count = rpd.part_range(self.n, part, parts)
        rows = self.perm[first:first + count]
        self.out = np.zeros((self.n, 4))
        self.st = np.full(self.n, -1, np.int32)
        self.out[first:first + count] = b[rows]
        self.st[first:first + count] = s[rows]
        fail = s[rows][s[rows] != 4]
        sums = np.bincount(fail, minlength=12)[:12].astype(np.int64)
        sums[11] = len(fail)
        self.reduced = reduce(sums, np.array([first], np.int64))
        return self

    def stored(self, first, count, out=None, status=None, device=False):
        return self.out[first:first + count].copy(), self.st[first:first + count].copy()

    def set_stored(self, out, status, device=False):
        self.out, self.st = np.asarray(out).copy(), np.asarray(status).copy()

    def moments(self):
        m = np.zeros((self.n, 4))
        m[self.perm] = self.out
        return m


def _rank_main(rank, world, port, q):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "gpu-restricted-power-diagrams_b200"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from seeds_util import jittered

    from rpd import split

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        x = jittered(14, seed=8, weights=True).astype(np.float64)
        s = OracleParts(x, K=12, P=14, V=18)  # tight caps: failing cells in both parts
        split.solve_split(s)
        dist.barrier()
        q.put((rank, s.moments(), s.st.copy(), s.reduced))
    finally:
        dist.destroy_process_group()


def test_split_over_two_gloo_ranks():
    import oracle

    from seeds_util import jittered

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=240) for _ in procs], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    x = jittered(14, seed=8, weights=True).astype(np.float64)
    b, s = oracle.solve(x, K=12, P=14, V=18, use_double=True, knn_mode=1, first_pass_only=True)
    _, perm, _ = oracle.bin_seeds(x)
    fail = s[s != 4]
    assert len(fail) > 0
    for rank, m, st, (sums, maxes) in res:
        assert np.array_equal(m, b)  # the whole diagram, user order
        assert np.array_equal(st, s[perm])  # stored order
        # the reduction gave every part the whole diagram's counts
        assert sums[11] == len(fail)
        assert np.array_equal(sums[:11], np.bincount(fail, minlength=11)[:11])
        assert maxes[0] == (len(x) + 1) // 2  # the larger part's first index
