"""The multi-GPU path of bench.py on world-size-2 gloo ranks (CPU): every
rank solves its own diagram (independent seed streams), the job's step time
is the slowest rank's, and the throughput counts all ranks' cells.  The
rank-local solve is the oracle here (no GPU on this path)."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, q):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "gpu-restricted-power-diagrams_b200"))
    import bench
    import oracle

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        cfg = dict(bench.CONFIGS["weighted-1m"], m=10)
        x = bench.make_seeds(cfg, rank)
        m, st = oracle.solve(x.astype(np.float64), K=cfg["K"], P=cfg["P"], V=cfg["V"], T=cfg["T"], use_double=True)
        ms = 10.0 + 5.0 * rank  # a slower second rank
        e2e = 0.02 + 0.01 * rank
        got = bench.aggregate_over_ranks(ms, e2e, len(x), world, "cpu")
        gathered = [None] * world
        dist.all_gather_object(gathered, (x[:5].tolist(), float(m[:, 3].sum())))
        dist.barrier()
        q.put((rank, got, gathered, int((st != 4).sum())))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_like_bench():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=240) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    for rank, (ms, e2e, value, e2e_value), gathered, failed in res:
        assert ms == pytest.approx(15.0) and e2e == pytest.approx(0.03)  # max over ranks
        assert value == pytest.approx(2 * 1000 / 0.015) and e2e_value == pytest.approx(2 * 1000 / 0.03)
        assert failed == 0
        # independent seed streams, and each rank's diagram fills the box
        assert gathered[0][0] != gathered[1][0]
        # weighted cells: the reference security radius over-counts by ~1e-9 relative
        assert gathered[0][1] == pytest.approx(1e9, rel=1e-7) and gathered[1][1] == pytest.approx(1e9, rel=1e-7)
