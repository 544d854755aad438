"""One diagram over the ranks of a torch.distributed group (one GPU each).

Every rank holds all seeds and the domain and solves the cells of its part
of the stored (binned) seeds (rpd_solver_launch_part); after each pass the
failing cells' status histogram and count are summed and the largest
triangle count settled ahead is maximised over the ranks (all_reduce), so
every part follows the whole diagram's retry schedule; then the parts'
stored-order results are all-gathered and installed on every rank's solver
(rpd_solver_set_stored).  With NCCL the gather runs on the device; with gloo
through host memory.  The results are rpd_solver_launch's on one GPU, bit
for bit.  No counterpart in the reference, which solves one batch of ids
after another on one device (voronoi.cpp:960-973)."""
from __future__ import annotations

import numpy as np


def solve_split(solver, group=None, params=None, **kw):
    """Solves `solver`'s diagram with the group's ranks, one part each;
    afterwards every rank's solver holds the whole diagram's results."""
    import torch
    import torch.distributed as dist

    import rpd

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    on_device = dist.get_backend(group) == "nccl"
    dev = torch.device("cuda", torch.cuda.current_device()) if on_device else torch.device("cpu")

    def reduce(sums, maxes):
        s = torch.from_numpy(np.asarray(sums, np.int64)).to(dev)
        m = torch.from_numpy(np.asarray(maxes, np.int64)).to(dev)
        dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
        dist.all_reduce(m, op=dist.ReduceOp.MAX, group=group)
        return s.cpu().numpy(), m.cpu().numpy()

    solver.launch_part(rank, world, reduce, params=params, **kw)
    n = solver.n
    first, count = rpd.part_range(n, rank, world)
    per = (n + world - 1) // world  # every part's rows, padded to the largest
    out = torch.zeros((per, 4), dtype=torch.float64, device=dev)
    st = torch.full((per,), -1, dtype=torch.int32, device=dev)
    if on_device:
        if count:
            solver.stored(first, count, out.data_ptr(), st.data_ptr(), device=True)
    else:
        o, s = solver.stored(first, count)
        out[:count] = torch.from_numpy(o)
        st[:count] = torch.from_numpy(s)
    outs = [torch.empty_like(out) for _ in range(world)]
    sts = [torch.empty_like(st) for _ in range(world)]
    dist.all_gather(outs, out, group=group)
    dist.all_gather(sts, st, group=group)
    # the parts' ranges are contiguous and in order: their rows, unpadded,
    # are the stored order
    counts = [rpd.part_range(n, r, world)[1] for r in range(world)]
    outs = torch.cat([o[:c] for o, c in zip(outs, counts)]).contiguous()
    sts = torch.cat([t[:c] for t, c in zip(sts, counts)]).contiguous()
    if on_device:
        # the gather ran on torch's stream, the copy runs on the engine's
        torch.cuda.current_stream().synchronize()
        solver.set_stored(outs.data_ptr(), sts.data_ptr(), device=True)
    else:
        solver.set_stored(outs.numpy(), sts.numpy())
    return solver
