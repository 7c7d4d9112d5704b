"""Work split and timing reductions for one process per GPU.

The Godunov step of independent problems needs no exchange: at N > 1 whole
problems (batch ensembles, request streams) are dealt to the ranks and only the
timings meet, as a max over ranks (the job ends when the slowest rank ends) and
sums of the work done.  ``dist`` is ``torch.distributed`` (NCCL on the GPU
box, gloo in the CPU tests) or None for a single process.
"""


def shard(items, rank, world):
    """Items rank ``rank`` of ``world`` owns: every world-th one from rank (a
    deal keeps the size mix of a sorted or random list balanced)."""
    return list(items)[rank::world]


def _reduce(values, dist, op, device):
    if dist is None:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return t.tolist()


def max_over_ranks(values, dist, device="cuda"):
    """Element-wise max over ranks of a list of floats."""
    return _reduce(values, dist, None if dist is None else dist.ReduceOp.MAX, device)


def sum_over_ranks(values, dist, device="cuda"):
    """Element-wise sum over ranks of a list of floats."""
    return _reduce(values, dist, None if dist is None else dist.ReduceOp.SUM, device)
