"""Several GPUs, one process each, for the batched form.

Independent clouds need no exchange: the clouds of a batch are dealt to the ranks
(each rank builds and evaluates one forest of its own clouds on its own GPU) and a
measurement is the slowest rank's.  Charge vectors of one cloud stay together (they
share the cloud's plan).  A single cloud split over ranks needs the reference's
ghost and multipole exchanges (fmm-exec/src/fmm.rs, "Several ranks"); that is not
built here.
"""


def shard_clouds(sizes, world):
    """Deals clouds (by point count) to `world` ranks, largest first onto the least
    loaded rank (ties to the lower rank): every rank computes the same answer.
    Returns the cloud indices of each rank in increasing order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    loads = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda j: (loads[j], j))
        parts[r].append(i)
        loads[r] += int(sizes[i])
    return [sorted(p) for p in parts]


def max_over_ranks(value, device=None):
    """The largest of every rank's `value` (a float), through torch.distributed; the
    value itself when no process group is initialised.  Every rank must call it, in the
    same order as its other collectives."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
