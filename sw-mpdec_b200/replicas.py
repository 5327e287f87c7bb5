"""Replica bookkeeping for runs on several GPUs of one node.

The time step does not shard: every problem runs whole on one GPU, so N GPUs run
N independent replicas (or split an ensemble's problem list) with no data-path
collective.  The only exchange is the timing: the timed region's length is the
maximum over ranks, and throughput is the total of all ranks' cell-steps over it.
"""


def shard(sizes, rank, world):
    """Indices of the problems this rank steps: longest-processing-time-first
    assignment of the problem sizes (cells) to `world` ranks; deterministic."""
    order = sorted(range(len(sizes)), key=lambda i: (-sizes[i], i))
    load = [0] * world
    owner = [0] * len(sizes)
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += sizes[i]
    return [i for i in range(len(sizes)) if owner[i] == rank]


def aggregate(local_ms, local_cell_steps, dist=None, device=None):
    """(max over ranks of local_ms, sum over ranks of local_cell_steps)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(local_ms), float(local_cell_steps)
    import torch
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    c = torch.tensor([float(local_cell_steps)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return float(t.item()), float(c.item())
