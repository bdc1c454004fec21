"""One process per GPU: the host-side logic of multi-GPU runs.

The multi-block path shards by independent cases (a case never spans
GPUs), so ranks exchange no data while they step; they only agree on the
timing (the slowest rank's device time) and on totals.  Everything here
works on any torch.distributed backend (NCCL between GPUs, gloo on the host
for tests).
"""
import datetime
import os


def env():
    """(rank, world, local_rank) from the launcher's environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend, timeout_s=120):
    """Initialise the default process group from the environment with a short
    timeout (ranks that wait for a missing peer fail instead of hanging)."""
    import torch.distributed as dist

    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def shard(case_ids, rank, world):
    """The cases of one rank: every world-th case starting at rank (the shards
    are disjoint and cover every case)."""
    return list(case_ids)[rank::world]


def balance(costs, rank, world):
    """The cases of one rank when cases differ in cost (cell updates per
    coarse step): longest-processing-time-first assignment, every case to the
    rank with the least total so far (ties to the lowest rank).  Every rank
    computes the same assignment from the same costs; the shards are disjoint,
    cover every case, and no rank's total exceeds the mean by more than the
    largest single cost.  Returns the case indices of `rank`, ascending."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world
    owner = [0] * len(costs)
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += costs[i]
    return [i for i in range(len(costs)) if owner[i] == rank]


def reduce(values, op, dist=None, device="cpu"):
    """Element-wise MAX or SUM of a list of floats over all ranks (identity
    without a process group); every rank gets the result."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return [float(v) for v in t.cpu()]
