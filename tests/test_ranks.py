"""Multi-rank host logic (mblbm.ranks) on two gloo processes on the CPU: the
case shards are disjoint and complete, and MAX / SUM reductions give every
rank the same result (the slowest rank's time, the total updates)."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "multi-block-lbm-gpu_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from mblbm import ranks

    r, w, lr = ranks.env()
    dist = ranks.init("gloo", timeout_s=60)
    mine = ranks.shard(range(10), r, w)
    mx = ranks.reduce([1.0 + r, 10.0 - r], "max", dist)
    sm = ranks.reduce([len(mine)], "sum", dist)
    # the batched workload's shards: cases of uneven cost, balanced by cost
    costs = [(7 * i * i + 3) % 41 + 1 for i in range(37)]
    bal = ranks.balance(costs, r, w)
    load = ranks.reduce([sum(costs[i] for i in bal), len(bal)], "sum", dist)
    dist.barrier()
    dist.destroy_process_group()
    q.put((r, w, lr, mine, mx, sm, bal, load))


def test_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, w0, l0, s0, mx0, sm0, b0, ld0), (r1, w1, l1, s1, mx1, sm1, b1, ld1) = out
    assert (r0, r1, w0, w1, l0, l1) == (0, 1, 2, 2, 0, 1)
    assert sorted(s0 + s1) == list(range(10)) and not set(s0) & set(s1)
    assert mx0 == mx1 == [2.0, 10.0]
    assert sm0 == sm1 == [10.0]
    costs = [(7 * i * i + 3) % 41 + 1 for i in range(37)]
    assert sorted(b0 + b1) == list(range(37)) and not set(b0) & set(b1)
    assert ld0 == ld1 == [float(sum(costs)), 37.0]
    t0, t1 = sum(costs[i] for i in b0), sum(costs[i] for i in b1)
    assert abs(t0 - t1) <= max(costs)


def test_single_rank_is_identity():
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "multi-block-lbm-gpu_b200"))
    from mblbm import ranks
    assert ranks.reduce([3.0, 4.0], "max") == [3.0, 4.0]
    assert ranks.shard(range(5), 0, 1) == [0, 1, 2, 3, 4]
    assert ranks.balance([5, 1, 9], 0, 1) == [0, 1, 2]


def test_balance_bound():
    """Greedy longest-first: disjoint, complete, within one largest cost of the mean."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                    "multi-block-lbm-gpu_b200"))
    from mblbm import ranks
    costs = [((i * 2654435761) % 1000) + 100 for i in range(256)]
    for world in (2, 3, 4, 8):
        shards = [ranks.balance(costs, r, world) for r in range(world)]
        assert sorted(sum(shards, [])) == list(range(256))
        loads = [sum(costs[i] for i in s) for s in shards]
        assert max(loads) - sum(costs) / world <= max(costs)
