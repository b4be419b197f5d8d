"""Multi-rank host logic on CPU: world_size 2 with the gloo backend (spawned processes)."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from helio_b200 import dist as D


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    r, w = D.init("gloo", timeout_s=60)
    from helio_b200 import scene as S

    views = S.multiview_set(S.SEED_BASE + 3, depth=False, scale=0.05)
    costs = [D.view_cost(v.width, v.height, 1000) for v in views]
    mine = D.shard_by_cost(costs, w)[r]
    step_ms = 1.0 + r  # rank 1 is slower
    result = {
        "rank": r,
        "views": mine,
        "max_ms": D.max_over_ranks(step_ms),
        "total_views": D.sum_over_ranks(len(mine)),
    }
    q.put(result)
    import torch.distributed as dist

    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_views_and_reduce_timing():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=120) for _ in procs], key=lambda x: x["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    a, b = res[0]["views"], res[1]["views"]
    assert not set(a) & set(b) and len(a) + len(b) == 85  # a partition of the 85 views
    assert all(r["max_ms"] == 2.0 for r in res)  # max over ranks
    assert all(r["total_views"] == 85 for r in res)


def test_shard_by_cost_is_balanced_and_deterministic():
    costs = [8.0 * 3840 * 2160] + [8.0 * 2048 * 2048] * 4 + [8.0 * 512 * 512] * 16 + [8.0 * 128 * 128] * 64
    for world in (1, 2, 4, 8):
        s1 = D.shard_by_cost(costs, world)
        assert s1 == D.shard_by_cost(costs, world)
        assert sorted(i for part in s1 for i in part) == list(range(len(costs)))
        loads = [sum(costs[i] for i in part) for part in s1]
        assert max(loads) <= max(costs) + sum(costs) / world  # LPT bound
