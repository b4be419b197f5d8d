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


def _view_digest(scene, v) -> str:
    """Digest of one view's cull outputs (the oracle stands in for the device on CPU)."""
    import hashlib

    import numpy as np

    from helio_b200 import native as N
    from oracle import oracle as O

    levels = O.hiz_build(v.depth)
    r = O.run_view(scene, v.camera, v.width, v.height, levels, v.lod_threshold_px, None, 11, 2,
                   np.dtype(N.InstanceCullData))
    h = hashlib.sha256()
    for k in ("selected", "counters", "indirect", "draws", "visibility"):
        h.update(np.ascontiguousarray(r[k]).tobytes())
    return h.hexdigest()


def _shard_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    r, w = D.init("gloo", timeout_s=60)
    from helio_b200 import scene as S

    wl = S.config(3, scale=0.02)
    mine = D.shard_views(wl.views, wl.scene.lod0_total, w, r)
    outs = {i: _view_digest(wl.scene, wl.views[i]) for i in mine}
    parts = D.gather_objects(outs)
    # the serving stream's owners: the same on every rank
    reqs = S.serving_requests(64, 2000.0)
    owners = D.assign_online([float(len(x.views)) for x in reqs], w)
    q.put({"rank": r, "parts": parts, "owners": owners})
    import torch.distributed as dist

    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_union_of_view_shards_equals_one_rank():
    """batched3 split across 2 ranks by cost: the union of what the ranks cull is every
    view exactly once, with the outputs one rank gets for all views."""
    from helio_b200 import scene as S

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_shard_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in procs], key=lambda x: x["rank"])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    parts = res[0]["parts"]
    assert res[1]["parts"] == parts and res[0]["owners"] == res[1]["owners"]
    assert not set(parts[0]) & set(parts[1])
    union = {**parts[0], **parts[1]}
    wl = S.config(3, scale=0.02)
    assert sorted(union) == list(range(len(wl.views)))
    one_rank = {i: _view_digest(wl.scene, v) for i, v in enumerate(wl.views)}
    assert union == one_rank


def test_assign_online_balances_a_stream():
    costs = [float(1 + (i * 37) % 85) for i in range(400)]
    for world in (1, 2, 4, 8):
        owner = D.assign_online(costs, world)
        loads = [sum(c for c, o in zip(costs, owner) if o == r) for r in range(world)]
        assert max(loads) - min(loads) <= max(costs)


def test_shard_by_cost_is_balanced_and_deterministic():
    costs = [8.0 * 3840 * 2160] + [8.0 * 2048 * 2048] * 4 + [8.0 * 512 * 512] * 16 + [8.0 * 128 * 128] * 64
    for world in (1, 2, 4, 8):
        s1 = D.shard_by_cost(costs, world)
        assert s1 == D.shard_by_cost(costs, world)
        assert sorted(i for part in s1 for i in part) == list(range(len(costs)))
        loads = [sum(costs[i] for i in part) for part in s1]
        assert max(loads) <= max(costs) + sum(costs) / world  # LPT bound
