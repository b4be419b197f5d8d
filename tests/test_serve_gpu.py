"""The serving loop (helio_serve): every request's results are the same whether it is
served alone or batched with others and run beside other batches, and match the
oracle; the HBM budget gates admission without changing results."""
import numpy as np
import pytest

from helpers import cull_dtype, u32
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _world(n_scenes=3, n_requests=24, seed=5):
    import torch
    from helio_b200 import scene as S
    from helio_b200.passes import VgScene

    scenes, vgs = [], []
    for k in range(n_scenes):
        sc = S.make_scene(1000 + k, [300, 900, 2000][k % 3], 100, 4, 0, 100.0, lod_error_mode=1, mesh_library=64)
        vs = VgScene()
        vs.upload(S.frame_data(sc))
        scenes.append(sc)
        vgs.append(vs)
    pool = S.multiview_set(77, depth=True, scale=0.1)
    depths = [torch.from_numpy(np.ascontiguousarray(v.depth)).cuda() for v in pool]
    rng = np.random.default_rng(seed)
    requests = []
    for i in range(n_requests):
        sid = int(rng.integers(n_scenes))
        pick = rng.integers(len(pool), size=int(rng.integers(1, 13)))
        requests.append((sid, [int(p) for p in pick]))
    return scenes, vgs, pool, depths, requests


def _spec(pool, depths, idx):
    return [{"camera": pool[p].camera, "depth": depths[p], "alias_mip0": True,
             "lod_threshold_px": pool[p].lod_threshold_px} for p in idx]


def _collect(loop, rid, n_views, n_objects):
    out = []
    for v in range(n_views):
        o = loop.outputs(rid, v)
        c = u32(o["counters"])
        n = int(min(c[0], o["capacity"]))
        out.append({"counters": c, "indirect": u32(o["indirect"])[:n], "draws": u32(o["draws"])[:n],
                    "lod": o["lod"].cpu().numpy()[:n_objects].copy()})
    return out


def _serve(vgs, scenes, pool, depths, requests, **cfg):
    """Submits every request at time 0 and pumps until all complete; returns
    ({request index: per-view outputs}, completions)."""
    import time

    from helio_b200.passes import ServeLoop

    loop = ServeLoop(**cfg)
    ids = [loop.add_scene(vs) for vs in vgs]
    rid_of = {}
    for i, (sid, idx) in enumerate(requests):
        rid_of[loop.submit(ids[sid], _spec(pool, depths, idx), 0.0, tag=i)] = i
    results, comps, peak = {}, [], 0
    t0 = time.perf_counter()
    while len(comps) < len(requests):
        loop.pump(time.perf_counter() - t0)
        peak = max(peak, loop.stats()["bytes_in_use"])
        for c in loop.completions():
            comps.append(c)
            i = c["tag"]
            if c["status"] == 0:
                results[i] = _collect(loop, c["request"], len(requests[i][1]), len(scenes[requests[i][0]].objects))
            loop.release(c["request"])
        assert time.perf_counter() - t0 < 120, "serving loop did not finish"
    st = loop.stats()
    st["peak_bytes"] = peak
    return results, comps, st


def _equal(a, b, what):
    for v, (x, y) in enumerate(zip(a, b)):
        for k in ("counters", "indirect", "draws", "lod"):
            np.testing.assert_array_equal(x[k], y[k], err_msg=f"{what}: view {v} {k}")


def test_results_same_alone_and_in_the_mix(cuda):
    scenes, vgs, pool, depths, requests = _world()
    mixed, comps, st = _serve(vgs, scenes, pool, depths, requests, slots=3, max_views=32)
    assert all(c["status"] == 0 for c in comps)
    assert max(c["batch_requests"] for c in comps) > 1, "requests of a scene were batched together"
    assert st["batches"] < len(requests)
    alone, comps1, _ = _serve(vgs, scenes, pool, depths, requests, slots=1, max_views=32, max_requests_per_batch=1)
    assert all(c["batch_requests"] == 1 for c in comps1)
    for i in range(len(requests)):
        _equal(mixed[i], alone[i], f"request {i}")
    # Against the oracle, for a few requests.
    for i in range(0, len(requests), 8):
        sid, idx = requests[i]
        for v, p in enumerate(idx[:3]):
            view = pool[p]
            ref = O.run_view(scenes[sid], view.camera, view.width, view.height, O.hiz_build(view.depth),
                             view.lod_threshold_px, None, 11, 4, cull_dtype())
            np.testing.assert_array_equal(mixed[i][v]["lod"], ref["selected"], err_msg=f"request {i} view {v}: LOD")
            np.testing.assert_array_equal(mixed[i][v]["counters"], ref["counters"], err_msg=f"request {i} view {v}")
            np.testing.assert_array_equal(mixed[i][v]["indirect"], ref["indirect"], err_msg=f"request {i} view {v}")


def test_budget_gates_admission(cuda):
    from helio_b200.passes import ServeLoop

    scenes, vgs, pool, depths, requests = _world(n_requests=8, seed=9)
    # One request at a time: the largest footprint of a single batch.
    alone, _, st1 = _serve(vgs, scenes, pool, depths, requests, slots=1, max_views=16, max_requests_per_batch=1)
    single = st1["peak_bytes"] - st1["scene_bytes"]
    # Two slots, but a budget that holds the scenes and one such batch: never two at once.
    tight, comps, st2 = _serve(vgs, scenes, pool, depths, requests, slots=2, max_views=16, max_requests_per_batch=1,
                               hbm_budget_bytes=st1["scene_bytes"] + single + single // 20)
    assert all(c["status"] == 0 for c in comps)
    assert st2["peak_bytes"] <= st1["scene_bytes"] + single + single // 20
    for i in range(len(requests)):
        _equal(alone[i], tight[i], f"request {i} under a tight budget")
    # A budget below a scene's own bytes refuses the scene.
    small = ServeLoop(slots=1, max_views=16, hbm_budget_bytes=1 << 10)
    with pytest.raises(Exception):
        small.add_scene(vgs[2])


def test_arrivals_while_running_match_alone(cuda):
    """Requests submitted while launches are on the device join at the next pump; every
    result equals the one the request gets alone."""
    import time

    from helio_b200.passes import ServeLoop

    scenes, vgs, pool, depths, requests = _world(n_requests=30, seed=21)
    alone, _, _ = _serve(vgs, scenes, pool, depths, requests, slots=1, max_views=32, max_requests_per_batch=1)
    loop = ServeLoop(slots=3, max_views=16)
    ids = [loop.add_scene(vs) for vs in vgs]
    t0 = time.perf_counter()
    got, comps, submitted_while_running = {}, [], 0

    def drain():
        for c in loop.completions():  # read and release as a server would
            assert c["status"] == 0
            i = c["tag"]
            got[i] = _collect(loop, c["request"], len(requests[i][1]), len(scenes[requests[i][0]].objects))
            loop.release(c["request"])
            comps.append(c)

    for i, (sid, idx) in enumerate(requests):
        if loop.stats()["running"] > 0:
            submitted_while_running += 1
        loop.submit(ids[sid], _spec(pool, depths, idx), time.perf_counter() - t0, tag=i)
        loop.pump(time.perf_counter() - t0)
        drain()
    while len(comps) < len(requests):
        loop.pump(time.perf_counter() - t0)
        drain()
        assert time.perf_counter() - t0 < 120, "serving loop did not finish"
    assert submitted_while_running > 0, "no request arrived while a launch was on the device"
    for i in range(len(requests)):
        _equal(alone[i], got[i], f"request {i}")


def test_launches_of_different_slots_overlap_on_the_device(cuda):
    """Three requests of 32 views over a 5M-meshlet scene, submitted together, go to three
    slots in one pump; once the slots' buffers are sized, their launches' device
    intervals (events on the slots' streams) intersect: the batches run on the device at
    the same time."""
    import time

    import torch
    from helio_b200 import scene as S
    from helio_b200.passes import ServeLoop, VgScene

    sc = S.make_scene(1100, 50000, 100, 4, 0, 100.0, lod_error_mode=1, mesh_library=64)
    vs = VgScene()
    vs.upload(S.frame_data(sc))
    pool = S.multiview_set(78, depth=True, scale=0.5)
    depths = [torch.from_numpy(np.ascontiguousarray(v.depth)).cuda() for v in pool]
    loop = ServeLoop(slots=3, max_views=32, max_requests_per_batch=1)
    sid = loop.add_scene(vs)
    for rnd in range(2):  # the first round sizes every slot's buffers (allocation is slow and synchronous)
        for r in range(3):
            loop.submit(sid, _spec(pool, depths, list(range(1 + 21 * r, 33 + 21 * r))), 0.0, tag=r)
        assert loop.pump(0.0) == 0 and loop.stats()["running"] == 3
        comps, t0 = [], time.perf_counter()
        while len(comps) < 3:
            loop.pump(time.perf_counter() - t0)
            comps.extend(loop.completions())
            assert time.perf_counter() - t0 < 60
        for c in comps:
            loop.release(c["request"])
    assert all(c["status"] == 0 for c in comps)
    iv = sorted((c["device_start_ms"], c["device_end_ms"]) for c in comps)
    assert len(set(iv)) == 3
    assert any(b[0] < a[1] for a, b in zip(iv, iv[1:])), f"no two launches overlapped on the device: {iv}"
