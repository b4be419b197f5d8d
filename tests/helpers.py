"""Shared drivers of the CUDA path (through the C-ABI) and of the oracle, for the tests."""
from __future__ import annotations

import os

import numpy as np

from oracle import oracle as O


def oracle_threads() -> int:
    """Host threads for the oracle's select / cull (its merge is deterministic)."""
    return max(1, os.cpu_count() or 1)


def u32(t) -> np.ndarray:
    """Device tensor (int32 words) -> numpy uint32 copy."""
    return t.cpu().numpy().view(np.uint32)


def cull_dtype():
    from helio_b200 import native as N

    return np.dtype(N.InstanceCullData)


def gpu_hiz(depth: np.ndarray, alias: bool = False, pitch: int | None = None, tma: bool = True):
    """Builds the pyramid on the GPU; returns (pass, list of numpy levels). tma=False
    forces the 128-bit-load path (depth TMA cannot address takes it anyway)."""
    import torch
    from helio_b200.passes import HiZBuildPass

    h, w = depth.shape
    if pitch and pitch != w:
        buf = torch.full((h, pitch), -7.0, dtype=torch.float32, device="cuda")
        buf[:, :w] = torch.from_numpy(np.ascontiguousarray(depth)).cuda()
        d = buf[:, :w]
    else:
        d = torch.from_numpy(np.ascontiguousarray(depth)).cuda()
    hz = HiZBuildPass(w, h, alias_mip0=alias, tma=tma)
    hz.prepare(d)
    hz.execute()
    torch.cuda.synchronize()
    hz.device_status()
    pyr = hz.publish()
    levels = [hz.level(l).cpu().numpy().copy() for l in range(pyr.mip_count)]
    hz._keep = d
    return hz, levels


def gpu_vg_view(scene, view, hz=None, lod_quality=1, publication_limit=0, counter_count=11, frame=None,
                vg_pass=None, execute_times=1):
    """Runs Hi-Z (unless given) + VirtualGeometryPass for one view; returns numpy outputs."""
    import torch
    from helio_b200 import scene as S
    from helio_b200.passes import VirtualGeometryPass, camera_bytes

    if hz is None:
        hz, _ = gpu_hiz(view.depth)
    vg = vg_pass or VirtualGeometryPass(view.width, view.height, lod_quality, publication_limit, counter_count)
    vg.prepare(frame or S.frame_data(scene))
    cam = torch.from_numpy(camera_bytes(view.camera)).cuda()
    for _ in range(execute_times):
        vg.execute(cam, hz.publish())
    torch.cuda.synchronize()
    vg.device_status()
    out = vg.outputs()
    counters = u32(out["counters"])
    n = int(min(counters[0], out["capacity"]))
    objects = u32(out["objects"])
    return {
        "counters": counters,
        "indirect": u32(out["indirect"])[:n],
        "draws": u32(out["draws"])[:n],
        "visibility": u32(out["visibility"])[: len(scene.work_items)],
        "selected": objects[: len(scene.objects), 3].copy(),
        "pass": vg,
        "hz": hz,
    }


def oracle_vg_view(scene, view, levels, lod_threshold=2.0, capacity=None, counter_count=11, threads=None):
    return O.run_view(scene, view.camera, view.width, view.height, levels, lod_threshold, capacity, counter_count,
                      threads or oracle_threads(), cull_dtype())


def assert_vg_equal(g, o, counter_count=11):
    np.testing.assert_array_equal(g["selected"], o["selected"], err_msg="selected LOD + 1 per object")
    np.testing.assert_array_equal(g["counters"][:counter_count], o["counters"][:counter_count], err_msg="counters")
    np.testing.assert_array_equal(g["visibility"], o["visibility"], err_msg="visibility bitmask")
    np.testing.assert_array_equal(g["indirect"], o["indirect"], err_msg="indirect args")
    np.testing.assert_array_equal(g["draws"], o["draws"], err_msg="draw metadata")


def benchmark_scene(objects, per_object):
    """The constant scene of crates/examples/meshlet_cull_benchmark.rs:468-560."""
    from helio_b200 import native as N
    from helio_b200 import scene as S

    m = np.zeros(per_object, S.DT_MESHLET)
    m["center"] = (0.0, 0.0, -10.0)
    m["radius"] = 0.25
    m["cone_apex"] = (0.0, 0.0, -10.0)
    m["cone_cutoff"] = 2.0
    m["cone_axis"] = (0.0, 0.0, 1.0)
    m["index_count"] = 3
    inst = np.zeros(objects, S.DT_INSTANCE)
    inst["model"] = np.eye(4, dtype=np.float32).reshape(16)
    inst["normal_mat"] = np.array([1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0], np.float32)
    inst["bounds"] = (0.0, 0.0, -10.0, 1.0)
    inst["lightmap_index"] = 0xFFFFFFFF
    obj = np.zeros(objects, S.DT_OBJECT)
    obj["instance_index"] = np.arange(objects)
    obj["lod_count"] = 1
    obj["max_meshlet_count"] = per_object
    obj["local_bounds"] = (0.0, 0.0, -10.0, 1.0)
    obj["lod_meshlet_counts"][:, 0] = per_object
    spans = (per_object + 63) // 64
    items = np.zeros(objects * spans, S.DT_ITEM)
    items["object_index"] = np.repeat(np.arange(objects), spans)
    items["local_meshlet_base"] = np.tile(np.arange(spans) * 64, objects)
    cam = S.perspective((0, 0, 0), (0, 0, -1), (0, 1, 0), 60.0, 16 / 9, 0.1, 1000.0)
    sc = S.Scene(m, obj, inst, items, np.zeros(objects, S.DT_AABB), np.zeros(objects, S.DT_DRAWCALL),
                 objects * per_object, per_object)
    return sc, S.View(cam, 1920, 1080, np.ones((1, 1), np.float32))


def random_library(seed: int, pool: int = 500, meshes: int = 40, slots: int = 600, max_count: int = 300):
    """A mesh library with the cases the rebuild skips or shares: free slots, indices past
    the table, meshes without descriptors or without LODs, repeated references."""
    from helio_b200 import native as N
    from helio_b200 import scene as S

    rng = np.random.default_rng(seed)
    p = np.frombuffer(rng.integers(0, 2**32, size=pool * 16, dtype=np.uint32).tobytes(), S.DT_MESHLET).copy()
    m = np.zeros(meshes, S.DT_MESH)
    m["meshlet_count"] = rng.integers(0, 40, meshes)
    m["meshlet_count"][rng.random(meshes) < 0.15] = 0
    m["first_meshlet"] = rng.integers(0, pool - m["meshlet_count"] + 1)
    m["lod_count"] = rng.integers(0, 9, meshes)
    m["lod_count"][rng.random(meshes) < 0.15] = 0
    m["max_meshlet_count"] = rng.integers(0, max_count, meshes)
    m["local_bounds"] = rng.normal(size=(meshes, 4)).astype(np.float32)
    m["lod_errors"] = rng.random((meshes, 8)).astype(np.float32)
    m["lod_first_meshlets"] = rng.integers(0, 1000, (meshes, 8))
    m["lod_meshlet_counts"] = rng.integers(0, 100, (meshes, 8))
    sm = rng.integers(0, meshes, slots).astype(np.uint32)
    r = rng.random(slots)
    sm[r < 0.1] = N.VG_NO_MESH
    sm[(r >= 0.1) & (r < 0.15)] = meshes + rng.integers(0, 5, int(((r >= 0.1) & (r < 0.15)).sum()))
    inst = np.frombuffer(rng.integers(0, 2**32, size=slots * 36, dtype=np.uint32).tobytes(), S.DT_INSTANCE).copy()
    return S.Library(p, m, sm, inst)


def kat_unique_meshlets_library(k: dict):
    """rebuild.rs repeated_instances_share_one_descriptor_copy as a library: mesh ids in
    ascending order become indices; the test's helper record has one LOD of one meshlet."""
    from helio_b200 import scene as S

    ids = sorted(k["meshes"], key=int)
    pool = np.zeros(sum(len(v) for v in k["meshes"].values()), S.DT_MESHLET)
    m = np.zeros(len(ids), S.DT_MESH)
    at = 0
    for i, mid in enumerate(ids):
        fi = k["meshes"][mid]
        pool["first_index"][at:at + len(fi)] = fi
        pool["index_count"][at:at + len(fi)] = 3
        m[i]["first_meshlet"], m[i]["meshlet_count"] = at, len(fi)
        at += len(fi)
    m["lod_count"] = 1
    m["max_meshlet_count"] = 1
    m["local_bounds"] = (0.0, 0.0, 0.0, 1.0)
    m["lod_meshlet_counts"] = 1
    slots = np.array([ids.index(str(r)) for r in k["references"]], np.uint32)
    inst = np.zeros(len(slots), S.DT_INSTANCE)
    return S.Library(pool, m, slots, inst), ids


def kat_work_spans_library(k: dict):
    """rebuild.rs work_items_cover_exact_fixed_meshlet_spans as a library: one used mesh
    per listed object with its max_meshlet_count, one slot each, in order."""
    from helio_b200 import scene as S

    n = len(k["objects"])
    pool = np.zeros(1, S.DT_MESHLET)
    m = np.zeros(n, S.DT_MESH)
    m["meshlet_count"] = 1
    m["lod_count"] = 1
    m["max_meshlet_count"] = [mx for _, mx in k["objects"]]
    return S.Library(pool, m, np.arange(n, dtype=np.uint32), np.zeros(n, S.DT_INSTANCE))


# ── batched multi-view cull ──────────────────────────────────────────────────

def run_batch(scene, views, span_visibility=True, alias=False, capacities=None, repeats=1, max_ctas=0, cull_ctas=0):
    import torch
    from helio_b200 import scene as S
    from helio_b200.passes import BatchedCull, VgScene

    vs = VgScene()
    vs.upload(S.frame_data(scene))
    depths = [torch.from_numpy(np.ascontiguousarray(v.depth)).cuda() for v in views]
    b = BatchedCull(len(views), span_visibility=span_visibility, max_ctas=max_ctas, cull_ctas=cull_ctas)
    specs = []
    for i, (v, d) in enumerate(zip(views, depths)):
        spec = {"camera": v.camera, "depth": d, "alias_mip0": alias, "lod_threshold_px": v.lod_threshold_px}
        if capacities:
            spec["draw_capacity"] = capacities[i]
        specs.append(spec)
    b.prepare(vs, specs)
    for _ in range(repeats):
        b.execute()
    torch.cuda.synchronize()
    b.status()
    return b, vs, depths


def gather(b, v, n_objects):
    from helio_b200.passes import device_view

    o = b.view_outputs(v)
    counters = u32(o["counters"])
    n = int(min(counters[0], o["capacity"]))
    p = o["pyramid"]
    levels = [device_view(p.levels[l], (p.height[l], p.width[l]), "<f4", (p.pitch[l] * 4, 4)).cpu().numpy()
              for l in range(p.mip_count)]
    return {"counters": counters, "indirect": u32(o["indirect"])[:n], "draws": u32(o["draws"])[:n],
            "lod": o["lod"].cpu().numpy()[:n_objects].astype(np.uint32), "levels": levels, "capacity": o["capacity"]}


def check_view(scene, view, got, spans_view, vis_view, cap):
    """One view of a batch against the oracle: every pyramid level, selected LOD per
    object, counters, indirect args and draws in canonical order, and (when given) the
    view's active spans and their visibility words. Returns the oracle's statistics."""
    levels = O.hiz_build(view.depth)
    for l, (a, r) in enumerate(zip(got["levels"], levels)):
        np.testing.assert_array_equal(a.view(np.uint32), r.view(np.uint32), err_msg=f"level {l}")
    ref = O.run_view(scene, view.camera, view.width, view.height, levels, view.lod_threshold_px, cap, 11,
                     oracle_threads(), cull_dtype())
    np.testing.assert_array_equal(got["lod"], ref["selected"], err_msg="selected LOD + 1")
    np.testing.assert_array_equal(got["counters"], ref["counters"], err_msg="counters")
    np.testing.assert_array_equal(got["indirect"], ref["indirect"], err_msg="indirect")
    np.testing.assert_array_equal(got["draws"], ref["draws"], err_msg="draws")
    if spans_view is not None:
        # active work items (span base below the selected LOD's count), in order
        items = scene.work_items
        sel = ref["selected"][items["object_index"]]
        lod = np.maximum(sel.astype(np.int64) - 1, 0)
        cnt = np.where(sel > 0, scene.objects["lod_meshlet_counts"][items["object_index"], lod], 0)
        active = items["local_meshlet_base"] < cnt
        real = spans_view[(spans_view[:, 1] & 0x7F) > 0]
        assert len(real) == int(active.sum())
        np.testing.assert_array_equal(real[:, 3], items["object_index"][active], err_msg="span objects")
        if vis_view is not None:
            np.testing.assert_array_equal(vis_view[(spans_view[:, 1] & 0x7F) > 0], ref["visibility"][active],
                                          err_msg="span visibility")
    return ref["stats"]


def check_batch(w, views, **kw):
    """Runs a batch over `views` of workload w and checks every view against the oracle."""
    b, vs, _ = run_batch(w.scene, views, **kw)
    sp = b.spans()
    spans = u32(sp["spans"])
    start = u32(sp["view_span_start"])
    vis = u32(sp["visibility"]) if "visibility" in sp else None
    totals = {"marginal_decisions": 0, "meshlets_tested": 0}
    for i, v in enumerate(views):
        got = gather(b, i, len(w.scene.objects))
        sv = spans[start[i]:start[i + 1]]
        st = check_view(w.scene, v, got, sv, vis[start[i]:start[i + 1]] if vis is not None else None, got["capacity"])
        totals["marginal_decisions"] += st.marginal_decisions
        totals["meshlets_tested"] += st.meshlets_tested
    b._parity_stats = totals
    return b
