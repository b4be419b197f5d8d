"""Shared drivers of the CUDA path (through the C-ABI) and of the oracle, for the tests."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O


def u32(t) -> np.ndarray:
    """Device tensor (int32 words) -> numpy uint32 copy."""
    return t.cpu().numpy().view(np.uint32)


def cull_dtype():
    from helio_b200 import native as N

    return np.dtype(N.InstanceCullData)


def gpu_hiz(depth: np.ndarray, alias: bool = False, pitch: int | None = None):
    """Builds the pyramid on the GPU; returns (pass, list of numpy levels)."""
    import torch
    from helio_b200.passes import HiZBuildPass

    h, w = depth.shape
    if pitch and pitch != w:
        buf = torch.full((h, pitch), -7.0, dtype=torch.float32, device="cuda")
        buf[:, :w] = torch.from_numpy(np.ascontiguousarray(depth)).cuda()
        d = buf[:, :w]
    else:
        d = torch.from_numpy(np.ascontiguousarray(depth)).cuda()
    hz = HiZBuildPass(w, h, alias_mip0=alias)
    hz.prepare(d)
    hz.execute()
    torch.cuda.synchronize()
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


def oracle_vg_view(scene, view, levels, lod_threshold=2.0, capacity=None, counter_count=11, threads=4):
    return O.run_view(scene, view.camera, view.width, view.height, levels, lod_threshold, capacity, counter_count,
                      threads, cull_dtype())


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
