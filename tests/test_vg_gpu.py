"""VirtualGeometryPass cull half: CUDA vs oracle. Bit-exact selected LODs, counters,
visibility bitmask, indirect args and draw metadata in the canonical (work item, lane)
order; plus the reference benchmark's invariants and edge cases."""
import numpy as np
import pytest

from helpers import assert_vg_equal, benchmark_scene as _benchmark_scene, gpu_hiz, gpu_vg_view, oracle_vg_view, u32

pytestmark = pytest.mark.gpu


def _workload(cfg, scale):
    from helio_b200 import scene as S

    return S.config(cfg, scale=scale)


@pytest.mark.parametrize("cfg,scale", [(0, 1.0), (1, 0.25), (2, 0.04), (3, 0.02)])
def test_vg_matches_oracle(cuda, cfg, scale):
    from oracle import oracle as O

    w = _workload(cfg, scale)
    for view in w.views[:6]:
        g = gpu_vg_view(w.scene, view)
        # Whole pipeline against the oracle's own pyramid (Hi-Z build included).
        o = oracle_vg_view(w.scene, view, O.hiz_build(view.depth))
        assert_vg_equal(g, o)


def _levels(hz):
    return [hz.level(l).cpu().numpy().copy() for l in range(hz.publish().mip_count)]


def test_vg_full_config1(cuda):
    """1M LOD0 meshlets, 1920x1080, bit-exact against the oracle."""
    w = _workload(1, 1.0)
    v = w.views[0]
    g = gpu_vg_view(w.scene, v)
    o = oracle_vg_view(w.scene, v, _levels(g["hz"]), threads=8)
    assert_vg_equal(g, o)
    assert o["counters"][0] > 0


@pytest.mark.parametrize("counter_count", [2, 11])
def test_vg_counter_layouts(cuda, counter_count):
    w = _workload(0, 1.0)
    v = w.views[0]
    g = gpu_vg_view(w.scene, v, counter_count=counter_count)
    o = oracle_vg_view(w.scene, v, _levels(g["hz"]), counter_count=counter_count)
    assert_vg_equal(g, o, counter_count)


@pytest.mark.parametrize("quality,thr", [(0, 4.0), (2, 1.0), (3, 0.5)])
def test_vg_lod_quality(cuda, quality, thr):
    w = _workload(1, 0.1)
    v = w.views[0]
    g = gpu_vg_view(w.scene, v, lod_quality=quality)
    o = oracle_vg_view(w.scene, v, _levels(g["hz"]), lod_threshold=thr)
    assert_vg_equal(g, o)


def test_vg_capacity_overflow(cuda):
    """Draws beyond the publication capacity are counted in counters[1], not written
    (vg_cull.wgsl:247-263)."""
    w = _workload(0, 1.0)
    v = w.views[0]
    cap = 1000
    g = gpu_vg_view(w.scene, v, publication_limit=cap)
    o = oracle_vg_view(w.scene, v, _levels(g["hz"]), capacity=cap)
    assert o["counters"][0] > cap
    assert o["counters"][1] == o["counters"][0] - cap
    assert_vg_equal(g, o)


def test_vg_deterministic_and_repeatable(cuda):
    w = _workload(2, 0.05)
    v = w.views[0]
    g1 = gpu_vg_view(w.scene, v, execute_times=3)
    g2 = gpu_vg_view(w.scene, v, hz=g1["hz"], vg_pass=g1["pass"])
    for k in ("counters", "indirect", "draws", "visibility", "selected"):
        np.testing.assert_array_equal(g1[k], g2[k])


def test_vg_device_resident_upload_and_dirty_patch(cuda):
    """buffer_version upload from device memory, then an instance_version dirty-range patch."""
    import torch
    from helio_b200 import scene as S

    w = _workload(1, 0.05)
    sc, v = w.scene, w.views[0]
    dev = {k: torch.from_numpy(getattr(sc, k).view(np.uint8)).cuda()
           for k in ("meshlets", "objects", "instances", "work_items")}
    g = gpu_vg_view(sc, v, frame=S.frame_data(sc, 7, 1, device=dev))
    o = oracle_vg_view(sc, v, _levels(g["hz"]))
    assert_vg_equal(g, o)
    # Move a dirty range of instances, publish it via instance_version.
    inst2 = sc.instances.copy()
    lo, n = 10, 40
    inst2["model"][lo:lo + n, 12:15] *= np.float32(0.5)
    sc2 = S.Scene(sc.meshlets, sc.objects, inst2, sc.work_items, sc.aabbs, sc.draw_calls, sc.max_draw_count,
                  sc.lod0_meshlets)
    vg = g["pass"]
    g2 = gpu_vg_view(sc2, v, hz=g["hz"], vg_pass=vg, frame=S.frame_data(sc2, 7, 2, dirty=(lo, n)))
    o2 = oracle_vg_view(sc2, v, _levels(g["hz"]))
    assert_vg_equal(g2, o2)


@pytest.mark.parametrize("objects,per_object", [(1, 65536), (16, 4096), (1024, 64), (8192, 8)])
def test_benchmark_cases_emit_every_meshlet(cuda, objects, per_object):
    """meshlet_cull_benchmark.rs:235-240,284-294: every meshlet is attempted, no overflow."""
    sc, v = _benchmark_scene(objects, per_object)
    total = objects * per_object
    hz, _ = gpu_hiz(np.ones((1, 1), np.float32))
    g = gpu_vg_view(sc, v, hz=hz, counter_count=2, publication_limit=total)
    assert list(g["counters"][:2]) == [total, 0]
    assert len(g["indirect"]) == total
    np.testing.assert_array_equal(g["indirect"][:, 4], np.arange(total))  # first_instance = slot
    np.testing.assert_array_equal(g["draws"][:, 1], np.tile(np.arange(per_object), objects))


def test_benchmark_overflow_probe(cuda):
    """meshlet_cull_benchmark.rs:368: capacity TOTAL - 17 gives counters [TOTAL, 17]."""
    sc, v = _benchmark_scene(1024, 64)
    total = 1024 * 64
    hz, _ = gpu_hiz(np.ones((1, 1), np.float32))
    g = gpu_vg_view(sc, v, hz=hz, counter_count=2, publication_limit=total - 17)
    assert list(g["counters"][:2]) == [total, 17]


def test_vg_edge_cases(cuda):
    """Out-of-range object / instance indices, zero-LOD objects, spans past the LOD,
    invalid transforms and objects without work items."""
    from helio_b200 import scene as S

    w = _workload(0, 0.05)
    sc, v = w.scene, w.views[0]
    obj = sc.objects.copy()
    inst = sc.instances.copy()
    items = sc.work_items.copy()
    n = len(obj)
    obj["lod_count"][0] = 0
    obj["instance_index"][1] = 10 ** 6
    inst["model"][2, :] = np.nan
    inst["model"][3, 0:3] = 0.0
    # an out-of-range object, a span beyond every LOD, a second span of a 64-meshlet LOD
    items = np.concatenate([items, np.array([(n + 5, 0), (4, 640), (5, 64)], S.DT_ITEM)])
    keep = items["object_index"] != 6  # object 6 keeps no work item
    items = items[keep]
    sc2 = S.Scene(sc.meshlets, obj, inst, items, sc.aabbs, sc.draw_calls, sc.max_draw_count, sc.lod0_meshlets)
    hz, levels = gpu_hiz(v.depth)
    g = gpu_vg_view(sc2, v, hz=hz)
    o = oracle_vg_view(sc2, v, levels)
    assert_vg_equal(g, o)


def test_vg_empty_scene_is_a_no_op(cuda):
    from helio_b200 import scene as S

    w = _workload(0, 0.02)
    sc = w.scene
    empty = S.Scene(sc.meshlets[:0], sc.objects[:0], sc.instances[:0], sc.work_items[:0], sc.aabbs[:0],
                    sc.draw_calls[:0], 0, 64)
    hz, _ = gpu_hiz(w.views[0].depth)
    import torch
    from helio_b200.passes import VirtualGeometryPass, camera_bytes

    vg = VirtualGeometryPass(w.views[0].width, w.views[0].height)
    vg.prepare(S.frame_data(empty))
    vg.execute(torch.from_numpy(camera_bytes(w.views[0].camera)).cuda(), hz.publish())
    torch.cuda.synchronize()
