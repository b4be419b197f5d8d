"""The seeded generator: deterministic bytes (independent of the thread count), the
reference's scene-build invariants, and the workload shapes."""
import hashlib

import numpy as np
import pytest

from helio_b200 import scene as S


def _digest(sc) -> str:
    h = hashlib.sha256()
    for a in (sc.meshlets, sc.objects, sc.instances, sc.work_items, sc.aabbs, sc.draw_calls):
        h.update(a.tobytes())
    return h.hexdigest()


def test_scene_is_deterministic_across_thread_counts(native_built):
    a = S.make_scene(123, 500, 100, 4, 1, 1000.0, 8, 20.0, threads=1)
    b = S.make_scene(123, 500, 100, 4, 1, 1000.0, 8, 20.0, threads=7)
    assert _digest(a) == _digest(b)
    c = S.make_scene(124, 500, 100, 4, 1, 1000.0, 8, 20.0, threads=7)
    assert _digest(a) != _digest(c)


def test_depth_is_deterministic(native_built):
    d1 = S.make_depth(5, 333, 211, 300, 0.1, 1000.0, False, threads=1)
    d2 = S.make_depth(5, 333, 211, 300, 0.1, 1000.0, False, threads=5)
    assert np.array_equal(d1, d2)
    assert d1.max() == 1.0 and 0.0 <= d1.min() < 1.0


def test_scene_build_invariants(native_built):
    """rebuild.rs:120-162: per-LOD ranges inside the descriptor array, spans of 64 over
    max_meshlet_count, max_draw_count = sum of max_meshlet_count."""
    sc = S.make_scene(7, 300, 100, 4, 0, 100.0)
    obj = sc.objects
    assert sc.max_draw_count == int(obj["max_meshlet_count"].sum())
    assert list(obj["lod_meshlet_counts"][0, :4]) == [100, 50, 25, 13]
    end = obj["lod_first_meshlets"][:, :4] + obj["lod_meshlet_counts"][:, :4]
    assert end.max() <= len(sc.meshlets)
    expect = S.work_items_for([(i, int(m)) for i, m in enumerate(obj["max_meshlet_count"])])
    assert [tuple(x) for x in sc.work_items.tolist()] == expect
    errs = obj["lod_errors"][:, 1:4]
    assert np.all(np.diff(errs, axis=1) >= 0) and errs.min() >= 1e-4 and errs.max() <= 1e-1
    # index counts <= 124 triangles, instance bounds / AABB consistency (helpers.rs:54-66)
    assert sc.meshlets["index_count"].max() <= 372
    c, r = sc.instances["bounds"][:, :3], sc.instances["bounds"][:, 3:]
    np.testing.assert_array_equal(sc.aabbs["min"], (c - r).astype(np.float32))


@pytest.mark.parametrize("cfg", [0, 1, 2, 3])
def test_workload_shapes(native_built, cfg):
    w = S.config(cfg, scale=0.01)
    assert len(w.views) == (85 if cfg == 3 else 1)
    kinds = [v.kind for v in w.views]
    if cfg == 3:
        assert kinds.count("main") == 1 and kinds.count("cascade") == 4
        assert kinds.count("spot") == 16 and kinds.count("probe") == 64
    per = {0: 64, 1: 100, 2: 100, 3: 50}[cfg]
    assert w.scene.lod0_meshlets == per
