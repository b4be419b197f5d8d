"""The oracle and the host helpers against every known-answer test that the
reference's own test files hold for this path (tests/golden/reference_kats.json,
regenerated by tests/golden/extract_kats.py). CPU only."""
import ctypes as C
import json
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle as O

KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())


@pytest.mark.parametrize("k", KATS["mip_levels"], ids=lambda k: k["at"].split("/")[-1])
def test_mip_levels(k):
    from helio_b200 import native as N

    assert O.mip_levels(k["w"], k["h"]) == k["levels"]
    assert N.cull_lib().helio_mip_levels(k["w"], k["h"]) == k["levels"]


@pytest.mark.parametrize("k", KATS["query_mip"], ids=lambda k: k["at"].split("/")[-1])
def test_query_mip_is_exact_ceil_log2(k):
    # u32(ceil(log2(max(w, h)))) as the shaders' pick_mip computes it, without the clamp.
    assert O.lib().oracle_ceil_log2(float(max(k["w"], k["h"]))) == k["mip"]


@pytest.mark.parametrize("k", KATS["mip_dim"], ids=lambda k: k["at"].split("/")[-1])
def test_mip_dimensions(k):
    base, mip = k["base"], k["mip"]
    if mip < 12 and mip < O.mip_levels(base, base):
        levels = O.hiz_build(np.zeros((1, base), np.float32))
        assert levels[mip].shape[1] == k["dim"]
    assert max(base >> mip, 1) == k["dim"]


@pytest.mark.parametrize("k", KATS["occluded"], ids=lambda k: k["at"].split("/")[-1])
def test_occlusion_rule(k):
    # The shaders add a 1/65536 bias to the strictly-greater rule of the test.
    assert O.hiz_occludes(k["near"], k["hiz"]) == k["occluded"]


@pytest.mark.parametrize("k", KATS["sphere_plane"], ids=lambda k: k["at"].split("/")[-1])
def test_sphere_vs_planes(k):
    planes = list(k["planes"])
    while len(planes) < 6:  # a single plane: pad with planes every point satisfies
        planes.append([0.0, 0.0, 0.0, 1e30])
    assert O.sphere_visible(planes, k["center"], k["radius"]) == k["visible"]


@pytest.mark.parametrize("k", KATS["instance_cull"], ids=lambda k: k["at"].split("/")[-1])
def test_instance_cull_data(k):
    from helio_b200 import native as N

    inst = np.zeros(1, np.dtype(N.GpuInstanceData))
    inst["model"][0] = [float(x) for x in k["model"]]
    out = O.instance_cull_data(inst, np.dtype(N.InstanceCullData))[0]
    if "valid" in k:
        assert out["valid_transform"] == k["valid"]
    if "cone" in k:
        assert out["cone_cull_enabled"] == k["cone"]
    if "max_scale" in k:
        assert out["max_scale"] == k["max_scale"] and out["min_scale"] == k["min_scale"]


@pytest.mark.parametrize("k", KATS["select_lod"], ids=lambda k: k["at"].split("/")[-1])
def test_select_object_lod(k):
    assert O.select_lod(k["errors"], k["lod_count"], k["max_scale"], k["focal"], k["closest"],
                        k["max_error"]) == k["lod"]


@pytest.mark.parametrize("k", KATS["cone_reject"], ids=lambda k: k["at"].split("/")[-1])
def test_cone_reject(k):
    assert O.cone_reject(k["camera"], k["apex"], k["axis"], k["cutoff"]) == k["reject"]


def test_farthest_corner_prevents_occlusion():
    k = KATS["farthest_corner"]
    far = float(np.max(np.array(k["samples"], np.float32)))
    assert far == pytest.approx(k["max"])
    assert O.hiz_occludes(k["near"], far) == k["occluded"]


def test_counter_decode():
    from helio_b200.passes import VirtualGeometryDebugStats

    k = KATS["counter_decode"]
    s = VirtualGeometryDebugStats.from_counters(k["counters"])
    assert s.visible_meshlets == k["visible_meshlets"] and s.rejected_meshlets == k["rejected_meshlets"]
    assert s.visible_objects() == k["visible_objects"]
    assert list(s.selected_lod_range()) == k["lod_range"]
    assert s.max_available_lod == k["max_available_lod"]
    assert VirtualGeometryDebugStats.from_counters([0] * k["short_is_none"]) is None


def test_lod_quality_thresholds():
    from helio_b200 import native as N

    k = KATS["lod_quality_px"]
    lib = N.cull_lib()
    for q, name in enumerate(["low", "medium", "high", "ultra"]):
        assert lib.helio_lod_max_error_pixels(q) == k[name]


def test_publication_budget():
    from helio_b200.passes import VirtualGeometryBudget

    k = KATS["budget"]
    b = VirtualGeometryBudget()
    assert b.max_published_meshlets == k["default"]
    assert b.publication_bytes() == k["publication_bytes"]
    for worst, got in k["clamp"]:
        assert b.clamp_draw_count(worst) == got
    with pytest.raises(ValueError):
        VirtualGeometryBudget(0)


def test_work_spans():
    from helio_b200.scene import work_items_for

    k = KATS["work_spans"]
    assert [list(x) for x in work_items_for(k["objects"])] == k["expected"]


def test_unique_meshlets_on_the_oracle():
    from helpers import kat_unique_meshlets_library

    k = KATS["unique_meshlets"]
    lib, ids = kat_unique_meshlets_library(k)
    out = O.vg_rebuild(lib.pool, lib.meshes, lib.slot_mesh, lib.slot_instances)
    assert out["meshlets"]["first_index"].tolist() == k["expected_first_index"]
    bases = [k["bases"][str(r)] for r in k["references"]]
    assert out["objects"]["lod_first_meshlets"][:, 0].tolist() == bases


def test_work_spans_on_the_oracle():
    from helpers import kat_work_spans_library

    k = KATS["work_spans"]
    lib = kat_work_spans_library(k)
    out = O.vg_rebuild(lib.pool, lib.meshes, lib.slot_mesh, lib.slot_instances)
    ids = [obj for obj, _ in k["objects"]]
    got = [[ids[i["object_index"]], int(i["local_meshlet_base"])] for i in out["work_items"]]
    assert got == k["expected"]
    assert out["max_draw_count"] == sum(mx for _, mx in k["objects"])


def test_layout_sizes():
    from helio_b200 import native as N

    k = KATS["layout_sizes"]
    for name in ("GpuMeshletEntry", "GpuVgObject", "GpuVgDraw", "GpuVgWorkItem", "InstanceCullData",
                 "GpuInstanceData", "GpuCameraUniforms"):
        assert C.sizeof(getattr(N, name)) == k[name], name
    assert C.sizeof(N.DrawIndexedIndirectArgs) == k["DrawIndexedIndirect"]


def test_benchmark_scene_on_the_oracle():
    """meshlet_cull_benchmark.rs:284-294 and :368 on the CPU restatement (smaller total)."""
    from helpers import benchmark_scene, cull_dtype

    sc, v = benchmark_scene(256, 64)
    total = 256 * 64
    levels = [np.ones((1, 1), np.float32)]
    r = O.run_view(sc, v.camera, v.width, v.height, levels, 2.0, total, 2, 1, cull_dtype())
    assert list(r["counters"][:2]) == [total, 0]
    r = O.run_view(sc, v.camera, v.width, v.height, levels, 2.0, total - 17, 2, 1, cull_dtype())
    assert list(r["counters"][:2]) == [total, 17]
