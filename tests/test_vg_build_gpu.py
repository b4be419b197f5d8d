"""The VG input producer (helio_vg_builder: rebuild_vg_buffers on the device) against
the oracle's restatement, byte for byte: descriptors in first-reference order, objects,
instances, work items and max_draw_count; the reference's own rebuild tests; the
panics of the reference as errors; and a built scene culled by the batched path."""
import json
from pathlib import Path

import numpy as np
import pytest

from helpers import kat_unique_meshlets_library, kat_work_spans_library, random_library
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KATS = json.loads((Path(__file__).parent / "golden" / "reference_kats.json").read_text())


def _dev(a: np.ndarray):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).cuda()


def gpu_build(lib, builder=None):
    from helio_b200.passes import VgBuilder

    b = builder or VgBuilder()
    keep = [_dev(lib.pool), _dev(lib.meshes), _dev(lib.slot_mesh), _dev(lib.slot_instances)]
    b.run(*keep)
    out = b.outputs()
    host = {k: (v.cpu().numpy() if hasattr(v, "cpu") else v) for k, v in out.items()}
    return b, host, keep


def assert_same(host, ref):
    for k in ("meshlets", "objects", "instances", "work_items"):
        np.testing.assert_array_equal(host[k], ref[k].view(np.uint8).reshape(-1), err_msg=k)
    assert host["max_draw_count"] == ref["max_draw_count"]


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_random_library_matches_oracle(cuda, seed):
    lib = random_library(seed)
    ref = O.vg_rebuild(lib.pool, lib.meshes, lib.slot_mesh, lib.slot_instances)
    assert ref is not None and len(ref["objects"]) > 0
    _, host, _ = gpu_build(lib)
    assert_same(host, ref)


def test_many_slots_shared_meshes(cuda):
    # Several blocks of the slot scan, few meshes: most slots are repeated references.
    lib = random_library(11, pool=4000, meshes=300, slots=70000, max_count=700)
    ref = O.vg_rebuild(lib.pool, lib.meshes, lib.slot_mesh, lib.slot_instances)
    _, host, _ = gpu_build(lib)
    assert_same(host, ref)


def test_large_library_takes_the_global_table(cuda):
    # More meshes than the per-block shared table holds: the first references go straight
    # to the one global table.
    lib = random_library(12, pool=20000, meshes=9000, slots=40000, max_count=200)
    ref = O.vg_rebuild(lib.pool, lib.meshes, lib.slot_mesh, lib.slot_instances)
    _, host, _ = gpu_build(lib)
    assert_same(host, ref)


def test_reference_rebuild_tests(cuda):
    k = KATS["unique_meshlets"]
    lib, _ = kat_unique_meshlets_library(k)
    _, host, _ = gpu_build(lib)
    from helio_b200 import scene as S

    m = host["meshlets"].view(S.DT_MESHLET)
    assert m["first_index"].tolist() == k["expected_first_index"]
    objs = host["objects"].view(S.DT_OBJECT)
    assert objs["lod_first_meshlets"][:, 0].tolist() == [k["bases"][str(r)] for r in k["references"]]

    k = KATS["work_spans"]
    lib = kat_work_spans_library(k)
    _, host, _ = gpu_build(lib)
    items = host["work_items"].view(S.DT_ITEM)
    ids = [obj for obj, _ in k["objects"]]
    assert [[ids[i["object_index"]], int(i["local_meshlet_base"])] for i in items] == k["expected"]


def test_reused_builder_grows_and_shrinks(cuda):
    """One builder over libraries of changing size: the output passes run before the host
    has read the totals, with the buffers the builder holds; when those are too small they
    leave and run again once sized. Every run matches the oracle byte for byte, and the
    error of a bad library leaves the builder usable."""
    libs = [random_library(21, slots=300), random_library(22, slots=5000), random_library(23, slots=300),
            random_library(24, slots=5000)]
    b = None
    for i, lib in enumerate(libs * 2):
        ref = O.vg_rebuild(lib.pool, lib.meshes, lib.slot_mesh, lib.slot_instances)
        b, host, _ = gpu_build(lib, b)
        assert_same(host, ref)
        assert b.frame_data().object_count == len(ref["objects"]), f"run {i}"
    bad = random_library(25, slots=5000)
    used = int(bad.slot_mesh[bad.slot_mesh < len(bad.meshes)][0])
    bad.meshes[used]["meshlet_count"] = max(int(bad.meshes[used]["meshlet_count"]), 1)
    bad.meshes[used]["lod_count"] = max(int(bad.meshes[used]["lod_count"]), 1)
    bad.meshes[used]["first_meshlet"] = len(bad.pool)
    from helio_b200 import native as N

    with pytest.raises(N.HelioError):
        gpu_build(bad, b)
    ref = O.vg_rebuild(libs[1].pool, libs[1].meshes, libs[1].slot_mesh, libs[1].slot_instances)
    _, host, _ = gpu_build(libs[1], b)
    assert_same(host, ref)


def test_empty_and_all_free(cuda):
    from helio_b200 import native as N

    lib = random_library(5, slots=64)
    lib.slot_mesh[:] = N.VG_NO_MESH
    b, host, _ = gpu_build(lib)
    f = b.frame_data()
    assert (f.meshlet_count, f.object_count, f.work_item_count, f.max_draw_count) == (0, 0, 0, 0)
    lib.slot_mesh = lib.slot_mesh[:0]
    lib.slot_instances = lib.slot_instances[:0]
    b, host, _ = gpu_build(lib, b)
    assert b.frame_data().object_count == 0


def test_reference_panics_are_errors(cuda):
    from helio_b200 import native as N

    # A used mesh whose descriptors leave the pool.
    lib = random_library(6)
    used = int(lib.slot_mesh[lib.slot_mesh < len(lib.meshes)][0])
    lib.meshes[used]["meshlet_count"] = max(int(lib.meshes[used]["meshlet_count"]), 1)
    lib.meshes[used]["lod_count"] = max(int(lib.meshes[used]["lod_count"]), 1)
    lib.meshes[used]["first_meshlet"] = len(lib.pool)
    assert O.vg_rebuild(lib.pool, lib.meshes, lib.slot_mesh, lib.slot_instances) is None
    with pytest.raises(N.HelioError) as e:
        gpu_build(lib)
    assert e.value.status == N.HELIO_ERR_INVALID_ARG
    # An LOD descriptor offset beyond u32 (mesh base + relative first).
    lib = random_library(7)
    order = [int(m) for m in lib.slot_mesh if m < len(lib.meshes)
             and lib.meshes[m]["meshlet_count"] > 0 and lib.meshes[m]["lod_count"] > 0]
    second = next(m for m in order if m != order[0])
    lib.meshes[second]["lod_first_meshlets"][3] = 0xFFFFFFFF
    assert O.vg_rebuild(lib.pool, lib.meshes, lib.slot_mesh, lib.slot_instances) is None
    with pytest.raises(N.HelioError):
        gpu_build(lib)
    # max_draw_count beyond u32.
    lib = random_library(8)
    lib.meshes["max_meshlet_count"] = 0x7FFFFFFF
    assert O.vg_rebuild(lib.pool, lib.meshes, lib.slot_mesh, lib.slot_instances) is None
    with pytest.raises(N.HelioError):
        gpu_build(lib)
    # A mesh outside the pool that no slot uses is never read.
    lib = random_library(9)
    unused = sorted(set(range(len(lib.meshes))) - set(int(m) for m in lib.slot_mesh))
    if unused:
        lib.meshes[unused[0]]["first_meshlet"] = 10**9
        lib.meshes[unused[0]]["meshlet_count"] = 5
        lib.meshes[unused[0]]["lod_count"] = 1
        ref = O.vg_rebuild(lib.pool, lib.meshes, lib.slot_mesh, lib.slot_instances)
        _, host, _ = gpu_build(lib)
        assert_same(host, ref)


def test_built_scene_culls_like_the_oracle(cuda):
    """Library of a generated scene with free slots -> device rebuild -> device upload ->
    batched cull, against the oracle on a host copy of the same rebuilt arrays."""
    import torch
    from helio_b200 import scene as S
    from helio_b200.passes import BatchedCull, VgScene
    from helpers import check_view, gather

    w = S.config(1, scale=0.05)
    lib = S.library_from_scene(w.scene, free_slots=0.2, seed=3)
    ref = O.vg_rebuild(lib.pool, lib.meshes, lib.slot_mesh, lib.slot_instances)
    b, host, keep = gpu_build(lib)
    assert_same(host, ref)
    # The rebuild of a one-mesh-per-object scene gives back its objects and instances.
    np.testing.assert_array_equal(ref["instances"].view(np.uint8), w.scene.instances.view(np.uint8))
    np.testing.assert_array_equal(ref["work_items"], w.scene.work_items)
    built = S.Scene(ref["meshlets"], ref["objects"], ref["instances"], ref["work_items"], w.scene.aabbs,
                    w.scene.draw_calls, ref["max_draw_count"], w.scene.lod0_meshlets)
    vs = VgScene()
    vs.upload(b.frame_data())
    views = w.views[:2]
    depths = [torch.from_numpy(np.ascontiguousarray(v.depth)).cuda() for v in views]
    bc = BatchedCull(len(views), span_visibility=False)
    bc.prepare(vs, [{"camera": v.camera, "depth": d, "lod_threshold_px": v.lod_threshold_px}
                    for v, d in zip(views, depths)])
    bc.execute()
    torch.cuda.synchronize()
    bc.status()
    for i, v in enumerate(views):
        got = gather(bc, i, len(built.objects))
        check_view(built, v, got, None, None, got["capacity"])
