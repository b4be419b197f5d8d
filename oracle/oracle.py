"""ctypes front-end of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline / reference arm, to compare the CUDA path with. The product package never
imports it.

Besides the raw restatements, ``run_view`` runs the whole single-view pipeline of the
reference (Hi-Z build → object select → meshlet cull with canonical compaction) on
numpy arrays and returns every output, so tests compare the CUDA path field by field.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SRC = HERE / "oracle.cpp"
LIB = HERE / "_build" / "liboracle.so"

u32, f32, vp = C.c_uint32, C.c_float, C.c_void_p


class OracleStats(C.Structure):
    _fields_ = [("objects_tested", C.c_uint64), ("objects_visible", C.c_uint64), ("meshlets_tested", C.c_uint64),
                ("meshlets_cone_loaded", C.c_uint64), ("meshlets_visible", C.c_uint64),
                ("marginal_decisions", C.c_uint64), ("marginal_meshlets", C.c_uint64),
                ("marginal_objects", C.c_uint64)]


class OracleVgUniforms(C.Structure):
    _fields_ = [("object_count", u32), ("screen_width", u32), ("screen_height", u32), ("hiz_mip_count", u32),
                ("draw_capacity", u32), ("lod_error_threshold_px", f32), ("work_item_count", u32),
                ("meshlet_count", u32), ("instance_count", u32), ("counter_count", u32)]


class Pyramid(C.Structure):  # helio_hiz_pyramid
    _fields_ = [("mip_count", u32), ("width", u32 * 12), ("height", u32 * 12), ("pitch", u32 * 12),
                ("levels", vp * 12)]


def build() -> Path:
    LIB.parent.mkdir(exist_ok=True)
    if not LIB.exists() or LIB.stat().st_mtime < max(SRC.stat().st_mtime, (HERE / "oracle.h").stat().st_mtime):
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                        "-pthread", str(SRC), "-o", str(LIB)], check=True)
    return LIB


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        L.oracle_mip_levels.argtypes = [u32, u32]
        L.oracle_mip_levels.restype = u32
        L.oracle_ceil_log2.argtypes = [f32]
        L.oracle_ceil_log2.restype = u32
        L.oracle_extract_frustum_planes.argtypes = [vp, vp]
        L.oracle_extract_frustum_planes.restype = None
        L.oracle_instance_cull_data.argtypes = [vp, u32, vp]
        L.oracle_instance_cull_data.restype = None
        L.oracle_hiz_build.argtypes = [vp, u32, u32, u32, vp]
        L.oracle_hiz_build.restype = u32
        L.oracle_indirect_dispatch.argtypes = [vp, vp, vp, vp, vp, u32, u32, vp, vp]
        L.oracle_indirect_dispatch.restype = None
        L.oracle_occlusion_cull.argtypes = [vp, u32, u32, C.POINTER(Pyramid), vp, vp, u32, u32, vp, vp,
                                            C.POINTER(OracleStats)]
        L.oracle_occlusion_cull.restype = None
        L.oracle_occlusion_cull_static.argtypes = [vp, u32, u32, C.POINTER(Pyramid), vp, vp, u32, u32, vp, vp,
                                                   C.POINTER(OracleStats), vp]
        L.oracle_occlusion_cull_static.restype = None
        L.oracle_vg_select.argtypes = [vp, C.POINTER(OracleVgUniforms), vp, vp, vp, vp, vp, C.POINTER(OracleStats),
                                       C.c_int]
        L.oracle_vg_select.restype = None
        L.oracle_vg_cull.argtypes = [vp, C.POINTER(OracleVgUniforms), vp, vp, vp, vp, vp, vp, C.POINTER(Pyramid), vp,
                                     vp, vp, vp, C.POINTER(OracleStats), C.c_int]
        L.oracle_vg_cull.restype = None
        fp = C.POINTER(C.c_float)
        L.oracle_sphere_visible.argtypes = [fp, fp, f32]
        L.oracle_sphere_visible.restype = C.c_int
        L.oracle_select_lod.argtypes = [fp, u32, f32, f32, f32, f32]
        L.oracle_select_lod.restype = u32
        L.oracle_cone_reject.argtypes = [fp, fp, fp, f32]
        L.oracle_cone_reject.restype = C.c_int
        L.oracle_hiz_occludes.argtypes = [f32, f32]
        L.oracle_hiz_occludes.restype = C.c_int
        L.oracle_vg_rebuild.argtypes = [vp, u32, vp, u32, vp, vp, u32, vp, vp, vp, vp, C.POINTER(C.c_uint64)]
        L.oracle_vg_rebuild.restype = C.c_int
        L.oracle_shadow_cull.argtypes = [vp, vp, u32, vp, u32, vp, u32, u32, vp, vp]
        L.oracle_shadow_cull.restype = C.c_int
        _lib = L
    return _lib


def _fa(values) -> C.Array:
    values = [float(v) for v in values]
    return (C.c_float * len(values))(*values)


def sphere_visible(planes, center, radius) -> bool:
    flat = [x for p in planes for x in p]
    return bool(lib().oracle_sphere_visible(_fa(flat), _fa(center), radius))


def select_lod(errors, lod_count, max_scale, focal, closest, max_error) -> int:
    return int(lib().oracle_select_lod(_fa(list(errors) + [0.0] * (8 - len(errors))), lod_count, max_scale, focal,
                                       closest, max_error))


def cone_reject(camera, apex, axis, cutoff) -> bool:
    return bool(lib().oracle_cone_reject(_fa(camera), _fa(apex), _fa(axis), cutoff))


def hiz_occludes(near_z, hiz) -> bool:
    return bool(lib().oracle_hiz_occludes(near_z, hiz))


def _p(a) -> int:
    return a.ctypes.data if a is not None else 0


def mip_levels(w: int, h: int) -> int:
    return lib().oracle_mip_levels(w, h)


def hiz_build(depth: np.ndarray) -> list:
    """All pyramid levels (dense float32 arrays) of `depth` (H x W, any row pitch)."""
    depth = np.ascontiguousarray(depth, np.float32)
    h, w = depth.shape
    mips = min(mip_levels(w, h), 12)
    levels = [np.empty((max(h >> l, 1), max(w >> l, 1)), np.float32) for l in range(mips)]
    ptrs = (vp * 12)(*[lv.ctypes.data for lv in levels])
    lib().oracle_hiz_build(depth.ctypes.data, w, h, w, ptrs)
    return levels


def pyramid(levels: list) -> Pyramid:
    p = Pyramid()
    p.mip_count = len(levels)
    for l, lv in enumerate(levels):
        p.height[l], p.width[l] = lv.shape
        p.pitch[l] = lv.shape[1]
        p.levels[l] = lv.ctypes.data
    return p


def extract_frustum_planes(view_proj) -> np.ndarray:
    vp16 = np.ascontiguousarray(np.asarray(view_proj, np.float32).reshape(16))
    out = np.empty(24, np.float32)
    lib().oracle_extract_frustum_planes(vp16.ctypes.data, out.ctypes.data)
    return out


def instance_cull_data(instances: np.ndarray, dtype) -> np.ndarray:
    out = np.zeros(len(instances), dtype)
    lib().oracle_instance_cull_data(_p(instances), len(instances), _p(out))
    return out


def camera_array(cam) -> np.ndarray:
    return np.frombuffer(bytes(cam), np.uint8).copy()


def indirect_dispatch(cam, instances, draw_calls, aabbs):
    cam_b = camera_array(cam)
    planes = extract_frustum_planes(np.frombuffer(bytes(cam), np.float32)[32:48])
    indirect = np.zeros((len(draw_calls), 5), np.uint32)
    stats = np.zeros(8, np.uint32)
    lib().oracle_indirect_dispatch(_p(cam_b), _p(planes), _p(instances), _p(draw_calls), _p(aabbs), len(draw_calls),
                                   len(instances), _p(indirect), _p(stats))
    return indirect, stats


def occlusion_cull(cam, screen_w, screen_h, levels, instances, draw_calls, indirect, stats, static_hiz=None):
    """In place on `indirect` / `stats` (as the reference pass). static_hiz: None, or a
    dict of level-0 texels (float32, x fastest), grid (3 ints), min and max (3 floats)."""
    from helio_b200 import native as N

    cam_b = camera_array(cam)
    pyr = pyramid(levels)
    st = OracleStats()
    sh = None
    if static_hiz is not None:
        tex = np.ascontiguousarray(static_hiz["texels"], dtype=np.float32)
        sh = N.StaticHiz(tex.ctypes.data, (C.c_uint32 * 3)(*static_hiz["grid"]), (C.c_float * 3)(*static_hiz["min"]),
                         (C.c_float * 3)(*static_hiz["max"]))
    lib().oracle_occlusion_cull_static(_p(cam_b), screen_w, screen_h, C.byref(pyr), _p(instances), _p(draw_calls),
                                       len(draw_calls), len(instances), _p(indirect), _p(stats), C.byref(st),
                                       C.byref(sh) if sh is not None else None)
    return st


def run_view(scene, cam, width: int, height: int, levels: list, lod_threshold: float = 2.0, capacity: int | None = None,
             counter_count: int = 11, threads: int = 1, cull_dtype=None, work_items=None) -> dict:
    """Select + cull of one view over a scene (numpy structured arrays)."""
    L = lib()
    cam_b = camera_array(cam)
    O = len(scene.objects)
    items = scene.work_items if work_items is None else work_items
    W = len(items)
    cull = instance_cull_data(scene.instances, cull_dtype)
    cap = min(scene.max_draw_count, 262144) if capacity is None else capacity
    u = OracleVgUniforms(O, width, height, mip_levels(width, height), cap, lod_threshold, W, len(scene.meshlets), O,
                         counter_count)
    selected = np.zeros(O, np.uint32)
    counters = np.zeros(max(counter_count, 2), np.uint32)
    st = OracleStats()
    L.oracle_vg_select(_p(cam_b), C.byref(u), _p(scene.objects), _p(scene.instances), _p(cull), _p(selected),
                       _p(counters), C.byref(st), threads)
    indirect = np.zeros((max(cap, 1), 5), np.uint32)
    draws = np.zeros((max(cap, 1), 4), np.uint32)
    vis = np.zeros((max(W, 1), 2), np.uint32)
    pyr = pyramid(levels)
    L.oracle_vg_cull(_p(cam_b), C.byref(u), _p(scene.meshlets), _p(scene.objects), _p(selected), _p(scene.instances),
                     _p(cull), _p(items), C.byref(pyr), _p(indirect), _p(draws), _p(counters), _p(vis), C.byref(st),
                     threads)
    n = int(min(counters[0], cap))
    return {"selected": selected, "counters": counters, "indirect": indirect[:n], "draws": draws[:n],
            "visibility": vis[:W], "stats": st, "cull": cull}


def vg_rebuild(pool: np.ndarray, meshes: np.ndarray, slot_mesh: np.ndarray, slot_instances: np.ndarray):
    """rebuild_vg_buffers over a mesh library (numpy arrays of GpuMeshletEntry, VgMeshRecord,
    u32 and GpuInstanceData). Returns a dict of the output arrays and max_draw_count, or None
    where the reference panics."""
    from helio_b200 import native as N

    L = lib()
    pool, meshes = np.ascontiguousarray(pool), np.ascontiguousarray(meshes)
    slot_mesh = np.ascontiguousarray(slot_mesh, dtype=np.uint32)
    slot_instances = np.ascontiguousarray(slot_instances)
    counts = (C.c_uint64 * 4)()
    args = (pool.ctypes.data, len(pool), meshes.ctypes.data, len(meshes), slot_mesh.ctypes.data,
            slot_instances.ctypes.data, len(slot_mesh))
    if L.oracle_vg_rebuild(*args, None, None, None, None, counts):
        return None
    out = {"meshlets": np.zeros(counts[0], N.np_dtype(N.GpuMeshletEntry)),
           "objects": np.zeros(counts[1], N.np_dtype(N.GpuVgObject)),
           "instances": np.zeros(counts[1], N.np_dtype(N.GpuInstanceData)),
           "work_items": np.zeros(counts[2], N.np_dtype(N.GpuVgWorkItem))}
    rc = L.oracle_vg_rebuild(*args, out["meshlets"].ctypes.data, out["objects"].ctypes.data,
                             out["instances"].ctypes.data, out["work_items"].ctypes.data, counts)
    assert rc == 0
    out["max_draw_count"] = int(counts[3])
    return out


def shadow_cull(matrices: np.ndarray, instances: np.ndarray, src: np.ndarray, face_dirty: np.ndarray,
                face_count: int, max_per_face: int = 4096, dst=None, counts=None):
    """ShadowCullPass over 256 faces (matrices float32 [256, 16] column-major, src
    uint32 [n, 5] DrawIndexedIndirect, face_dirty uint32 [256]). dst / counts carry the
    previous frame (the pass keeps them when it returns early). Returns (dst [256 *
    max_per_face, 5], counts [256], ran)."""
    L = lib()
    matrices = np.ascontiguousarray(matrices, dtype=np.float32)
    src = np.ascontiguousarray(src, dtype=np.uint32).reshape(-1, 5)
    face_dirty = np.ascontiguousarray(face_dirty, dtype=np.uint32)
    instances = np.ascontiguousarray(instances)
    dst = np.zeros((256 * max_per_face, 5), np.uint32) if dst is None else dst.copy()
    counts = np.zeros(256, np.uint32) if counts is None else counts.copy()
    ran = L.oracle_shadow_cull(matrices.ctypes.data, instances.ctypes.data, len(instances), src.ctypes.data,
                               len(src), face_dirty.ctypes.data, face_count, max_per_face, dst.ctypes.data,
                               counts.ctypes.data)
    return dst, counts, bool(ran)
