"""ctypes binding of ``include/helio_cull.h`` (the C-ABI of libhelio_cull.so).

The structures mirror the libhelio byte layouts; their sizes are asserted at import.
Loading fails loudly when the library is missing: there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_DIR = Path(__file__).resolve().parent / "lib"
CULL_LIB = LIB_DIR / "libhelio_cull.so"
SCENEGEN_LIB = LIB_DIR / "libhelio_scenegen.so"

u32, i32, u64, f32 = C.c_uint32, C.c_int32, C.c_uint64, C.c_float
vp = C.c_void_p

HELIO_OK = 0
HELIO_ERR_CUDA = 1
HELIO_ERR_INVALID_ARG = 2
HELIO_ERR_RESOURCE = 3
HELIO_ERR_CAPACITY = 4
HELIO_ERR_TIMEOUT = 5
HELIO_ERR_BUDGET = 6
HELIO_ERR_NOT_READY = 7
HELIO_MEM_HOST = 0
HELIO_MEM_DEVICE = 1
HELIO_VG_CLEAR_INDIRECT = 1
HELIO_HIZ_MAX_MIPS = 12
HELIO_HIZ_ALIAS_MIP0 = 1
HELIO_HIZ_NO_TMA = 2
HELIO_VG_COUNTER_COUNT = 11
HELIO_VG_DEFAULT_PUBLICATION_LIMIT = 262144
HELIO_LOD_LOW, HELIO_LOD_MEDIUM, HELIO_LOD_HIGH, HELIO_LOD_ULTRA = 0, 1, 2, 3


class GpuCameraUniforms(C.Structure):
    _fields_ = [("view", f32 * 16), ("proj", f32 * 16), ("view_proj", f32 * 16), ("inv_view_proj", f32 * 16),
                ("position_near", f32 * 4), ("forward_far", f32 * 4), ("jitter_frame", f32 * 4),
                ("prev_view_proj", f32 * 16)]


class GpuInstanceData(C.Structure):
    _fields_ = [("model", f32 * 16), ("normal_mat", f32 * 12), ("bounds", f32 * 4), ("mesh_id", u32),
                ("material_id", u32), ("flags", u32), ("lightmap_index", u32)]


class GpuInstanceAabb(C.Structure):
    _fields_ = [("min", f32 * 3), ("pad0", f32), ("max", f32 * 3), ("pad1", f32)]


class GpuDrawCall(C.Structure):
    _fields_ = [("index_count", u32), ("first_index", u32), ("vertex_offset", i32), ("first_instance", u32),
                ("instance_count", u32)]


class DrawIndexedIndirectArgs(C.Structure):
    _fields_ = [("index_count", u32), ("instance_count", u32), ("first_index", u32), ("base_vertex", i32),
                ("first_instance", u32)]


class GpuMeshletEntry(C.Structure):
    _fields_ = [("center", f32 * 3), ("radius", f32), ("cone_apex", f32 * 3), ("cone_cutoff", f32),
                ("cone_axis", f32 * 3), ("lod_error", f32), ("first_index", u32), ("index_count", u32),
                ("vertex_offset", i32), ("instance_index", u32)]


class GpuVgObject(C.Structure):
    _fields_ = [("instance_index", u32), ("lod_count", u32), ("max_meshlet_count", u32), ("reserved", u32),
                ("local_bounds", f32 * 4), ("lod_errors", f32 * 8), ("lod_first_meshlets", u32 * 8),
                ("lod_meshlet_counts", u32 * 8)]


class GpuVgDraw(C.Structure):
    _fields_ = [("instance_index", u32), ("meshlet_index", u32), ("lod_level", u32), ("reserved", u32)]


class GpuVgWorkItem(C.Structure):
    _fields_ = [("object_index", u32), ("local_meshlet_base", u32)]


class InstanceCullData(C.Structure):
    _fields_ = [("max_scale", f32), ("min_scale", f32), ("cone_cull_enabled", u32), ("valid_transform", u32)]


class KernelTiming(C.Structure):
    _fields_ = [("name", C.c_char * 40), ("launches", u64), ("total_ms", C.c_double)]


def profiler_collect() -> dict:
    """{kernel name: (launches, total device ms)} accumulated since the last reset."""
    lib = cull_lib()
    n = u32(0)
    check(lib.helio_profiler_collect(None, 0, C.byref(n)))
    arr = (KernelTiming * max(n.value, 1))()
    check(lib.helio_profiler_collect(C.cast(arr, vp), n.value, C.byref(n)))
    return {arr[i].name.decode(): (int(arr[i].launches), float(arr[i].total_ms)) for i in range(n.value)}


class HizConfig(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("flags", u32)]


class HizPyramid(C.Structure):
    _fields_ = [("mip_count", u32), ("width", u32 * 12), ("height", u32 * 12), ("pitch", u32 * 12),
                ("levels", vp * 12)]


class HizViewInput(C.Structure):
    _fields_ = [("depth", vp), ("width", u32), ("height", u32), ("pitch", u32), ("flags", u32)]


class SceneBuffers(C.Structure):
    _fields_ = [("camera", vp), ("instances", vp), ("instance_count", u32), ("draw_calls", vp),
                ("draw_count", u32), ("aabbs", vp), ("indirect", vp)]


class VgMeshRecord(C.Structure):
    """HelioVgMeshRecord: a library mesh whose descriptors are pool[first_meshlet, +meshlet_count)."""
    _fields_ = [("first_meshlet", u32), ("meshlet_count", u32), ("lod_count", u32), ("max_meshlet_count", u32),
                ("local_bounds", f32 * 4), ("lod_errors", f32 * 8), ("lod_first_meshlets", u32 * 8),
                ("lod_meshlet_counts", u32 * 8)]


class VgBuildInputs(C.Structure):
    _fields_ = [("pool", vp), ("meshes", vp), ("slot_mesh", vp), ("slot_instances", vp), ("pool_count", u32),
                ("mesh_count", u32), ("slot_count", u32), ("reserved0", u32)]


VG_NO_MESH = 0xFFFFFFFF


class StaticHiz(C.Structure):
    """helio_static_hiz: level 0 of a baked static Hi-Z grid (six direction layers along z)."""
    _fields_ = [("texels", vp), ("grid_resolution", u32 * 3), ("world_bounds_min", f32 * 3),
                ("world_bounds_max", f32 * 3)]


class ShadowCullInputs(C.Structure):
    _fields_ = [("shadow_matrices", vp), ("instances", vp), ("src_indirect", vp), ("face_dirty", vp),
                ("instance_count", u32), ("draw_count", u32), ("face_count", u32), ("reserved0", u32)]


class ShadowCullOutputs(C.Structure):
    _fields_ = [("face_indirect", vp), ("face_counts", vp), ("max_faces", u32), ("max_draws_per_face", u32)]


SHADOW_MAX_FACES = 256
SHADOW_MAX_DRAWS_PER_FACE = 4096


class VgFrameData(C.Structure):
    _fields_ = [("meshlets", vp), ("objects", vp), ("instances", vp), ("work_items", vp),
                ("meshlet_count", u32), ("object_count", u32), ("work_item_count", u32), ("max_draw_count", u32),
                ("buffer_version", u64), ("instance_version", u64), ("instance_dirty_start", u32),
                ("instance_dirty_count", u32), ("memory", u32), ("reserved0", u32)]


class VgConfig(C.Structure):
    _fields_ = [("width", u32), ("height", u32), ("lod_quality", u32), ("publication_limit", u32),
                ("counter_count", u32), ("flags", u32)]


class VgOutputs(C.Structure):
    _fields_ = [("indirect", vp), ("draws", vp), ("counters", vp), ("visibility", vp), ("objects", vp),
                ("capacity", u32), ("counter_count", u32), ("work_item_count", u32), ("object_count", u32)]


class VgSceneInfo(C.Structure):
    _fields_ = [("meshlet_count", u32), ("object_count", u32), ("lod0_meshlets", u64), ("max_spans", u64),
                ("device_bytes", u64)]


class BatchConfig(C.Structure):
    _fields_ = [("max_views", u32), ("flags", u32), ("max_spans", u64), ("max_ctas", u32), ("select_views", u32),
                ("cull_ctas", u32), ("reserved", u32)]


class BatchTuning(C.Structure):
    _fields_ = [("select_views", u32), ("ctas", u32), ("candidates", u32), ("cull_ctas", u32),
                ("best_ms", C.c_double), ("default_ms", C.c_double)]


class BatchView(C.Structure):
    _fields_ = [("camera", GpuCameraUniforms), ("depth", vp), ("depth_pitch", u32), ("width", u32), ("height", u32),
                ("lod_error_threshold_px", f32), ("draw_capacity", u32), ("flags", u32)]


class BatchViewOutputs(C.Structure):
    _fields_ = [("indirect", vp), ("draws", vp), ("counters", vp), ("lod", vp), ("capacity", u32),
                ("object_count", u32), ("pyramid", HizPyramid)]


class BatchSpanList(C.Structure):
    _fields_ = [("spans", vp), ("visibility", vp), ("view_span_start", vp), ("span_capacity", u32),
                ("view_count", u32)]


class ServeConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", u64), ("slots", u32), ("max_views", u32), ("ctas_per_slot", u32),
                ("max_requests_per_batch", u32), ("spans_per_view", u64)]


class ServeRequest(C.Structure):
    _fields_ = [("scene", u32), ("view_count", u32), ("views", C.POINTER(BatchView)), ("arrival_s", C.c_double),
                ("tag", u64)]


class ServeCompletion(C.Structure):
    _fields_ = [("request", u64), ("tag", u64), ("status", i32), ("batch_requests", u32), ("view_count", u32),
                ("reserved", u32), ("arrival_s", C.c_double), ("launch_s", C.c_double), ("done_s", C.c_double),
                ("batch_device_ms", C.c_double), ("device_start_ms", C.c_double), ("device_end_ms", C.c_double)]


class ServePending(C.Structure):
    _fields_ = [("scene", u32), ("view_count", u32)]


class ServeStats(C.Structure):
    _fields_ = [("pending", u32), ("running", u32), ("ctas_per_slot", u32), ("reserved", u32), ("batches", u64),
                ("bytes_in_use", u64), ("scene_bytes", u64)]


HELIO_BATCH_MAX_VIEWS = 128
HELIO_BATCH_SPAN_VISIBILITY = 1

_SIZES = {GpuCameraUniforms: 368, GpuInstanceData: 144, GpuInstanceAabb: 32, GpuDrawCall: 20,
          DrawIndexedIndirectArgs: 20, GpuMeshletEntry: 64, GpuVgObject: 128, GpuVgDraw: 16, GpuVgWorkItem: 8,
          InstanceCullData: 16, VgFrameData: 80, BatchConfig: 32, ServeConfig: 32, ServeRequest: 32,
          ServeCompletion: 80, ServeStats: 40}
for _t, _n in _SIZES.items():
    assert C.sizeof(_t) == _n, (_t.__name__, C.sizeof(_t), _n)


def np_dtype(struct_type) -> np.dtype:
    """numpy structured dtype with the byte layout of a ctypes structure."""
    return np.dtype(np.ctypeslib.as_ctypes_type(np.dtype(struct_type)))


# Every exported entry point with its signature: (restype, argtypes).
CULL_EXPORTS = {
    "helio_abi_version": (i32, []),
    "helio_last_error": (C.c_char_p, []),
    "helio_status_string": (C.c_char_p, [i32]),
    "helio_kernel_launch_count": (u64, []),
    "helio_profiler_enable": (i32, [i32]),
    "helio_profiler_collect": (i32, [vp, u32, C.POINTER(u32)]),
    "helio_profiler_reset": (None, []),
    "helio_mip_levels": (u32, [u32, u32]),
    "helio_extract_frustum_planes": (None, [vp, vp]),
    "helio_instance_cull_data": (i32, [vp, u32, vp, vp]),
    "helio_hiz_create": (i32, [C.POINTER(HizConfig), C.POINTER(vp)]),
    "helio_hiz_prepare": (i32, [vp, vp, u32, u64]),
    "helio_hiz_execute": (i32, [vp, vp]),
    "helio_hiz_resize": (i32, [vp, u32, u32]),
    "helio_hiz_publish": (i32, [vp, C.POINTER(HizPyramid)]),
    "helio_hiz_device_status": (i32, [vp, vp]),
    "helio_hiz_destroy": (None, [vp]),
    "helio_hiz_build_noalloc": (i32, [u32, C.POINTER(HizViewInput), vp, C.c_size_t, C.POINTER(HizPyramid), vp]),
    "helio_indirect_dispatch_create": (i32, [vp, C.POINTER(vp)]),
    "helio_indirect_dispatch_prepare": (i32, [vp, C.POINTER(GpuCameraUniforms), u32]),
    "helio_indirect_dispatch_execute": (i32, [vp, C.POINTER(SceneBuffers), vp]),
    "helio_indirect_dispatch_destroy": (None, [vp]),
    "helio_occlusion_cull_create": (i32, [u32, u32, vp, C.POINTER(vp)]),
    "helio_occlusion_cull_prepare": (i32, [vp, u32]),
    "helio_occlusion_cull_execute": (i32, [vp, C.POINTER(SceneBuffers), C.POINTER(HizPyramid), u64, vp]),
    "helio_occlusion_cull_resize": (i32, [vp, u32, u32]),
    "helio_occlusion_cull_destroy": (None, [vp]),
    "helio_instance_cull_fused_execute": (i32, [vp, vp, C.POINTER(SceneBuffers), C.POINTER(HizPyramid), u64, vp]),
    "helio_lod_max_error_pixels": (f32, [u32]),
    "helio_vg_create": (i32, [C.POINTER(VgConfig), C.POINTER(vp)]),
    "helio_vg_prepare": (i32, [vp, C.POINTER(VgFrameData), vp]),
    "helio_vg_execute": (i32, [vp, vp, C.POINTER(HizPyramid), vp]),
    "helio_vg_resize": (i32, [vp, u32, u32]),
    "helio_vg_set_lod_quality": (i32, [vp, u32]),
    "helio_vg_publish": (i32, [vp, C.POINTER(VgOutputs)]),
    "helio_vg_device_status": (i32, [vp, vp]),
    "helio_vg_destroy": (None, [vp]),
    "helio_vg_scene_create": (i32, [C.POINTER(vp)]),
    "helio_vg_scene_upload": (i32, [vp, C.POINTER(VgFrameData), vp]),
    "helio_vg_scene_info_get": (i32, [vp, C.POINTER(VgSceneInfo)]),
    "helio_vg_scene_destroy": (None, [vp]),
    "helio_batch_create": (i32, [C.POINTER(BatchConfig), C.POINTER(vp)]),
    "helio_batch_prepare": (i32, [vp, vp, u32, C.POINTER(BatchView), vp]),
    "helio_batch_set_cameras": (i32, [vp, u32, C.POINTER(GpuCameraUniforms), vp]),
    "helio_batch_set_cameras_device": (i32, [vp, u32, vp, vp]),
    "helio_batch_execute": (i32, [vp, vp]),
    "helio_batch_get_view_outputs": (i32, [vp, u32, C.POINTER(BatchViewOutputs)]),
    "helio_batch_get_spans": (i32, [vp, C.POINTER(BatchSpanList)]),
    "helio_batch_set_wait_limit": (i32, [vp, u32, u32]),
    "helio_batch_status": (i32, [vp, vp]),
    "helio_batch_get_phase_times": (i32, [vp, C.POINTER(C.c_double), u32, C.POINTER(u32), vp]),
    "helio_batch_estimate_bytes": (i32, [C.POINTER(BatchConfig), vp, u32, C.POINTER(BatchView), C.POINTER(u64)]),
    "helio_batch_device_bytes": (i32, [vp, C.POINTER(u64)]),
    "helio_batch_growth_bytes": (i32, [vp, C.POINTER(BatchConfig), vp, u32, C.POINTER(BatchView), C.POINTER(u64)]),
    "helio_batch_reconfigure": (i32, [vp, C.POINTER(BatchConfig)]),
    "helio_batch_autotune": (i32, [vp, u32, C.POINTER(BatchTuning), vp]),
    "helio_batch_pack_draws": (i32, [vp, vp, vp, vp, u64, vp]),
    "helio_batch_destroy": (None, [vp]),
    "helio_serve_create": (i32, [C.POINTER(ServeConfig), C.POINTER(vp)]),
    "helio_serve_add_scene": (i32, [vp, vp, C.POINTER(u32)]),
    "helio_serve_submit": (i32, [vp, C.POINTER(ServeRequest), C.POINTER(u64)]),
    "helio_serve_pump": (i32, [vp, C.c_double, C.POINTER(u32)]),
    "helio_serve_completions": (i32, [vp, C.POINTER(ServeCompletion), u32, C.POINTER(u32)]),
    "helio_serve_outputs": (i32, [vp, u64, u32, C.POINTER(BatchViewOutputs)]),
    "helio_serve_release": (i32, [vp, u64]),
    "helio_serve_stats_get": (i32, [vp, C.POINTER(ServeStats)]),
    "helio_serve_plan_batch": (i32, [C.POINTER(ServePending), u32, u32, u32, C.POINTER(u32), C.POINTER(u32)]),
    "helio_serve_destroy": (None, [vp]),
    "helio_occlusion_cull_set_static_hiz": (i32, [vp, C.POINTER(StaticHiz)]),
    "helio_vg_builder_create": (i32, [C.POINTER(vp)]),
    "helio_vg_builder_run": (i32, [vp, C.POINTER(VgBuildInputs), vp]),
    "helio_vg_builder_frame_data": (i32, [vp, C.POINTER(VgFrameData)]),
    "helio_vg_builder_destroy": (None, [vp]),
    "helio_shadow_cull_create": (i32, [C.POINTER(vp)]),
    "helio_shadow_cull_prepare": (i32, [vp, C.POINTER(ShadowCullInputs)]),
    "helio_shadow_cull_execute": (i32, [vp, vp]),
    "helio_shadow_cull_publish": (i32, [vp, C.POINTER(ShadowCullOutputs)]),
    "helio_shadow_cull_destroy": (None, [vp]),
    "helio_batch_attach_shadow": (i32, [vp, vp]),
}

_cull = None
_scenegen = None


class HelioError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"helio status {status}: {message}")
        self.status = status


def cull_lib() -> C.CDLL:
    """The CUDA library; raises if it was not built (no CPU fallback exists)."""
    global _cull
    if _cull is None:
        if not CULL_LIB.exists():
            raise FileNotFoundError(f"{CULL_LIB} missing: run `python -m helio_b200.build`")
        lib = C.CDLL(str(CULL_LIB))
        for name, (res, args) in CULL_EXPORTS.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _cull = lib
    return _cull


def check(status: int) -> None:
    if status != HELIO_OK:
        msg = cull_lib().helio_last_error()
        raise HelioError(status, msg.decode() if msg else "")


class SceneParams(C.Structure):
    _fields_ = [("seed", u64), ("instance_count", u32), ("lod0_meshlets", u32), ("lod_count", u32),
                ("placement", u32), ("cube_half", f32), ("blob_count", u32), ("blob_sigma", f32),
                ("lod_error_mode", u32), ("coverage_height_px", f32), ("coverage_tau_px", f32),
                ("mesh_library", u32), ("threads", u32), ("scale_min", f32), ("scale_max", f32)]


class SceneCounts(C.Structure):
    _fields_ = [("meshlets", u64), ("objects", u64), ("work_items", u64), ("max_draw_count", u64),
                ("mesh_count", u64), ("meshlets_per_mesh", u64)]


def scenegen_lib() -> C.CDLL:
    global _scenegen
    if _scenegen is None:
        if not SCENEGEN_LIB.exists():
            raise FileNotFoundError(f"{SCENEGEN_LIB} missing: run `python -m helio_b200.build`")
        lib = C.CDLL(str(SCENEGEN_LIB))
        lib.sg_scene_counts_fn.argtypes = [C.POINTER(SceneParams), C.POINTER(SceneCounts)]
        lib.sg_scene_counts_fn.restype = i32
        lib.sg_scene_generate.argtypes = [C.POINTER(SceneParams), vp, vp, vp, vp, vp, vp]
        lib.sg_scene_generate.restype = i32
        d3 = C.POINTER(C.c_double)
        lib.sg_camera_perspective.argtypes = [d3, d3, d3, C.c_double, C.c_double, C.c_double, C.c_double,
                                              C.POINTER(GpuCameraUniforms)]
        lib.sg_camera_perspective.restype = None
        lib.sg_camera_ortho.argtypes = [d3, d3, d3] + [C.c_double] * 6 + [C.POINTER(GpuCameraUniforms)]
        lib.sg_camera_ortho.restype = None
        lib.sg_depth.argtypes = [u64, u32, u32, u32, u32, f32, f32, f32, u32, vp, u32]
        lib.sg_depth.restype = i32
        _scenegen = lib
    return _scenegen
