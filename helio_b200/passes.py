"""Python mirror of the reference passes, over the C-ABI of libhelio_cull.so.

Each class follows the reference ``RenderPass`` lifecycle (crates/helio-core/src/
traits.rs:276-470): ``prepare`` → ``execute`` → ``publish``, with ``on_resize``.
Device memory and streams come from PyTorch (plumbing only); every kernel is in the
native library, and a missing library raises instead of falling back.

  HiZBuildPass           crates/helio-pass-hiz/src/lib.rs:381-548
  IndirectDispatchPass   crates/helio-pass-indirect-dispatch/src/lib.rs:164-258
  OcclusionCullPass      crates/helio-pass-occlusion-cull/src/lib.rs:279-411
  VirtualGeometryPass    crates/helio-pass-virtual-geometry/src/rendering.rs:703-1165 (cull half)
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import native as N

UINT64_MAX = (1 << 64) - 1


LOD_LEVEL_COUNT = 8
DEFAULT_MAX_PUBLISHED_MESHLETS = 262_144


class VirtualGeometryDebugStats:
    """Decoded VG counters (crates/helio-pass-virtual-geometry/src/lib.rs:30-67)."""

    def __init__(self, visible_meshlets, rejected_meshlets, lod_object_counts, max_available_lod):
        self.visible_meshlets = visible_meshlets
        self.rejected_meshlets = rejected_meshlets
        self.lod_object_counts = list(lod_object_counts)
        self.max_available_lod = max_available_lod

    @classmethod
    def from_counters(cls, counters):
        """None unless all 11 counters are present (the 2-counter layout has no histogram)."""
        c = [int(x) for x in counters]
        if len(c) < 11:
            return None
        return cls(c[0], c[1], c[2:10], min(c[10], LOD_LEVEL_COUNT - 1))

    def visible_objects(self) -> int:
        return sum(self.lod_object_counts)

    def selected_lod_range(self):
        nz = [i for i, n in enumerate(self.lod_object_counts) if n]
        return (nz[0], nz[-1]) if nz else None


class VirtualGeometryBudget:
    """Publication budget (crates/helio-pass-virtual-geometry/src/lib.rs:78-117): 36 bytes
    per published meshlet (20-byte indirect command + 16-byte GpuVgDraw) plus 11 counters."""

    def __init__(self, max_published_meshlets: int = DEFAULT_MAX_PUBLISHED_MESHLETS):
        if max_published_meshlets <= 0:
            raise ValueError("virtual geometry publication budget must be non-zero")
        self.max_published_meshlets = int(max_published_meshlets)

    def publication_bytes(self) -> int:
        return self.max_published_meshlets * 36 + 11 * 4

    def clamp_draw_count(self, worst_case: int) -> int:
        return min(int(worst_case), self.max_published_meshlets)


class _CudaArray:
    """Zero-copy __cuda_array_interface__ view of library-owned device memory."""

    def __init__(self, ptr: int, shape, typestr: str, strides=None):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2, "strides": strides}


def device_view(ptr: int, shape, dtype: str = "<i4", strides=None) -> torch.Tensor:
    """torch tensor aliasing `ptr` (int32 words by default)."""
    if not ptr:
        raise N.HelioError(N.HELIO_ERR_RESOURCE, "null device pointer")
    return torch.as_tensor(_CudaArray(ptr, shape, dtype, strides), device="cuda")


def _stream_ptr(stream) -> C.c_void_p:
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


def _ptr(t) -> C.c_void_p:
    if t is None:
        return C.c_void_p(0)
    if isinstance(t, torch.Tensor):
        return C.c_void_p(t.data_ptr())
    if isinstance(t, np.ndarray):
        return C.c_void_p(t.ctypes.data)
    return C.c_void_p(int(t))


def camera_bytes(cam: N.GpuCameraUniforms) -> np.ndarray:
    return np.frombuffer(bytes(cam), dtype=np.uint8).copy()


class HiZBuildPass:
    """Hi-Z pyramid (max reduction, standard Z) built by one fused launch."""

    def __init__(self, width: int, height: int, alias_mip0: bool = False, tma: bool = True):
        self._lib = N.cull_lib()
        flags = (N.HELIO_HIZ_ALIAS_MIP0 if alias_mip0 else 0) | (0 if tma else N.HELIO_HIZ_NO_TMA)
        cfg = N.HizConfig(width, height, flags)
        h = C.c_void_p()
        N.check(self._lib.helio_hiz_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.width, self.height = width, height
        self._depth = None

    def name(self) -> str:
        return "HiZBuild"

    def prepare(self, depth: torch.Tensor, camera_generation: int = UINT64_MAX) -> None:
        assert depth.is_cuda and depth.dtype == torch.float32 and depth.dim() == 2
        assert depth.stride(1) == 1 and depth.shape[0] == self.height and depth.shape[1] == self.width
        self._depth = depth  # keep alive while the pyramid may alias it
        N.check(self._lib.helio_hiz_prepare(self._h, _ptr(depth), depth.stride(0), camera_generation))

    def execute(self, stream=None) -> None:
        N.check(self._lib.helio_hiz_execute(self._h, _stream_ptr(stream)))

    def device_status(self, stream=None) -> None:
        """Raises if a bounded device wait of an earlier execute gave up (synchronises)."""
        N.check(self._lib.helio_hiz_device_status(self._h, _stream_ptr(stream)))

    def on_resize(self, width: int, height: int) -> None:
        N.check(self._lib.helio_hiz_resize(self._h, width, height))
        self.width, self.height = width, height

    def publish(self) -> N.HizPyramid:
        pyr = N.HizPyramid()
        N.check(self._lib.helio_hiz_publish(self._h, C.byref(pyr)))
        return pyr

    def level(self, l: int) -> torch.Tensor:
        pyr = self.publish()
        w, h, p = pyr.width[l], pyr.height[l], pyr.pitch[l]
        return device_view(pyr.levels[l], (h, w), "<f4", (p * 4, 4))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.helio_hiz_destroy(h)
            self._h = None


def scene_buffers(camera_dev, instances, draw_calls, aabbs, indirect) -> N.SceneBuffers:
    return N.SceneBuffers(_ptr(camera_dev), _ptr(instances), instances.shape[0] if instances is not None else 0,
                          _ptr(draw_calls), draw_calls.shape[0], _ptr(aabbs), _ptr(indirect))


class IndirectDispatchPass:
    """Per-draw frustum + sub-pixel cull writing DrawIndexedIndirect (non-compacting)."""

    def __init__(self, stats: torch.Tensor):
        self._lib = N.cull_lib()
        assert stats.is_cuda and stats.numel() >= 8
        self.stats = stats
        h = C.c_void_p()
        N.check(self._lib.helio_indirect_dispatch_create(_ptr(stats), C.byref(h)))
        self._h = h

    def name(self) -> str:
        return "IndirectDispatch"

    def prepare(self, camera: N.GpuCameraUniforms, draw_count: int) -> None:
        N.check(self._lib.helio_indirect_dispatch_prepare(self._h, C.byref(camera), draw_count))

    def execute(self, scene: N.SceneBuffers, stream=None) -> None:
        N.check(self._lib.helio_indirect_dispatch_execute(self._h, C.byref(scene), _stream_ptr(stream)))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.helio_indirect_dispatch_destroy(h)
            self._h = None


class OcclusionCullPass:
    """Per-draw Hi-Z occlusion test against the (previous frame's) pyramid."""

    def __init__(self, width: int, height: int, stats: torch.Tensor):
        self._lib = N.cull_lib()
        self.stats = stats
        h = C.c_void_p()
        N.check(self._lib.helio_occlusion_cull_create(width, height, _ptr(stats), C.byref(h)))
        self._h = h

    def name(self) -> str:
        return "OcclusionCull"

    def prepare(self, draw_count: int) -> None:
        N.check(self._lib.helio_occlusion_cull_prepare(self._h, draw_count))

    def execute(self, scene: N.SceneBuffers, hiz: N.HizPyramid, frame_num: int, stream=None) -> None:
        N.check(self._lib.helio_occlusion_cull_execute(self._h, C.byref(scene), C.byref(hiz), frame_num,
                                                       _stream_ptr(stream)))

    def on_resize(self, width: int, height: int) -> None:
        N.check(self._lib.helio_occlusion_cull_resize(self._h, width, height))

    def set_static_hiz(self, texels, grid=(0, 0, 0), bounds_min=(0.0, 0.0, 0.0), bounds_max=(0.0, 0.0, 0.0)) -> None:
        """Static Hi-Z for the following executes (texels: device float32 tensor of level
        0, grid[0] x grid[1] x grid[2] * 6, x fastest), or None to switch it off."""
        if texels is None:
            N.check(self._lib.helio_occlusion_cull_set_static_hiz(self._h, None))
            self._static = None
            return
        assert texels.is_cuda and texels.dtype == torch.float32 and texels.is_contiguous()
        assert texels.numel() == grid[0] * grid[1] * grid[2] * 6
        s = N.StaticHiz(texels.data_ptr(), (C.c_uint32 * 3)(*grid), (C.c_float * 3)(*bounds_min),
                        (C.c_float * 3)(*bounds_max))
        N.check(self._lib.helio_occlusion_cull_set_static_hiz(self._h, C.byref(s)))
        self._static = texels

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.helio_occlusion_cull_destroy(h)
            self._h = None


def fused_instance_cull(frustum: IndirectDispatchPass, occlusion: OcclusionCullPass, scene: N.SceneBuffers,
                        hiz: N.HizPyramid, frame_num: int, stream=None) -> None:
    lib = N.cull_lib()
    N.check(lib.helio_instance_cull_fused_execute(frustum._h, occlusion._h, C.byref(scene), C.byref(hiz), frame_num,
                                                  _stream_ptr(stream)))


class VgScene:
    """Device-resident virtual-geometry scene shared by batches (helio_vg_scene)."""

    def __init__(self):
        self._lib = N.cull_lib()
        h = C.c_void_p()
        N.check(self._lib.helio_vg_scene_create(C.byref(h)))
        self._h = h

    def upload(self, frame: N.VgFrameData, stream=None) -> None:
        N.check(self._lib.helio_vg_scene_upload(self._h, C.byref(frame), _stream_ptr(stream)))

    def info(self) -> N.VgSceneInfo:
        out = N.VgSceneInfo()
        N.check(self._lib.helio_vg_scene_info_get(self._h, C.byref(out)))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.helio_vg_scene_destroy(h)
            self._h = None


class ShadowCullPass:
    """Per-face shadow frustum cull (helio_shadow_cull_*; ShadowCullPass,
    crates/helio-pass-shadow-cull/src/lib.rs:57-328)."""

    def __init__(self):
        self._lib = N.cull_lib()
        h = C.c_void_p()
        N.check(self._lib.helio_shadow_cull_create(C.byref(h)))
        self._h = h

    def name(self) -> str:
        return "ShadowCull"

    def prepare(self, matrices: torch.Tensor, instances: torch.Tensor, src_indirect: torch.Tensor,
                face_dirty: torch.Tensor, face_count: int) -> None:
        """Device tensors: matrices float32 [256, 16], instances bytes (144 per instance),
        src_indirect int32 [n, 5], face_dirty int32 [256]."""
        for t in (matrices, instances, src_indirect, face_dirty):
            assert t.is_cuda and t.is_contiguous()
        assert matrices.numel() == 256 * 16 and face_dirty.numel() == 256
        self._keep = (matrices, instances, src_indirect, face_dirty)
        inp = N.ShadowCullInputs(_ptr(matrices), _ptr(instances), _ptr(src_indirect), _ptr(face_dirty),
                                 instances.numel() * instances.element_size() // C.sizeof(N.GpuInstanceData),
                                 src_indirect.numel() * src_indirect.element_size() // 20, face_count, 0)
        N.check(self._lib.helio_shadow_cull_prepare(self._h, C.byref(inp)))

    def execute(self, stream=None) -> None:
        N.check(self._lib.helio_shadow_cull_execute(self._h, _stream_ptr(stream)))

    def outputs(self) -> dict:
        o = N.ShadowCullOutputs()
        N.check(self._lib.helio_shadow_cull_publish(self._h, C.byref(o)))
        return {"face_indirect": device_view(o.face_indirect, (o.max_faces * o.max_draws_per_face, 5)),
                "face_counts": device_view(o.face_counts, (o.max_faces,))}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.helio_shadow_cull_destroy(h)
            self._h = None


class VgBuilder:
    """The VG input producer (helio_vg_builder): rebuild_vg_buffers on the device, from a
    descriptor pool, mesh records and dense object slots held in device memory
    (crates/helio/src/scene/virtual_geometry/rebuild.rs:98-172)."""

    def __init__(self):
        self._lib = N.cull_lib()
        h = C.c_void_p()
        N.check(self._lib.helio_vg_builder_create(C.byref(h)))
        self._h = h

    def run(self, pool: torch.Tensor, meshes: torch.Tensor, slot_mesh: torch.Tensor, slot_instances: torch.Tensor,
            stream=None) -> N.VgFrameData:
        """Byte tensors on the device (64 B per descriptor, 128 B per mesh record, u32 per
        slot, 144 B per slot instance). Returns the outputs as device frame data."""
        for t in (pool, meshes, slot_mesh, slot_instances):
            assert t.is_cuda and t.is_contiguous()
        inp = N.VgBuildInputs(_ptr(pool), _ptr(meshes), _ptr(slot_mesh), _ptr(slot_instances),
                              pool.numel() * pool.element_size() // C.sizeof(N.GpuMeshletEntry),
                              meshes.numel() * meshes.element_size() // C.sizeof(N.VgMeshRecord),
                              slot_mesh.numel() * slot_mesh.element_size() // 4, 0)
        assert slot_instances.numel() * slot_instances.element_size() == inp.slot_count * C.sizeof(N.GpuInstanceData)
        N.check(self._lib.helio_vg_builder_run(self._h, C.byref(inp), _stream_ptr(stream)))
        return self.frame_data()

    def frame_data(self) -> N.VgFrameData:
        out = N.VgFrameData()
        N.check(self._lib.helio_vg_builder_frame_data(self._h, C.byref(out)))
        return out

    def outputs(self) -> dict:
        """The last run's arrays as device byte tensors (aliasing the builder's buffers)."""
        f = self.frame_data()

        def view(ptr, n, size):
            return device_view(ptr, (max(n, 1) * size,), "|u1")[: n * size] if n else torch.empty(0, dtype=torch.uint8)

        return {"meshlets": view(f.meshlets, f.meshlet_count, C.sizeof(N.GpuMeshletEntry)),
                "objects": view(f.objects, f.object_count, C.sizeof(N.GpuVgObject)),
                "instances": view(f.instances, f.object_count, C.sizeof(N.GpuInstanceData)),
                "work_items": view(f.work_items, f.work_item_count, C.sizeof(N.GpuVgWorkItem)),
                "max_draw_count": f.max_draw_count}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.helio_vg_builder_destroy(h)
            self._h = None


def batch_views(views: list):
    """helio_batch_view array of view dicts (camera, device depth H x W float32, optional
    lod_threshold_px, draw_capacity, alias_mip0)."""
    arr = (N.BatchView * len(views))()
    for i, v in enumerate(views):
        d = v["depth"]
        assert d.is_cuda and d.dtype == torch.float32 and d.stride(1) == 1
        arr[i].camera = v["camera"]
        arr[i].depth = d.data_ptr()
        arr[i].depth_pitch = d.stride(0)
        arr[i].height, arr[i].width = d.shape
        arr[i].lod_error_threshold_px = v.get("lod_threshold_px", 0.0)
        arr[i].draw_capacity = v.get("draw_capacity", 0)
        arr[i].flags = N.HELIO_HIZ_ALIAS_MIP0 if v.get("alias_mip0", False) else 0
    return arr


def _batch_outputs(o: N.BatchViewOutputs) -> dict:
    cap = max(o.capacity, 1)
    return {"indirect": device_view(o.indirect, (cap, 5)), "draws": device_view(o.draws, (cap, 4)),
            "counters": device_view(o.counters, (11,)), "lod": device_view(o.lod, (max(o.object_count, 1),), "|u1"),
            "capacity": o.capacity, "pyramid": o.pyramid}


class BatchedCull:
    """Every view of a batch culled against one VgScene in one cooperative launch
    (Hi-Z of each view, object LOD select for every (object, view), meshlet cull and
    per-view deterministic compaction)."""

    def __init__(self, max_views: int = N.HELIO_BATCH_MAX_VIEWS, span_visibility: bool = False, max_spans: int = 0,
                 max_ctas: int = 0, cull_ctas: int = 0):
        self._lib = N.cull_lib()
        cfg = N.BatchConfig(max_views, N.HELIO_BATCH_SPAN_VISIBILITY if span_visibility else 0, max_spans, max_ctas,
                            0, cull_ctas)
        h = C.c_void_p()
        N.check(self._lib.helio_batch_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._keep = None
        self.view_count = 0

    def prepare(self, scene: VgScene, views: list, stream=None) -> None:
        """views: sequence of dicts with camera (GpuCameraUniforms), depth (device
        float32 tensor H x W), optional lod_threshold_px, draw_capacity, alias_mip0."""
        arr = batch_views(views)
        self._keep = (scene, [v["depth"] for v in views])
        N.check(self._lib.helio_batch_prepare(self._h, scene._h, len(views), arr, _stream_ptr(stream)))
        self.view_count = len(views)

    def pack_draws(self, indirect, draws, offsets, stream=None) -> None:
        """Every view's published draws into one pair of device tensors (int32 [cap, 5]
        and [cap, 4]), view after view; offsets (int32 [views + 1]) receives the view starts."""
        N.check(self._lib.helio_batch_pack_draws(self._h, indirect.data_ptr(), draws.data_ptr(), offsets.data_ptr(),
                                                 indirect.shape[0], _stream_ptr(stream)))

    def autotune(self, repeats: int = 3, stream=None) -> dict:
        """Times the prepared batch under every launch-shape candidate (views per
        select unit x CTAs per SM of the first launch, then CTAs per SM of the
        meshlet-test launch) and keeps the fastest (helio_batch_autotune)."""
        t = N.BatchTuning()
        N.check(self._lib.helio_batch_autotune(self._h, repeats, C.byref(t), _stream_ptr(stream)))
        return {"select_views": t.select_views, "ctas": t.ctas, "cull_ctas": t.cull_ctas,
                "candidates": t.candidates, "best_ms": t.best_ms, "default_ms": t.default_ms}

    def set_cameras_device(self, cameras: torch.Tensor, stream=None) -> None:
        """Cameras from a device tensor of view_count x 368 bytes (stream-ordered)."""
        assert cameras.is_cuda and cameras.numel() * cameras.element_size() >= 368 * self.view_count
        N.check(self._lib.helio_batch_set_cameras_device(self._h, self.view_count, cameras.data_ptr(),
                                                         _stream_ptr(stream)))

    def set_cameras(self, cameras: list, stream=None) -> None:
        arr = (N.GpuCameraUniforms * len(cameras))(*cameras)
        N.check(self._lib.helio_batch_set_cameras(self._h, len(cameras), arr, _stream_ptr(stream)))

    def attach_shadow(self, shadow: "ShadowCullPass | None") -> None:
        """Runs a prepared ShadowCullPass inside this batch's launches from the next
        execute on (helio_batch_attach_shadow); its outputs stay the pass's. None detaches."""
        N.check(self._lib.helio_batch_attach_shadow(self._h, shadow._h if shadow is not None else None))
        self._shadow = shadow  # kept alive while attached

    def execute(self, stream=None) -> None:
        N.check(self._lib.helio_batch_execute(self._h, _stream_ptr(stream)))

    def status(self, stream=None) -> None:
        N.check(self._lib.helio_batch_status(self._h, _stream_ptr(stream)))

    def set_wait_limit(self, max_polls: int = 0, extra_arrivals: int = 0) -> None:
        """Bounds of the device waits (0 = default, about 1 s); extra_arrivals > 0 makes
        every grid barrier wait for CTAs that never arrive (tests of the bounded waits)."""
        N.check(self._lib.helio_batch_set_wait_limit(self._h, max_polls, extra_arrivals))

    PHASES = ("view_setup", "hiz_and_select", "span_count_scan", "span_expand", "meshlet_test",
              "group_count_scan", "emit", "max_cta_hiz_busy", "max_cta_select_busy")

    def phase_times(self, stream=None) -> dict:
        """Device microseconds of each phase of the last execute, then the largest
        per-CTA busy time on Hi-Z tiles and on object chunks within phase 1. view_setup is
        CTA 0's part of the view setup (the other CTAs start on Hi-Z tiles meanwhile), and
        hiz_and_select runs from there to the end of phase 1."""
        arr = (C.c_double * 9)()
        n = N.u32(0)
        N.check(self._lib.helio_batch_get_phase_times(self._h, arr, 9, C.byref(n), _stream_ptr(stream)))
        return {name: arr[i] for i, name in enumerate(self.PHASES[: n.value])}

    def view_outputs(self, v: int) -> dict:
        o = N.BatchViewOutputs()
        N.check(self._lib.helio_batch_get_view_outputs(self._h, v, C.byref(o)))
        return _batch_outputs(o)

    def spans(self) -> dict:
        s = N.BatchSpanList()
        N.check(self._lib.helio_batch_get_spans(self._h, C.byref(s)))
        out = {"spans": device_view(s.spans, (s.span_capacity, 4)),
               "view_span_start": device_view(s.view_span_start, (s.view_count + 1,))}
        if s.visibility:
            out["visibility"] = device_view(s.visibility, (s.span_capacity, 2))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.helio_batch_destroy(h)
            self._h = None


class ServeLoop:
    """Continuous batching of cull requests over device-resident scenes (helio_serve):
    submit requests as they arrive, pump with the current time, read completions and
    their outputs, release them. Times are seconds on the caller's clock."""

    def __init__(self, hbm_budget_bytes: int = 0, slots: int = 4, max_views: int = N.HELIO_BATCH_MAX_VIEWS,
                 ctas_per_slot: int = 0, max_requests_per_batch: int = 0, spans_per_view: int = 0):
        self._lib = N.cull_lib()
        cfg = N.ServeConfig(hbm_budget_bytes, slots, max_views, ctas_per_slot, max_requests_per_batch, spans_per_view)
        h = C.c_void_p()
        N.check(self._lib.helio_serve_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._scenes = []
        self._depths = {}  # request -> depth tensors kept alive until completion

    def add_scene(self, scene: VgScene) -> int:
        sid = N.u32(0)
        N.check(self._lib.helio_serve_add_scene(self._h, scene._h, C.byref(sid)))
        self._scenes.append(scene)
        return sid.value

    def submit(self, scene_id: int, views: list, arrival_s: float, tag: int = 0) -> int:
        arr = batch_views(views)
        rq = N.ServeRequest(scene_id, len(views), arr, arrival_s, tag)
        rid = N.u64(0)
        N.check(self._lib.helio_serve_submit(self._h, C.byref(rq), C.byref(rid)))
        self._depths[rid.value] = [v["depth"] for v in views]
        return rid.value

    def pump(self, now_s: float) -> int:
        ready = N.u32(0)
        N.check(self._lib.helio_serve_pump(self._h, now_s, C.byref(ready)))
        return ready.value

    def completions(self, capacity: int = 256) -> list:
        arr = (N.ServeCompletion * capacity)()
        n = N.u32(0)
        N.check(self._lib.helio_serve_completions(self._h, arr, capacity, C.byref(n)))
        return [{f: getattr(arr[i], f) for f, _ in N.ServeCompletion._fields_ if f != "reserved"}
                for i in range(n.value)]

    def outputs(self, request: int, view: int) -> dict:
        o = N.BatchViewOutputs()
        N.check(self._lib.helio_serve_outputs(self._h, request, view, C.byref(o)))
        return _batch_outputs(o)

    def release(self, request: int) -> None:
        N.check(self._lib.helio_serve_release(self._h, request))
        self._depths.pop(request, None)

    def stats(self) -> dict:
        s = N.ServeStats()
        N.check(self._lib.helio_serve_stats_get(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in N.ServeStats._fields_ if f != "reserved"}

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.helio_serve_destroy(h)
            self._h = None


def plan_batch(queue: list, max_views: int, max_requests: int = 0) -> list:
    """The server's batch rule (helio_serve_plan_batch) on a queue of (scene, view_count)."""
    lib = N.cull_lib()
    arr = (N.ServePending * max(1, len(queue)))(*[N.ServePending(s, v) for s, v in queue])
    chosen = (N.u32 * max(1, len(queue)))()
    n = N.u32(0)
    N.check(lib.helio_serve_plan_batch(arr, len(queue), max_views, max_requests, chosen, C.byref(n)))
    return [chosen[i] for i in range(n.value)]


class VirtualGeometryPass:
    """Virtual-geometry cull: object LOD select + meshlet cull + deterministic compaction."""

    def __init__(self, width: int, height: int, lod_quality: int = N.HELIO_LOD_MEDIUM, publication_limit: int = 0,
                 counter_count: int = 11, clear_indirect: bool = False):
        self._lib = N.cull_lib()
        cfg = N.VgConfig(width, height, lod_quality, publication_limit, counter_count,
                         N.HELIO_VG_CLEAR_INDIRECT if clear_indirect else 0)
        h = C.c_void_p()
        N.check(self._lib.helio_vg_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.width, self.height = width, height

    def name(self) -> str:
        return "VirtualGeometry"

    def prepare(self, frame: N.VgFrameData, stream=None) -> None:
        N.check(self._lib.helio_vg_prepare(self._h, C.byref(frame), _stream_ptr(stream)))

    def execute(self, camera_dev: torch.Tensor, hiz: N.HizPyramid, stream=None) -> None:
        N.check(self._lib.helio_vg_execute(self._h, _ptr(camera_dev), C.byref(hiz), _stream_ptr(stream)))

    def on_resize(self, width: int, height: int) -> None:
        N.check(self._lib.helio_vg_resize(self._h, width, height))
        self.width, self.height = width, height

    def set_lod_quality(self, q: int) -> None:
        N.check(self._lib.helio_vg_set_lod_quality(self._h, q))

    def publish(self) -> N.VgOutputs:
        out = N.VgOutputs()
        N.check(self._lib.helio_vg_publish(self._h, C.byref(out)))
        return out

    def device_status(self, stream=None) -> None:
        N.check(self._lib.helio_vg_device_status(self._h, _stream_ptr(stream)))

    def outputs(self) -> dict:
        """Zero-copy torch views of the published buffers (int32 words)."""
        o = self.publish()
        cap = max(o.capacity, 1)
        return {
            "indirect": device_view(o.indirect, (cap, 5)),
            "draws": device_view(o.draws, (cap, 4)),
            "counters": device_view(o.counters, (o.counter_count,)),
            "visibility": device_view(o.visibility, (max(o.work_item_count, 1), 2)),
            "objects": device_view(o.objects, (max(o.object_count, 1), 32)),
            "capacity": o.capacity,
        }

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.helio_vg_destroy(h)
            self._h = None
