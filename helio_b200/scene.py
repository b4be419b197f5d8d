"""Seeded synthetic workloads of the visibility path (numpy arrays in libhelio layouts).

Scenes, cameras and depth come from libhelio_scenegen.so (deterministic for a given
seed, independent of the thread count). The workloads:

  0  plain single view: 4,096 instances x 64 LOD0 meshlets (LOD k = ceil(64 / 2^k), 4 levels),
     200 m cube, LOD errors from coverage thresholds 0.25/0.06/0.015; 1024x1024 depth,
     256 occluder rectangles, perspective fov 60 deg, aspect 1, near 0.1, far 1000.
  1  10,000 x 100 meshlets (1M), LOD errors log-uniform in [1e-4, 1e-1]; 1920x1080, 2,000 rectangles.
  2  100,000 x 100 (10M), 64 Gaussian blobs (sigma 20 m) in a 2 km cube; 3840x2160, 20,000 rectangles.
  3  200,000 x 50 (10M), distributions of 2; 85 views (1 main 3840x2160, 4 orthographic cascades
     2048^2, 16 spot 512^2, 64 probe 128^2), occluder count proportional to pixel count.
  4  8 scenes, instance counts log-uniform in [10k, 2M] x 100 meshlets sharing a library of
     4,096 meshes per scene; requests carry 1..85 views of the configuration-3 mix.

Occluder rectangles: side ~ U[W/64, W/4] scaled so every view keeps configuration 0's
expected coverage; linear depth t ~ U[0, 1] of the near..far range stored as NDC depth.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field

import numpy as np

from . import native as N

SEED_BASE = 0x48454C494F00
DT_MESHLET = np.dtype(N.GpuMeshletEntry)
DT_OBJECT = np.dtype(N.GpuVgObject)
DT_INSTANCE = np.dtype(N.GpuInstanceData)
DT_ITEM = np.dtype(N.GpuVgWorkItem)
DT_AABB = np.dtype(N.GpuInstanceAabb)
DT_DRAWCALL = np.dtype(N.GpuDrawCall)


@dataclass
class Scene:
    meshlets: np.ndarray
    objects: np.ndarray
    instances: np.ndarray
    work_items: np.ndarray
    aabbs: np.ndarray
    draw_calls: np.ndarray
    max_draw_count: int
    lod0_meshlets: int  # LOD0 meshlets per instance (unit of the meshlets/s metric)

    @property
    def lod0_total(self) -> int:
        return self.lod0_meshlets * len(self.objects)

    def device_bytes(self) -> int:
        return (self.meshlets.nbytes + self.objects.nbytes + self.instances.nbytes + self.work_items.nbytes
                + len(self.objects) * 16 + len(self.objects) * 16 + self.work_items.nbytes)


@dataclass
class View:
    camera: N.GpuCameraUniforms
    width: int
    height: int
    depth: np.ndarray  # (height, width) float32
    kind: str = "perspective"
    lod_threshold_px: float = 2.0


@dataclass
class Workload:
    config_id: int
    scene: Scene
    views: list = field(default_factory=list)


def _threads() -> int:
    return max(1, min(32, os.cpu_count() or 1))


def make_scene(seed: int, instances: int, lod0: int, lod_count: int = 4, placement: int = 0, cube_half: float = 100.0,
               blobs: int = 0, sigma: float = 0.0, lod_error_mode: int = 1, coverage_height: float = 1024.0,
               mesh_library: int = 0, threads: int | None = None) -> Scene:
    lib = N.scenegen_lib()
    p = N.SceneParams(seed, instances, lod0, lod_count, placement, cube_half, blobs, sigma, lod_error_mode,
                      coverage_height, 2.0, mesh_library, threads or _threads(), 0.5, 4.0)
    cnt = N.SceneCounts()
    N.check(lib.sg_scene_counts_fn(C.byref(p), C.byref(cnt)))
    meshlets = np.zeros(cnt.meshlets, DT_MESHLET)
    objects = np.zeros(cnt.objects, DT_OBJECT)
    inst = np.zeros(cnt.objects, DT_INSTANCE)
    items = np.zeros(cnt.work_items, DT_ITEM)
    aabbs = np.zeros(cnt.objects, DT_AABB)
    draws = np.zeros(cnt.objects, DT_DRAWCALL)
    N.check(lib.sg_scene_generate(C.byref(p), meshlets.ctypes.data, objects.ctypes.data, inst.ctypes.data,
                                  items.ctypes.data, aabbs.ctypes.data, draws.ctypes.data))
    return Scene(meshlets, objects, inst, items, aabbs, draws, int(cnt.max_draw_count), lod0)


def _d3(v):
    return (C.c_double * 3)(*[float(x) for x in v])


def perspective(eye, target, up, fov_y_deg, aspect, near=0.1, far=1000.0) -> N.GpuCameraUniforms:
    cam = N.GpuCameraUniforms()
    N.scenegen_lib().sg_camera_perspective(_d3(eye), _d3(target), _d3(up), math.radians(fov_y_deg), aspect, near,
                                           far, C.byref(cam))
    return cam


def orthographic(eye, target, up, half, near, far) -> N.GpuCameraUniforms:
    cam = N.GpuCameraUniforms()
    N.scenegen_lib().sg_camera_ortho(_d3(eye), _d3(target), _d3(up), -half, half, -half, half, near, far,
                                     C.byref(cam))
    return cam


def make_depth(seed: int, width: int, height: int, n_rects: int, near: float, far: float, ortho: bool,
               pitch: int | None = None, threads: int | None = None) -> np.ndarray:
    pitch = pitch or width
    out = np.empty((height, pitch), np.float32)
    side = math.sqrt((256.0 / max(n_rects, 1)) * (width * height) / (1024.0 * 1024.0))
    N.check(N.scenegen_lib().sg_depth(seed, width, height, pitch, n_rects, side, near, far, 1 if ortho else 0,
                                      out.ctypes.data, threads or _threads()))
    return out[:, :width] if pitch != width else out


class _Split:
    """splitmix64 uniform stream for view parameters."""

    def __init__(self, seed: int):
        self.x = seed & 0xFFFFFFFFFFFFFFFF

    def u(self, a=0.0, b=1.0) -> float:
        self.x = (self.x + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
        z = self.x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
        z ^= z >> 31
        return a + (b - a) * ((z >> 11) / float(1 << 53))


def main_view(seed: int, width: int, height: int, n_rects: int) -> View:
    cam = perspective((0, 0, 0), (0, 0, -1), (0, 1, 0), 60.0, width / height)
    depth = make_depth(seed, width, height, n_rects, 0.1, 1000.0, False)
    return View(cam, width, height, depth)


def multiview_set(seed: int, depth: bool = True, scale: float = 1.0) -> list:
    """The 85-view mix: main 3840x2160, 4 orthographic cascades 2048^2, 16 spot 512^2, 64 probes 128^2.
    `scale` shrinks every view size (tests); occluder counts stay proportional to pixels."""
    rng = _Split(seed ^ 0x5EED)
    views = []

    def n_rects(w, h):
        return max(1, int(round(20000 * (w * h) / (3840 * 2160))))

    def add(cam, w, h, kind, idx, ortho=False):
        w, h = max(1, int(w * scale)), max(1, int(h * scale))
        d = make_depth(seed + 1000 + idx, w, h, n_rects(w, h), cam.position_near[3], cam.forward_far[3], ortho) \
            if depth else np.ones((h, w), np.float32)
        views.append(View(cam, w, h, d, kind))

    add(perspective((0, 0, 0), (0, 0, -1), (0, 1, 0), 60.0, 16 / 9), 3840, 2160, "main", 0)
    light = np.array([-0.3, -1.0, -0.2])
    light /= np.linalg.norm(light)
    t30 = math.tan(math.radians(30.0))
    for i, (n, f) in enumerate([(0.0, 8.0), (8.0, 32.0), (32.0, 128.0), (128.0, 512.0)]):
        hh, hw = f * t30, f * t30 * 16 / 9
        r = math.sqrt(hw * hw + hh * hh + ((f - n) / 2) ** 2)
        center = np.array([0.0, 0.0, -(n + f) / 2])
        eye = center - light * (r + 600.0)
        add(orthographic(eye, center, (0, 0, 1), r, 0.1, 2 * r + 1200.0), 2048, 2048, "cascade", 1 + i, ortho=True)
    for i in range(16):
        pos = [rng.u(-150, 150) for _ in range(3)]
        z = rng.u(-1, 1)
        phi = rng.u(0, 2 * math.pi)
        s = math.sqrt(max(0.0, 1 - z * z))
        d = (s * math.cos(phi), s * math.sin(phi), z)
        up = (0, 1, 0) if abs(d[1]) < 0.95 else (1, 0, 0)
        fov = rng.u(30.0, 90.0)
        add(perspective(pos, [pos[k] + d[k] for k in range(3)], up, fov, 1.0, 0.1, 500.0), 512, 512, "spot", 5 + i)
    dirs = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    k = 0
    for ix in range(4):
        for iy in range(4):
            for iz in range(4):
                pos = (-150 + 100 * ix, -150 + 100 * iy, -150 + 100 * iz)
                d = dirs[k % 6]
                up = (0, 0, 1) if d[1] != 0 else (0, 1, 0)
                add(perspective(pos, [pos[j] + d[j] for j in range(3)], up, 90.0, 1.0, 0.1, 500.0), 128, 128,
                    "probe", 21 + k)
                k += 1
    return views


def config(config_id: int, scale: float = 1.0, with_depth: bool = True, threads: int | None = None) -> Workload:
    """Builds workload `config_id` (0..3). `scale` (<= 1) shrinks instance counts and view
    sizes for quick tests while keeping every distribution."""
    seed = SEED_BASE + config_id

    def cnt(n):
        return max(1, int(round(n * scale)))

    if config_id == 0:
        sc = make_scene(seed, cnt(4096), 64, 4, 0, 100.0, lod_error_mode=0, coverage_height=1024.0 * scale,
                        threads=threads)
        w = max(8, int(1024 * scale))
        return Workload(0, sc, [main_view(seed, w, w, 256)])
    if config_id == 1:
        sc = make_scene(seed, cnt(10000), 100, 4, 0, 100.0, lod_error_mode=1, threads=threads)
        w, h = max(16, int(1920 * scale)), max(9, int(1080 * scale))
        return Workload(1, sc, [main_view(seed, w, h, max(1, int(2000 * scale)))])
    if config_id == 2:
        sc = make_scene(seed, cnt(100000), 100, 4, 1, 1000.0, 64, 20.0, lod_error_mode=1, threads=threads)
        w, h = max(16, int(3840 * scale)), max(9, int(2160 * scale))
        return Workload(2, sc, [main_view(seed, w, h, max(1, int(20000 * scale)))])
    if config_id == 3:
        sc = make_scene(seed, cnt(200000), 50, 4, 1, 1000.0, 64, 20.0, lod_error_mode=1, threads=threads)
        return Workload(3, sc, multiview_set(seed, with_depth, scale))
    raise ValueError(f"unknown config {config_id}")


@dataclass
class ServeRequestSpec:
    arrival_s: float
    scene: int
    views: list  # indices into the view pool


def serving_counts(scale: float = 1.0) -> list:
    """Instance counts of the serving workload's 8 scenes: log-uniform in [10k, 2M] (times `scale`)."""
    rng = _Split(SEED_BASE + 4)
    return [max(1, int(round(math.exp(rng.u(math.log(1e4), math.log(2e6))) * scale))) for _ in range(8)]


def serving_scene(k: int, scale: float = 1.0, threads: int | None = None) -> Scene:
    """Scene k of the serving workload: 100 LOD0 meshlets per instance, configs-1
    distributions (uniform in a 200 m cube, log-uniform LOD errors); the instances draw
    their meshes from a library of 256."""
    n = serving_counts(scale)[k]
    return make_scene(SEED_BASE + 5 + k, n, 100, 4, 0, 100.0, lod_error_mode=1, mesh_library=256, threads=threads)


def serving_scenes(scale: float = 1.0, threads: int | None = None) -> list:
    """The serving workload's 8 scenes (serving_scene 0..7)."""
    return [serving_scene(k, scale, threads) for k in range(8)]


def serving_requests(n: int, rate_hz: float = 2000.0, n_scenes: int = 8, pool: int = 85, max_views: int = 85,
                     seed: int = SEED_BASE + 4) -> list:
    """A seeded Poisson request stream: exponential inter-arrival times at `rate_hz`;
    each request names a scene uniformly and carries 1..max_views views drawn uniformly
    (with replacement) from a pool of `pool` views, so the view sizes follow the pool's mix."""
    g = np.random.default_rng(seed)
    t = np.cumsum(g.exponential(1.0 / rate_hz, size=n))
    out = []
    for i in range(n):
        k = int(g.integers(1, max_views + 1))
        out.append(ServeRequestSpec(float(t[i]), int(g.integers(n_scenes)), [int(x) for x in g.integers(pool, size=k)]))
    return out


def shadow_faces(seed: int, n_spot: int = 16, n_point: int = 4) -> tuple:
    """Shadow faces of the per-face shadow cull: ([256, 16] column-major view-projection
    matrices, faces in use): 4 orthographic cascades of growing size, spot lights, point
    lights (6 cube faces each); the rest zero."""
    rng = np.random.default_rng(seed)
    mats = []
    d = np.array([0.3, -1.0, 0.2])
    for half in (8.0, 32.0, 128.0, 512.0):
        mats.append(orthographic(tuple(-d * 600.0), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0), half, 1.0, 1500.0))
    for _ in range(n_spot):
        eye = rng.uniform(-150, 150, 3)
        target = eye + rng.normal(size=3) * 50.0
        mats.append(perspective(tuple(eye), tuple(target), (0.0, 1.0, 0.0) if abs(target[1] - eye[1]) < 40 else
                                  (1.0, 0.0, 0.0), float(rng.uniform(30, 90)), 1.0, 0.5, 300.0))
    axes = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    for _ in range(n_point):
        eye = rng.uniform(-100, 100, 3)
        for a in axes:
            up = (0.0, 1.0, 0.0) if a[1] == 0 else (0.0, 0.0, 1.0)
            mats.append(perspective(tuple(eye), tuple(eye + np.array(a, float)), up, 90.0, 1.0, 0.1, 60.0))
    out = np.zeros((256, 16), np.float32)
    for i, c in enumerate(mats):
        out[i] = np.ctypeslib.as_array(c.view_proj)
    return out, len(mats)


def shadow_draws(seed: int, instances: int, draws: int, spread: float = 200.0) -> tuple:
    """(instances, DrawIndexedIndirect [draws, 5] uint32) of the per-face shadow cull:
    spheres uniform in a cube, with radius 0, -1 and NaN mixed in, and 1% of the draws
    naming an instance past the array."""
    rng = np.random.default_rng(seed)
    inst = np.zeros(instances, DT_INSTANCE)
    inst["bounds"][:, :3] = rng.uniform(-spread, spread, (instances, 3))
    inst["bounds"][:, 3] = rng.uniform(0.2, 6.0, instances)
    k = max(1, instances // 50)
    inst["bounds"][rng.choice(instances, k, replace=False), 3] = 0.0
    inst["bounds"][rng.choice(instances, k, replace=False), 3] = -1.0
    inst["bounds"][rng.choice(instances, 2, replace=False), 3] = np.nan
    src = np.zeros((draws, 5), np.uint32)
    src[:, 0] = rng.integers(3, 3000, draws)
    src[:, 1] = 1
    src[:, 2] = rng.integers(0, 1 << 20, draws)
    src[:, 3] = rng.integers(0, 1 << 16, draws)
    src[:, 4] = rng.integers(0, instances, draws)
    src[rng.choice(draws, max(1, draws // 100), replace=False), 4] = instances + 7  # past the array
    return inst, src



def work_items_for(objects) -> list:
    """64-meshlet work spans of (object_index, max_meshlet_count) pairs, in order
    (crates/helio/src/scene/virtual_geometry/rebuild.rs:45-58): one span per started
    block of 64 meshlets of the largest LOD; an object without meshlets has none."""
    out = []
    for obj, max_count in objects:
        out.extend((obj, base) for base in range(0, max_count, 64))
    return out


DT_MESH = np.dtype(N.np_dtype(N.VgMeshRecord))


@dataclass
class Library:
    """Input of the VG input producer: a descriptor pool, mesh records and dense object
    slots (mesh index, VG_NO_MESH for a free slot, and instance data)."""
    pool: np.ndarray
    meshes: np.ndarray
    slot_mesh: np.ndarray
    slot_instances: np.ndarray


def library_from_scene(scene: Scene, free_slots: float = 0.0, seed: int = 1) -> Library:
    """Mesh library whose rebuild gives back the scene's objects: one record per distinct
    (descriptor range, LOD table) of the scene's objects, the scene's meshlets as the
    pool, and one slot per object in order, with free slots mixed in at rate free_slots."""
    obj = scene.objects
    lc = np.minimum(obj["lod_count"], 8).astype(np.int64)
    used = np.arange(8)[None, :] < lc[:, None]
    firsts = obj["lod_first_meshlets"].astype(np.int64)
    counts = obj["lod_meshlet_counts"].astype(np.int64)
    big = np.int64(1) << 40
    first = np.where(used, firsts, big).min(axis=1)
    end = np.where(used, firsts + counts, 0).max(axis=1)
    first = np.where(lc > 0, first, 0)
    rec = np.zeros(len(obj), DT_MESH)
    rec["first_meshlet"] = first
    rec["meshlet_count"] = np.where(lc > 0, end - first, 0)
    rec["lod_count"] = obj["lod_count"]
    rec["max_meshlet_count"] = obj["max_meshlet_count"]
    rec["local_bounds"] = obj["local_bounds"]
    rec["lod_errors"] = obj["lod_errors"]
    rec["lod_first_meshlets"] = np.where(used, firsts - first[:, None], 0)
    rec["lod_meshlet_counts"] = obj["lod_meshlet_counts"]
    meshes, mesh_of = np.unique(rec.view(np.dtype((np.void, DT_MESH.itemsize))), return_inverse=True)
    meshes = meshes.view(DT_MESH)
    mesh_of = mesh_of.astype(np.uint32).reshape(-1)
    rng = np.random.default_rng(seed)
    n_free = int(round(free_slots * len(obj)))
    slot_mesh = np.full(len(obj) + n_free, N.VG_NO_MESH, np.uint32)
    slot_inst = np.zeros(len(obj) + n_free, DT_INSTANCE)
    taken = np.sort(rng.choice(len(slot_mesh), size=len(obj), replace=False)) if n_free else np.arange(len(obj))
    slot_mesh[taken] = mesh_of
    slot_inst[taken] = scene.instances
    return Library(scene.meshlets, meshes, slot_mesh, slot_inst)


def frame_data(scene: Scene, buffer_version: int = 1, instance_version: int = 1, dirty=(0, 0),
               device: dict | None = None) -> N.VgFrameData:
    """VgFrameData over host arrays (or device tensors when `device` holds them)."""
    src = device or {"meshlets": scene.meshlets, "objects": scene.objects, "instances": scene.instances,
                     "work_items": scene.work_items}

    def p(a):
        return a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data

    return N.VgFrameData(p(src["meshlets"]), p(src["objects"]), p(src["instances"]), p(src["work_items"]),
                         len(scene.meshlets), len(scene.objects), len(scene.work_items),
                         min(scene.max_draw_count, 0xFFFFFFFF), buffer_version, instance_version, dirty[0], dirty[1],
                         N.HELIO_MEM_DEVICE if device else N.HELIO_MEM_HOST, 0)
