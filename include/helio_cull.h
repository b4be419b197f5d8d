/*
 * helio_cull.h — C-ABI of the B200 (sm_100a) GPU visibility path:
 *   Hi-Z pyramid → instance frustum / Hi-Z occlusion cull → virtual-geometry
 *   object LOD select + meshlet frustum / normal-cone / Hi-Z cull →
 *   deterministic draw-argument compaction.
 *
 * Each reference RenderPass (crates/helio-core/src/traits.rs:276-470) becomes one
 * opaque context with the same lifecycle:
 *     create  (RenderPass::new)
 *     prepare (RenderPass::prepare, PrepareContext: uploads, uniforms)
 *     execute (RenderPass::execute, PassContext: GPU work on one stream)
 *     resize  (RenderPass::on_resize)
 *     publish (RenderPass::publish: device pointers of the outputs)
 *     destroy
 * Byte layouts of every buffer are libhelio's (crates/libhelio/src/*.rs) and are
 * asserted by static_assert in the library.
 *
 * Conventions
 *   - Every entry point returns an int32_t status (HELIO_OK on success). No
 *     exception or abort crosses this boundary; helio_last_error() returns the
 *     message of the calling thread's last failure.
 *   - `stream` arguments are cudaStream_t passed as void* (NULL = legacy stream).
 *   - Pointers documented "device" are CUDA device pointers owned by the caller
 *     and borrowed for the duration of the call's GPU work. Pointers returned by
 *     *_publish stay owned by the context and remain valid until the next
 *     prepare/resize/destroy of that context.
 *   - A context is externally synchronised: one thread and one stream at a time
 *     (reference: RenderPass is Send + Sync and driven by one thread per frame,
 *     crates/helio-core/src/graph/execution.rs:343-606). Distinct contexts may
 *     run concurrently on distinct streams.
 *   - execute() never allocates device memory (reference rule for the hot path,
 *     crates/helio-core/src/traits.rs:164-166); buffers grow in prepare().
 *   - Arithmetic is IEEE-754 binary32 without contraction (no FMA), with
 *     correctly-rounded division and square root, in the WGSL operation order
 *     of the reference shaders, so decisions are bit-reproducible.
 */
#ifndef HELIO_CULL_H
#define HELIO_CULL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HELIO_ABI_VERSION 1

/* ── Status codes (reference: helio_core::Error, crates/helio-core/src/error.rs:62-167) ── */
#define HELIO_OK 0
#define HELIO_ERR_CUDA 1          /* a CUDA runtime call failed (Error::Gpu)                 */
#define HELIO_ERR_INVALID_ARG 2   /* bad pointer / size / config (Error::InvalidPassConfig)   */
#define HELIO_ERR_RESOURCE 3      /* missing input: no Hi-Z, no scene (Error::ResourceNotFound) */
#define HELIO_ERR_CAPACITY 4      /* soft: visible draws exceeded capacity; counters valid    */
#define HELIO_ERR_TIMEOUT 5       /* a bounded device-side wait gave up; outputs invalid      */
#define HELIO_ERR_BUDGET 6        /* admission refused: device-memory budget exceeded         */
#define HELIO_ERR_NOT_READY 7     /* nothing to return yet (serving poll)                     */

/* Memory space of caller-provided input arrays. */
#define HELIO_MEM_HOST 0u
#define HELIO_MEM_DEVICE 1u

/* ════════════════════════════════════════════════════════════════════════════
 * libhelio byte layouts (all little-endian, 4-byte aligned, tightly packed)
 * ════════════════════════════════════════════════════════════════════════════ */

/* GpuCameraUniforms, crates/libhelio/src/camera.rs:10-57. 368 bytes.
 * Matrices are column-major: m[c*4 + r]. view_proj = proj * view. */
typedef struct HelioGpuCameraUniforms {
    float view[16];
    float proj[16];
    float view_proj[16];
    float inv_view_proj[16];
    float position_near[4]; /* xyz = camera position, w = near plane */
    float forward_far[4];   /* xyz = forward, w = far plane */
    float jitter_frame[4];
    float prev_view_proj[16];
} HelioGpuCameraUniforms;

/* GpuInstanceData, crates/libhelio/src/instance.rs:28-45. 144 bytes. */
typedef struct HelioGpuInstanceData {
    float model[16];      /* column-major model matrix */
    float normal_mat[12]; /* three vec4 columns of the normal matrix (w unused) */
    float bounds[4];      /* world-space sphere: xyz centre, w radius */
    uint32_t mesh_id;
    uint32_t material_id;
    uint32_t flags;       /* bit 0 = casts shadow */
    uint32_t lightmap_index;
} HelioGpuInstanceData;

/* GpuInstanceAabb, crates/libhelio/src/instance.rs:47-65. 32 bytes. */
typedef struct HelioGpuInstanceAabb {
    float min[3];
    float pad0;
    float max[3];
    float pad1;
} HelioGpuInstanceAabb;

/* GpuDrawCall, crates/libhelio/src/draw.rs:26-37. 20 bytes. */
typedef struct HelioGpuDrawCall {
    uint32_t index_count;
    uint32_t first_index;
    int32_t vertex_offset;
    uint32_t first_instance;
    uint32_t instance_count;
} HelioGpuDrawCall;

/* DrawIndexedIndirectArgs, crates/libhelio/src/draw.rs:39-50. 20 bytes. */
typedef struct HelioDrawIndexedIndirectArgs {
    uint32_t index_count;
    uint32_t instance_count;
    uint32_t first_index;
    int32_t base_vertex;
    uint32_t first_instance;
} HelioDrawIndexedIndirectArgs;

/* GpuMeshletEntry, crates/libhelio/src/meshlet.rs:41-70. 64 bytes. */
typedef struct HelioGpuMeshletEntry {
    float center[3];
    float radius;
    float cone_apex[3];
    float cone_cutoff; /* > 1 disables the cone test */
    float cone_axis[3];
    float lod_error;
    uint32_t first_index;
    uint32_t index_count;
    int32_t vertex_offset;
    uint32_t instance_index; /* reserved */
} HelioGpuMeshletEntry;

#define HELIO_VG_LOD_LEVELS 8
#define HELIO_VG_MESHLETS_PER_WORK_ITEM 64

/* GpuVgObject, crates/libhelio/src/meshlet.rs:72-97. 128 bytes. `reserved` receives
 * selected LOD + 1 (0 = culled) from the object-select stage. */
typedef struct HelioGpuVgObject {
    uint32_t instance_index;
    uint32_t lod_count;
    uint32_t max_meshlet_count;
    uint32_t reserved;
    float local_bounds[4];
    float lod_errors[HELIO_VG_LOD_LEVELS];
    uint32_t lod_first_meshlets[HELIO_VG_LOD_LEVELS];
    uint32_t lod_meshlet_counts[HELIO_VG_LOD_LEVELS];
} HelioGpuVgObject;

/* GpuVgDraw, crates/libhelio/src/meshlet.rs:99-111. 16 bytes. */
typedef struct HelioGpuVgDraw {
    uint32_t instance_index;
    uint32_t meshlet_index;
    uint32_t lod_level;
    uint32_t reserved;
} HelioGpuVgDraw;

/* GpuVgWorkItem, crates/libhelio/src/meshlet.rs:113-124. 8 bytes. */
typedef struct HelioGpuVgWorkItem {
    uint32_t object_index;
    uint32_t local_meshlet_base;
} HelioGpuVgWorkItem;

/* InstanceCullData, crates/helio-pass-virtual-geometry/src/lib.rs:122-130. 16 bytes. */
typedef struct HelioInstanceCullData {
    float max_scale;
    float min_scale;
    uint32_t cone_cull_enabled;
    uint32_t valid_transform;
} HelioInstanceCullData;

/* ════════════════════════════════════════════════════════════════════════════
 * Library-wide
 * ════════════════════════════════════════════════════════════════════════════ */

int32_t helio_abi_version(void);
/* Message of this thread's last failing call ("" if none). */
const char* helio_last_error(void);
const char* helio_status_string(int32_t status);
/* Number of kernels this library has launched in this process (all contexts). */
uint64_t helio_kernel_launch_count(void);

/* GPU-side kernel profiler (reference: the GPU timestamp profiler,
 * crates/helio-core/src/profiling/gpu.rs:106-155). While enabled, every kernel
 * launch of this library is bracketed by CUDA events on its own stream;
 * helio_profiler_collect synchronises those events and returns, per kernel
 * name, the launch count and the summed device time. */
typedef struct helio_kernel_timing {
    char name[40];
    uint64_t launches;
    double total_ms;
} helio_kernel_timing;
int32_t helio_profiler_enable(int32_t enabled);
int32_t helio_profiler_collect(helio_kernel_timing* out, uint32_t capacity, uint32_t* count);
void helio_profiler_reset(void);

/* mip_levels(w, h) = bit length of max(w, h), at least 1.
 * Reference: crates/helio-pass-hiz/src/lib.rs:376-379. */
uint32_t helio_mip_levels(uint32_t width, uint32_t height);

/* CPU Gribb–Hartmann plane extraction with the len > 1e-10 guard, used by the
 * instance frustum pass. planes_out[6*4] = left, right, bottom, top, near, far.
 * Reference: crates/helio-pass-indirect-dispatch/src/lib.rs:271-300. */
void helio_extract_frustum_planes(const float view_proj[16], float planes_out[24]);

/* InstanceCullData::from_instance over `count` instances, computed on the GPU
 * (device in, device out). Reference: crates/helio-pass-virtual-geometry/src/lib.rs:132-167. */
int32_t helio_instance_cull_data(const HelioGpuInstanceData* instances_dev, uint32_t count,
                                 HelioInstanceCullData* out_dev, void* stream);

/* ════════════════════════════════════════════════════════════════════════════
 * Hi-Z pyramid — HiZBuildPass (crates/helio-pass-hiz/src/lib.rs:381-548)
 *   hiz_depth_copy.wgsl:13-19 + hiz_build.wgsl:12-23, fused into one launch.
 * ════════════════════════════════════════════════════════════════════════════ */

#define HELIO_HIZ_MAX_MIPS 12 /* crates/helio-pass-hiz/src/lib.rs:27 */

/* Level 0 is the caller's depth buffer itself instead of a copy (saves 8 B/px).
 * Only valid while the depth buffer is not overwritten before the pyramid is read. */
#define HELIO_HIZ_ALIAS_MIP0 1u
/* Read level 0 with 128-bit loads instead of TMA tile loads (the same results; for
 * comparing the two). Depth that TMA cannot address (not 16-byte aligned, or a row
 * pitch that is not a multiple of 4 floats) always takes the 128-bit-load path. */
#define HELIO_HIZ_NO_TMA 2u

typedef struct helio_hiz_config {
    uint32_t width;
    uint32_t height;
    uint32_t flags;
} helio_hiz_config;

/* The published pyramid: R32Float levels, level l is width[l] x height[l] floats,
 * row-major with row pitch pitch[l] floats. width[l] = max(1, width >> l). */
typedef struct helio_hiz_pyramid {
    uint32_t mip_count; /* min(helio_mip_levels(w, h), 12) */
    uint32_t width[HELIO_HIZ_MAX_MIPS];
    uint32_t height[HELIO_HIZ_MAX_MIPS];
    uint32_t pitch[HELIO_HIZ_MAX_MIPS];
    const float* levels[HELIO_HIZ_MAX_MIPS];
} helio_hiz_pyramid;

typedef struct helio_hiz_pass helio_hiz_pass;

int32_t helio_hiz_create(const helio_hiz_config* config, helio_hiz_pass** out);
/* depth_dev: device, width x height floats, row pitch depth_pitch floats (0 = width).
 * camera_generation: the pass skips the rebuild when it equals the previous
 * frame's value (reference lib.rs:472-478); pass UINT64_MAX to always rebuild. */
int32_t helio_hiz_prepare(helio_hiz_pass* pass, const float* depth_dev, uint32_t depth_pitch,
                          uint64_t camera_generation);
int32_t helio_hiz_execute(helio_hiz_pass* pass, void* stream);
/* Synchronises `stream`; HELIO_ERR_TIMEOUT if a TMA tile load of an earlier execute
 * never completed (its bounded wait gave up; sticky for the pass). The reference's
 * dispatches have no device-side waits (crates/helio-pass-hiz/src/lib.rs:503-531). */
int32_t helio_hiz_device_status(const helio_hiz_pass* pass, void* stream);
int32_t helio_hiz_resize(helio_hiz_pass* pass, uint32_t width, uint32_t height);
int32_t helio_hiz_publish(const helio_hiz_pass* pass, helio_hiz_pyramid* out);
void helio_hiz_destroy(helio_hiz_pass* pass);

/* Hi-Z build without any device allocation. This entry point has no counterpart in
 * the reference: it is for callers that cannot allocate device memory when they
 * build the pyramid (an engine whose pools own every allocation and forbid new
 * ones during its frame loop, a plugin whose device-memory use must stay fixed, a
 * frame loop that cannot take an allocation's implicit synchronisation).
 * HiZBuildPass allocates its scratch in create(); this call keeps it — one
 * completion ticket per view — in a fixed device array inside the library instead,
 * and passes the views' descriptors as the kernel's parameter (no upload):
 *   - at most 32 views per call; every GPU that loads the library holds the array
 *     (128 bytes) until the process exits; more views are rejected with
 *     HELIO_ERR_INVALID_ARG;
 *   - every call shares the array and clears the tickets first, so calls whose GPU
 *     work overlaps (other streams or threads) race and must be ordered by the caller;
 *   - the first call on each device looks the array's device address up and caches
 *     it; make that first call before any stream capture.
 * The caller passes each view's depth (device) and one device buffer `levels` of
 * `levels_floats` floats, 16-byte aligned (else HELIO_ERR_INVALID_ARG), that
 * receives every view's levels one after another (levels 1.. and, unless
 * HELIO_HIZ_ALIAS_MIP0, a copy of level 0); a view needs sum over its levels of
 * pitch * height floats with pitch = width rounded up to 4, each view starting on a
 * 4-float boundary. pyramids_out[v] describes view v. A CUDA error already pending
 * on the calling thread is reported as HELIO_ERR_CUDA and left pending.
 * No cudaMalloc, cudaFree or allocating library routine is called. */
typedef struct helio_hiz_view_input {
    const float* depth; /* device, width x height, row pitch `pitch` floats (0 = width) */
    uint32_t width;
    uint32_t height;
    uint32_t pitch;
    uint32_t flags;     /* HELIO_HIZ_ALIAS_MIP0 or 0 */
} helio_hiz_view_input;
int32_t helio_hiz_build_noalloc(uint32_t view_count, const helio_hiz_view_input* views, float* levels,
                                size_t levels_floats, helio_hiz_pyramid* pyramids_out, void* stream);

/* ════════════════════════════════════════════════════════════════════════════
 * Instance-level culling — IndirectDispatchPass + OcclusionCullPass
 * ════════════════════════════════════════════════════════════════════════════ */

/* SceneResources subset (crates/helio-core/src/scene/resources.rs:118-131); all device. */
typedef struct helio_scene_buffers {
    const HelioGpuCameraUniforms* camera;
    const HelioGpuInstanceData* instances;
    uint32_t instance_count;
    const HelioGpuDrawCall* draw_calls;
    uint32_t draw_count;
    const HelioGpuInstanceAabb* aabbs; /* one per instance */
    uint32_t* indirect;                /* draw_count x 5 u32 (DrawIndexedIndirectArgs) */
} helio_scene_buffers;

/* Cull statistics (crates/helio-pass-indirect-dispatch/shaders/indirect_dispatch.wgsl:69-77):
 * [0] total draws [1] frustum culled [2] sub-pixel culled [3] frustum visible
 * [4] occlusion culled [5] shadow casters [6] shadow visible [7] shadow occlusion culled.
 * Passes accumulate; the caller clears once per frame (crates/helio/src/renderer/render.rs:441). */
#define HELIO_CULL_STATS_COUNT 8

typedef struct helio_indirect_dispatch_pass helio_indirect_dispatch_pass;

/* stats_dev: device u32[8] shared with the occlusion pass (reference: new(device, cull_stats_buf)). */
int32_t helio_indirect_dispatch_create(uint32_t* stats_dev, helio_indirect_dispatch_pass** out);
/* Extracts the frustum planes on the host from camera->view_proj (host pointer) and
 * records draw_count. Reference: crates/helio-pass-indirect-dispatch/src/lib.rs:178-191. */
int32_t helio_indirect_dispatch_prepare(helio_indirect_dispatch_pass* pass,
                                        const HelioGpuCameraUniforms* camera_host,
                                        uint32_t draw_count);
/* One thread per draw: indirect_dispatch.wgsl:100-176. */
int32_t helio_indirect_dispatch_execute(helio_indirect_dispatch_pass* pass,
                                        const helio_scene_buffers* scene, void* stream);
void helio_indirect_dispatch_destroy(helio_indirect_dispatch_pass* pass);

typedef struct helio_occlusion_cull_pass helio_occlusion_cull_pass;

int32_t helio_occlusion_cull_create(uint32_t screen_width, uint32_t screen_height,
                                    uint32_t* stats_dev, helio_occlusion_cull_pass** out);
/* Reference: crates/helio-pass-occlusion-cull/src/lib.rs:297-317 (the static Hi-Z:
 * helio_occlusion_cull_set_static_hiz). */
int32_t helio_occlusion_cull_prepare(helio_occlusion_cull_pass* pass, uint32_t draw_count);
/* One thread per draw: occlusion_cull.wgsl:146-220. Frame 0 is skipped
 * (no temporal pyramid yet, reference lib.rs:321). */
int32_t helio_occlusion_cull_execute(helio_occlusion_cull_pass* pass,
                                     const helio_scene_buffers* scene,
                                     const helio_hiz_pyramid* hiz, uint64_t frame_num,
                                     void* stream);
int32_t helio_occlusion_cull_resize(helio_occlusion_cull_pass* pass, uint32_t w, uint32_t h);

/* A baked static Hi-Z (HiZBuildPass::load_static_hiz, crates/helio-pass-hiz/src/lib.rs:272-373):
 * level 0 of its R32Float 3-D texture, grid_resolution[0] x [1] x ([2] * 6) texels with x
 * fastest, the six direction layers (+X, -X, +Y, -Y, +Z, -Z) stacked along z, over the
 * world box [world_bounds_min, world_bounds_max]. */
typedef struct helio_static_hiz {
    const float* texels; /* device */
    uint32_t grid_resolution[3];
    float world_bounds_min[3];
    float world_bounds_max[3];
} helio_static_hiz;

/* The static Hi-Z branch of the occlusion test (occlusion_cull.wgsl:222-259), for this
 * pass's executes, separate or fused, until the next call: `hiz` non-NULL switches it
 * on (OcclusionCullPass::set_static_hiz_metadata plus a static Hi-Z in the frame
 * resources, occlusion-cull/src/lib.rs:267-276, 297-299), NULL off (the default). A draw
 * that the dynamic test keeps is culled when its camera distance exceeds the texture's
 * distance at its centre plus 0.1. The texture is read with the reference's linear
 * filter and clamp-to-edge addressing; WebGPU leaves the filter's weight precision to
 * the implementation, and this library rounds the weights to 8 fractional bits (the
 * precision CUDA documents for its texture unit) and interpolates x, then y, then z as
 * (1 - t) a + t b. The texels stay borrowed until the next call. */
int32_t helio_occlusion_cull_set_static_hiz(helio_occlusion_cull_pass* pass, const helio_static_hiz* hiz);
void helio_occlusion_cull_destroy(helio_occlusion_cull_pass* pass);

/* Both instance passes in one kernel launch (frustum + sub-pixel, then the Hi-Z
 * test when frame_num > 0). Writes the same indirect bytes and stats as
 * helio_indirect_dispatch_execute followed by helio_occlusion_cull_execute. */
int32_t helio_instance_cull_fused_execute(helio_indirect_dispatch_pass* frustum,
                                          helio_occlusion_cull_pass* occlusion,
                                          const helio_scene_buffers* scene,
                                          const helio_hiz_pyramid* hiz, uint64_t frame_num,
                                          void* stream);

/* ════════════════════════════════════════════════════════════════════════════
 * Virtual geometry — VirtualGeometryPass cull half
 *   (crates/helio-pass-virtual-geometry/src/rendering.rs:703-1165,
 *    shaders/vg_cull.wgsl:126-405)
 * ════════════════════════════════════════════════════════════════════════════ */

/* VgFrameData, crates/libhelio/src/frame.rs:485-516. `memory` says whether the four
 * arrays are host or device pointers. instances has one entry per object. */
typedef struct helio_vg_frame_data {
    const HelioGpuMeshletEntry* meshlets;
    const HelioGpuVgObject* objects;
    const HelioGpuInstanceData* instances;
    const HelioGpuVgWorkItem* work_items;
    uint32_t meshlet_count;
    uint32_t object_count;
    uint32_t work_item_count;
    uint32_t max_draw_count;
    uint64_t buffer_version;
    uint64_t instance_version;
    uint32_t instance_dirty_start;
    uint32_t instance_dirty_count;
    uint32_t memory; /* HELIO_MEM_HOST or HELIO_MEM_DEVICE */
    uint32_t reserved0;
} helio_vg_frame_data;

/* LodQuality, crates/helio-pass-virtual-geometry/src/lib.rs:174-203. */
#define HELIO_LOD_LOW 0u    /* 4.0 px */
#define HELIO_LOD_MEDIUM 1u /* 2.0 px (default) */
#define HELIO_LOD_HIGH 2u   /* 1.0 px */
#define HELIO_LOD_ULTRA 3u  /* 0.5 px */
float helio_lod_max_error_pixels(uint32_t lod_quality);

/* DEFAULT_MAX_PUBLISHED_MESHLETS, crates/helio-pass-virtual-geometry/src/lib.rs:76. */
#define HELIO_VG_DEFAULT_PUBLICATION_LIMIT 262144u
/* Counter layout (lib.rs:21-28): [0] attempted visible draws, [1] rejected by
 * capacity, [2..9] selected-LOD object histogram, [10] deepest LOD among visible objects. */
#define HELIO_VG_COUNTER_COUNT 11u

typedef struct helio_vg_config {
    uint32_t width;             /* render size: CullUniforms.screen_width/height */
    uint32_t height;
    uint32_t lod_quality;       /* HELIO_LOD_* */
    uint32_t publication_limit; /* 0 = HELIO_VG_DEFAULT_PUBLICATION_LIMIT */
    uint32_t counter_count;     /* 2 (benchmark layout) or 11 (production layout); 0 = 11 */
    uint32_t flags;             /* HELIO_VG_CLEAR_INDIRECT */
} helio_vg_config;

/* For a draw side without multi_draw_indexed_indirect_count: execute zeroes the whole
 * indirect buffer before the cull, so that drawing all `capacity` records draws exactly
 * the visible ones (the zeroed records are empty draws). The reference clears it when
 * the device lacks the count feature (rendering.rs:1127-1130, 1203-1208). Without the
 * flag only the first min(counters[0], capacity) records are defined: the count form
 * reads the draw count from byte 0 of `counters` (rendering.rs:648-660, 1194-1201). */
#define HELIO_VG_CLEAR_INDIRECT 1u

/* Published outputs (device pointers owned by the pass). */
typedef struct helio_vg_outputs {
    HelioDrawIndexedIndirectArgs* indirect; /* [capacity]; first `min(counters[0], capacity)` valid */
    HelioGpuVgDraw* draws;                  /* [capacity] */
    uint32_t* counters;                     /* [counter_count] */
    uint32_t* visibility;                   /* [2 * work_item_count]: bit l of word 2w+(l>>5)
                                               = meshlet l of work item w visible */
    HelioGpuVgObject* objects;              /* [object_count]; reserved = selected LOD + 1 */
    uint32_t capacity;
    uint32_t counter_count;
    uint32_t work_item_count;
    uint32_t object_count;
} helio_vg_outputs;

typedef struct helio_vg_pass helio_vg_pass;

int32_t helio_vg_create(const helio_vg_config* config, helio_vg_pass** out);
/* Uploads on buffer_version change, else patches [instance_dirty_start, +count) on
 * instance_version change; recomputes InstanceCullData on the GPU for what changed.
 * Reference: rendering.rs:708-859. May allocate (growth). */
int32_t helio_vg_prepare(helio_vg_pass* pass, const helio_vg_frame_data* frame, void* stream);
/* Clears the counters, runs object select then meshlet cull with deterministic
 * compaction: the visible draws are stored in (work item, lane) order and
 * first_instance = slot. camera: device pointer. hiz: published pyramid.
 * Returns HELIO_ERR_CAPACITY only if the caller asks for it via
 * helio_vg_check_overflow(); execute itself never reads back. */
int32_t helio_vg_execute(helio_vg_pass* pass, const HelioGpuCameraUniforms* camera_dev,
                         const helio_hiz_pyramid* hiz, void* stream);
int32_t helio_vg_resize(helio_vg_pass* pass, uint32_t width, uint32_t height);
int32_t helio_vg_set_lod_quality(helio_vg_pass* pass, uint32_t lod_quality);
int32_t helio_vg_publish(const helio_vg_pass* pass, helio_vg_outputs* out);
/* Synchronises `stream` and reports any asynchronous CUDA error of the queued
 * work (the cull kernels themselves never wait on one another). */
int32_t helio_vg_device_status(helio_vg_pass* pass, void* stream);
void helio_vg_destroy(helio_vg_pass* pass);

/* ════════════════════════════════════════════════════════════════════════════
 * Batched multi-view culling (no single reference counterpart: it performs, for
 * every view of a batch, what HiZBuildPass + VirtualGeometryPass's cull half do
 * for one view, against one device-resident scene, in one cooperative launch).
 * ════════════════════════════════════════════════════════════════════════════ */

/* A device-resident virtual-geometry scene shared by batches. Upload follows the
 * VgFrameData version rules of helio_vg_prepare (rendering.rs:708-819). Work items
 * are not used: a batch derives the 64-meshlet spans of each object's selected LOD. */
typedef struct helio_vg_scene helio_vg_scene;
typedef struct helio_vg_scene_info {
    uint32_t meshlet_count;
    uint32_t object_count;
    uint64_t lod0_meshlets; /* sum over objects of lod_meshlet_counts[0] */
    uint64_t max_spans;     /* sum over objects of ceil(max_meshlet_count / 64) */
    uint64_t device_bytes;
} helio_vg_scene_info;
int32_t helio_vg_scene_create(helio_vg_scene** out);
int32_t helio_vg_scene_upload(helio_vg_scene* scene, const helio_vg_frame_data* frame, void* stream);
int32_t helio_vg_scene_info_get(const helio_vg_scene* scene, helio_vg_scene_info* out);
void helio_vg_scene_destroy(helio_vg_scene* scene);

#define HELIO_BATCH_MAX_VIEWS 128u
/* helio_batch_config.flags: also write per-span visibility words. */
#define HELIO_BATCH_SPAN_VISIBILITY 1u

typedef struct helio_batch_config {
    uint32_t max_views; /* <= HELIO_BATCH_MAX_VIEWS */
    uint32_t flags;
    uint64_t max_spans; /* capacity of the active-span list; 0 = every view at LOD 0 */
    uint32_t max_ctas;     /* CTAs of the cooperative launch; 0 = as many as fit on the device.
                            * Fewer CTAs leave SMs free for batches launched on other streams. */
    uint32_t select_views; /* views tested per object load in the select (1..32); 0 = 32 */
    uint32_t cull_ctas;    /* CTAs of the meshlet-test launch; 0 = the same share of the device
                            * as max_ctas gives the first launch. Capped at what fits. */
    uint32_t reserved;     /* 0 */
} helio_batch_config;

/* One view of a batch. */
typedef struct helio_batch_view {
    HelioGpuCameraUniforms camera; /* host copy, uploaded by prepare / set_cameras */
    const float* depth;            /* device, width x height floats, row pitch depth_pitch */
    uint32_t depth_pitch;          /* floats; 0 = width */
    uint32_t width;                /* render size (Hi-Z size, CullUniforms.screen_*) */
    uint32_t height;
    float lod_error_threshold_px;  /* 0 = LodQuality::Medium (2 px) */
    uint32_t draw_capacity;        /* 0 = min(sum of max_meshlet_count, 262144) */
    uint32_t flags;                /* HELIO_HIZ_ALIAS_MIP0: level 0 is the depth buffer itself */
} helio_batch_view;

/* Per-view results (device pointers owned by the batch). indirect / draws hold
 * min(counters[0], capacity) draws in (object, span, lane) order, first_instance = slot;
 * counters use the 11-word VG layout; lod[o] = selected LOD + 1 of object o (0 = culled). */
typedef struct helio_batch_view_outputs {
    HelioDrawIndexedIndirectArgs* indirect;
    HelioGpuVgDraw* draws;
    uint32_t* counters;
    uint8_t* lod;
    uint32_t capacity;
    uint32_t object_count;
    helio_hiz_pyramid pyramid;
} helio_batch_view_outputs;

/* The active spans of the last execute: spans[4 * k + 0..3] = first meshlet,
 * n | lod << 8 | view << 16, instance, object; view v owns spans
 * [view_span_start[v], view_span_start[v + 1]) (padded with n = 0 to a multiple of 32).
 * visibility (if enabled) holds 2 words per span: bit l = meshlet l of the span visible. */
typedef struct helio_batch_span_list {
    const uint32_t* spans;
    const uint32_t* visibility;
    const uint32_t* view_span_start;
    uint32_t span_capacity;
    uint32_t view_count;
} helio_batch_span_list;

typedef struct helio_batch helio_batch;
int32_t helio_batch_create(const helio_batch_config* config, helio_batch** out);
/* Binds a scene and a set of views; (re)allocates pyramids, outputs and scratch. */
int32_t helio_batch_prepare(helio_batch* batch, const helio_vg_scene* scene, uint32_t view_count,
                            const helio_batch_view* views, void* stream);
/* Replaces the cameras of the prepared views (no allocation). */
int32_t helio_batch_set_cameras(helio_batch* batch, uint32_t view_count, const HelioGpuCameraUniforms* cameras,
                                void* stream);
/* The same from device memory (stream-ordered; for hosts that upload cameras with
 * their other per-frame inputs in one copy). */
int32_t helio_batch_set_cameras_device(helio_batch* batch, uint32_t view_count, const HelioGpuCameraUniforms* cameras,
                                       void* stream);
/* Clears the counters and runs the persistent cooperative kernel on `stream`. */
int32_t helio_batch_execute(helio_batch* batch, void* stream);
int32_t helio_batch_get_view_outputs(const helio_batch* batch, uint32_t view, helio_batch_view_outputs* out);
int32_t helio_batch_get_spans(const helio_batch* batch, helio_batch_span_list* out);
/* Packs every view's published draws (min(counters[0], capacity) each) into one pair
 * of device arrays, view after view, on `stream` (after helio_batch_execute):
 * offsets[v] = first draw of view v, offsets[view_count] = the total; draws past
 * `capacity` are not written. Lets a host read all views' draws back in one copy. */
int32_t helio_batch_pack_draws(const helio_batch* batch, HelioDrawIndexedIndirectArgs* indirect, HelioGpuVgDraw* draws,
                               uint32_t* offsets, uint64_t capacity, void* stream);
/* Tracing: device time (us) of the phases of the last execute, read from timer
 * stamps the kernel takes at its grid barriers (synchronises `stream`). Order:
 * view setup, Hi-Z + object select, span-count scan, span expansion, meshlet tests,
 * group-count scan, emission; then the largest per-CTA busy time on Hi-Z tiles and
 * on object chunks within the Hi-Z + select phase. */
int32_t helio_batch_get_phase_times(helio_batch* batch, double* us_out, uint32_t capacity, uint32_t* count,
                                    void* stream);
/* Synchronises `stream`; HELIO_ERR_TIMEOUT if a bounded grid barrier gave up,
 * HELIO_ERR_CAPACITY if the active spans exceeded max_spans (outputs incomplete). */
int32_t helio_batch_status(helio_batch* batch, void* stream);
/* Bounds of the batch's device waits (the reference has no device-side waits: its
 * passes are separate dispatches, crates/helio-core/src/graph/execution.rs:504-598).
 * Every grid barrier and the wait for the published views give up after max_polls
 * polls (0 = the default, about 1 s), set the timeout bit and end their CTA; the
 * second launch then returns at once, and helio_batch_status reports
 * HELIO_ERR_TIMEOUT (that execute's outputs are invalid; the next execute starts
 * clean). extra_arrivals > 0 makes every grid barrier wait for that many CTAs beyond
 * the grid, which never arrive: a way to run the bounded waits out in tests (0 in
 * normal use). Applies from the next execute. */
int32_t helio_batch_set_wait_limit(helio_batch* batch, uint32_t max_polls, uint32_t extra_arrivals);
/* Device bytes helio_batch_prepare would allocate for these views of `scene` (a
 * batch grows its buffers and never shrinks them). For admission against a memory budget. */
int32_t helio_batch_estimate_bytes(const helio_batch_config* config, const helio_vg_scene* scene, uint32_t view_count,
                                   const helio_batch_view* views, uint64_t* bytes);
/* Launch-shape autotuner: times helio_batch_execute of the prepared views (on
 * `stream`, `repeats` runs per candidate, median) in two stages: every select_views
 * {8, 16, 24, 32} x CTAs {1, 2, 3} per SM of the first launch (at most the prepared grid),
 * then, at the fastest of those, the meshlet-test launch at 1, 2, ... CTAs per SM (as many
 * as fit). Keeps the fastest in the batch's configuration and reports it. Synchronises
 * `stream`. */
typedef struct helio_batch_tuning {
    uint32_t select_views;
    uint32_t ctas;
    uint32_t candidates;
    uint32_t cull_ctas; /* CTAs of the meshlet-test launch chosen */
    double best_ms;
    double default_ms; /* the configuration before tuning */
} helio_batch_tuning;
int32_t helio_batch_autotune(helio_batch* batch, uint32_t repeats, helio_batch_tuning* out, void* stream);
/* Device bytes the batch holds now. */
int32_t helio_batch_device_bytes(const helio_batch* batch, uint64_t* bytes);
/* Device bytes helio_batch_prepare of these views under `config` would add to what the
 * batch holds now (buffers that must grow, counted whole). */
int32_t helio_batch_growth_bytes(const helio_batch* batch, const helio_batch_config* config,
                                 const helio_vg_scene* scene, uint32_t view_count, const helio_batch_view* views,
                                 uint64_t* bytes);
/* Replaces the configuration the next helio_batch_prepare uses (view limit, span
 * capacity, launch size); the batch must be prepared again before it executes. */
int32_t helio_batch_reconfigure(helio_batch* batch, const helio_batch_config* config);
void helio_batch_destroy(helio_batch* batch);

/* ── Serving: continuous batching of cull requests (no counterpart in the reference) ──
 * Requests name a device-resident scene and carry views; a pump admits them, as batch
 * slots and the HBM budget allow, into batched launches that run concurrently on the
 * slots' streams. The caller supplies the clock (seconds, any origin) so that latency
 * is measured on the caller's timeline: completion time - arrival time. */
typedef struct helio_serve_config {
    uint64_t hbm_budget_bytes;       /* scenes + every slot's batch scratch; 0 = no limit */
    uint32_t slots;                  /* batches in flight at once, each on its own stream: 1..16 */
    uint32_t max_views;              /* views per batch: 1..HELIO_BATCH_MAX_VIEWS */
    uint32_t ctas_per_slot;          /* CTAs of each launch; 0 = the device's co-resident grid / slots */
    uint32_t max_requests_per_batch; /* 0 = no limit */
    uint64_t spans_per_view;         /* active-span capacity per view; 0 = the scene's bound (never overflows) */
} helio_serve_config;

typedef struct helio_serve_request {
    uint32_t scene;                 /* index from helio_serve_add_scene */
    uint32_t view_count;            /* 1..max_views */
    const helio_batch_view* views;  /* copied; the depth buffers must stay valid until completion */
    double arrival_s;               /* arrival time on the caller's clock */
    uint64_t tag;                   /* caller's value, echoed in the completion */
} helio_serve_request;

typedef struct helio_serve_completion {
    uint64_t request;
    uint64_t tag;
    int32_t status;           /* HELIO_OK, the batch's status, or HELIO_ERR_CAPACITY if it can never fit */
    uint32_t batch_requests;  /* requests that shared its launch */
    uint32_t view_count;
    uint32_t reserved;
    double arrival_s, launch_s, done_s; /* caller's clock: arrival, launch, completion seen by a pump */
    double batch_device_ms;             /* device time of the launch that carried it */
    double device_start_ms, device_end_ms; /* that launch's start and end on the device clock (ms since the
                                               server was created): launches of different slots overlap */
} helio_serve_completion;

typedef struct helio_serve_pending {
    uint32_t scene;
    uint32_t view_count;
} helio_serve_pending;

typedef struct helio_serve_stats {
    uint32_t pending;
    uint32_t running;
    uint32_t ctas_per_slot;
    uint32_t reserved;
    uint64_t batches;
    uint64_t bytes_in_use;   /* scenes + slot scratch */
    uint64_t scene_bytes;
} helio_serve_stats;

typedef struct helio_serve helio_serve;
int32_t helio_serve_create(const helio_serve_config* config, helio_serve** out);
/* Registers an uploaded scene (it must outlive the server); its bytes count against the budget. */
int32_t helio_serve_add_scene(helio_serve* server, const helio_vg_scene* scene, uint32_t* scene_id);
int32_t helio_serve_submit(helio_serve* server, const helio_serve_request* request, uint64_t* request_id);
/* One scheduling step at time now_s: retires finished launches (no blocking), then
 * admits and launches batches while a slot and memory are free. *ready = completions
 * waiting to be read. */
int32_t helio_serve_pump(helio_serve* server, double now_s, uint32_t* ready);
/* Moves up to `capacity` completions out, oldest first. */
int32_t helio_serve_completions(helio_serve* server, helio_serve_completion* out, uint32_t capacity, uint32_t* count);
/* Outputs of view `view` of a completed request; valid until helio_serve_release. */
int32_t helio_serve_outputs(const helio_serve* server, uint64_t request_id, uint32_t view,
                            helio_batch_view_outputs* out);
/* Frees a completed request's outputs; a slot is reused once all its requests are released. */
int32_t helio_serve_release(helio_serve* server, uint64_t request_id);
int32_t helio_serve_stats_get(const helio_serve* server, helio_serve_stats* out);
/* The scheduler's batch rule, on the pending queue (oldest first): the oldest request,
 * then later requests of the same scene, in arrival order, that keep the batch within
 * max_views (and max_requests, 0 = no limit). Writes their queue positions. */
int32_t helio_serve_plan_batch(const helio_serve_pending* queue, uint32_t n, uint32_t max_views,
                               uint32_t max_requests, uint32_t* chosen, uint32_t* count);
void helio_serve_destroy(helio_serve* server);

/* ════════════════════════════════════════════════════════════════════════════
 * Per-face shadow cull — ShadowCullPass
 *   (crates/helio-pass-shadow-cull/src/lib.rs:37-328, shaders/shadow_cull.wgsl:1-96)
 *
 * Every movable draw against every dirty shadow face (CSM cascade, spot, point-light
 * cube face): the instance's world sphere (GpuInstanceData.bounds of the draw's
 * first_instance) against the six planes built from the columns of the face's matrix.
 * The visible draws of face f go to face_indirect[f * 4096 + i], in draw order (the
 * reference appends them with an atomic counter, in no defined order), and
 * face_counts[f] counts them all, also past 4096. Faces whose dirty word is zero keep
 * their records; their counts are cleared. Nothing runs, and the counts keep their
 * values, when face_count or draw_count is zero (lib.rs:261-263).
 * ════════════════════════════════════════════════════════════════════════════ */

#define HELIO_SHADOW_MAX_FACES 256u           /* MAX_FACES, lib.rs:37 */
#define HELIO_SHADOW_MAX_DRAWS_PER_FACE 4096u /* MAX_DRAWS_PER_FACE, lib.rs:40 */

typedef struct helio_shadow_cull_inputs {
    const float* shadow_matrices;                    /* device [256][16] column-major (GpuShadowMatrix) */
    const HelioGpuInstanceData* instances;           /* device [instance_count] */
    const HelioDrawIndexedIndirectArgs* src_indirect; /* device [draw_count]: the movable draws */
    const uint32_t* face_dirty;                      /* device [256]: non-zero = cull this face */
    uint32_t instance_count;                         /* draws naming an instance past it are skipped */
    uint32_t draw_count;                             /* shadow_movable_draw_count */
    uint32_t face_count;                             /* shadow_count: 0 skips the pass */
    uint32_t reserved0;
} helio_shadow_cull_inputs;

typedef struct helio_shadow_cull_outputs {
    HelioDrawIndexedIndirectArgs* face_indirect; /* [256 * 4096] */
    uint32_t* face_counts;                       /* [256] */
    uint32_t max_faces;
    uint32_t max_draws_per_face;
} helio_shadow_cull_outputs;

typedef struct helio_shadow_cull_pass helio_shadow_cull_pass;
/* Allocates the 256 x 4096 indirect records (lib.rs:104-117). */
int32_t helio_shadow_cull_create(helio_shadow_cull_pass** out);
/* Binds the inputs (kept until the next prepare) and grows the scratch for draw_count.
 * shadow_matrices and instances must be 16-byte aligned. */
int32_t helio_shadow_cull_prepare(helio_shadow_cull_pass* pass, const helio_shadow_cull_inputs* in);
/* Three launches on `stream`; no allocation, no read-back. */
int32_t helio_shadow_cull_execute(helio_shadow_cull_pass* pass, void* stream);
int32_t helio_shadow_cull_publish(const helio_shadow_cull_pass* pass, helio_shadow_cull_outputs* out);
void helio_shadow_cull_destroy(helio_shadow_cull_pass* pass);

/* Folds a prepared shadow cull pass into a batch: from the next helio_batch_execute on,
 * the pass's test, scan and placement run as units of the batch's own phases (the
 * persistent launch's work queue and barriers) instead of three launches of their own,
 * with the outputs of helio_shadow_cull_execute, read with helio_shadow_cull_publish.
 * The pass stays the caller's: it must stay alive, and its inputs valid, while it is
 * attached; a pass with no face or no draw in use does nothing, as in the standalone
 * form (lib.rs:261-263). pass = NULL detaches. The attached pass's parameters are
 * read at each execute (a CUDA graph captures them, as it captures the views). */
int32_t helio_batch_attach_shadow(helio_batch* batch, helio_shadow_cull_pass* pass);

/* ════════════════════════════════════════════════════════════════════════════
 * VG input producer: rebuild_vg_buffers on the device
 *   (crates/helio/src/scene/virtual_geometry/rebuild.rs:18-58, 98-172)
 *
 * Input, in device memory: a descriptor pool holding the meshlets of every mesh of
 * a library, the library's mesh records, and the scene's dense object slots (each
 * slot's mesh and instance data). Output, in device memory: the VgFrameData arrays
 * of the reference's rebuild (each referenced mesh's descriptors once, in
 * first-reference order; one object and one instance per slot whose mesh exists
 * and has descriptors and LODs; 64-meshlet work items) and max_draw_count, ready
 * for helio_vg_scene_upload / helio_vg_prepare with memory = HELIO_MEM_DEVICE.
 * ════════════════════════════════════════════════════════════════════════════ */

#define HELIO_VG_NO_MESH 0xFFFFFFFFu /* slot_mesh of a free slot (any value >= mesh_count acts alike) */

/* VirtualMeshRecord (crates/helio/src/scene/types.rs:211-236); its descriptors are
 * pool[first_meshlet .. first_meshlet + meshlet_count). 128 bytes. */
typedef struct HelioVgMeshRecord {
    uint32_t first_meshlet;
    uint32_t meshlet_count;
    uint32_t lod_count;
    uint32_t max_meshlet_count;
    float local_bounds[4];
    float lod_errors[HELIO_VG_LOD_LEVELS];
    uint32_t lod_first_meshlets[HELIO_VG_LOD_LEVELS]; /* relative to the mesh's first descriptor */
    uint32_t lod_meshlet_counts[HELIO_VG_LOD_LEVELS];
} HelioVgMeshRecord;

typedef struct helio_vg_build_inputs {
    const HelioGpuMeshletEntry* pool;           /* device */
    const HelioVgMeshRecord* meshes;            /* device */
    const uint32_t* slot_mesh;                  /* device, [slot_count] */
    const HelioGpuInstanceData* slot_instances; /* device, [slot_count] */
    uint32_t pool_count;
    uint32_t mesh_count;
    uint32_t slot_count;
    uint32_t reserved0;
} helio_vg_build_inputs;

typedef struct helio_vg_builder helio_vg_builder;
int32_t helio_vg_builder_create(helio_vg_builder** out);
/* Rebuilds the frame data from `in` on `stream` and waits for it (the totals are
 * read back once to size the outputs). pool, meshes and slot_instances must be
 * 16-byte aligned. HELIO_ERR_INVALID_ARG when a used mesh's
 * descriptor range leaves the pool, or when a count, max_draw_count or an LOD
 * descriptor offset exceeds u32 (where the reference panics); the previous outputs
 * are then gone. The outputs stay valid until the next run or destroy. */
int32_t helio_vg_builder_run(helio_vg_builder* builder, const helio_vg_build_inputs* in, void* stream);
/* The last run's outputs as frame data: device pointers, memory = HELIO_MEM_DEVICE,
 * buffer_version and instance_version = the number of successful runs, no dirty range. */
int32_t helio_vg_builder_frame_data(const helio_vg_builder* builder, helio_vg_frame_data* out);
void helio_vg_builder_destroy(helio_vg_builder* builder);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* HELIO_CULL_H */
