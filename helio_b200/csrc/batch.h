// batch.h — the persistent multi-view visibility kernel (one cooperative launch
// culls every view of a batch against one device-resident scene).
#pragma once

#include "common.cuh"
#include "kernels.h"
#include "shadow_device.cuh"
#include "vg.h"

namespace helio {

constexpr uint32_t kBatchMaxViews = 128;
constexpr uint32_t kBatchThreads = 256;
constexpr uint32_t kBatchChunk = 256;  // objects per select unit and per count chunk

// Per view, in device memory; filled by the host except where noted. 16-byte
// aligned: the camera matrices are read with 128-bit loads.
struct alignas(16) BatchViewDev {
    HelioGpuCameraUniforms camera;
    HizJob hiz;
    uint32_t width, height;
    uint32_t hiz_mip_count;  // mip_levels(width, height), unclamped (rendering.rs:828-829)
    float lod_threshold_px;
    uint32_t capacity;       // publication capacity of this view
    uint32_t pad;
    HelioDrawIndexedIndirectArgs* indirect;  // [capacity]
    HelioGpuVgDraw* draws;                   // [capacity]
    uint32_t* counters;                      // [16]; layout of the VG counters
    float reject_box[6];  // written by phase 0: x/y/z lower bounds, then upper bounds
    uint32_t hiz_pair_begin;  // first Hi-Z unit (pair of tiles) of this view in the batch
    uint32_t pad2;
};

static_assert(sizeof(BatchViewDev) % 16 == 0, "view table entries stay 16-byte aligned");

// An active span: up to 64 meshlets of the selected LOD of one object in one view.
// x = first meshlet, y = n | lod << 8 | view << 16, z = instance, w = object.
using ActiveSpan = uint4;

__host__ __device__ inline uint32_t span_n(const ActiveSpan& s) { return s.y & 0x7Fu; }
__host__ __device__ inline uint32_t span_lod(const ActiveSpan& s) { return (s.y >> 8) & 0xFu; }
__host__ __device__ inline uint32_t span_view(const ActiveSpan& s) { return s.y >> 16; }

enum : uint32_t { kBatchErrTimeout = 1u, kBatchErrSpanCapacity = 2u };

struct BatchParams {
    VgSceneDev scene;
    const uint32_t* scene_bounds;  // [2] launch_scene_bounds output
    BatchViewDev* views;      // [view_count]
    CullView* cviews;         // [view_count], written by phase 0
    uint8_t* lod;             // [view_count * lod_pitch]: LOD + 1 per (view, object), 0 = culled
    uint32_t lod_pitch;       // bytes per view row: object_count rounded up to kBatchChunk
    uint32_t view_count;
    uint32_t select_views;    // views per select unit, 1..32
    uint32_t object_chunks;   // ceil(object_count / kBatchChunk)
    uint32_t hiz_tiles;       // Hi-Z units of all views: pairs of horizontally consecutive tiles
    uint32_t* barrier;        // [2] arrival count (zero before the launch), generation
    uint32_t spin_limit;      // polls before a bounded wait gives up (kSpinLimit by default)
    uint32_t barrier_extra;   // arrivals a grid barrier waits for beyond the grid (0; tests only)
    uint32_t* error;          // [1] kBatchErr* bits, zero before the launch
    uint32_t* work;           // [1] phase-1 work queue head, zero before the launch
    uint32_t* setup_done;     // [1] views whose constants are published, zero before the launch
    uint32_t* expand_work;    // [1] expansion work queue head, zero before the launch
    uint32_t* test_work;      // [1] meshlet-test work queue head, zero before the launch
    uint32_t* chunk_counts;   // [view_count * object_chunks] active spans per (view, chunk)
    uint32_t* chunk_vis;      // [view_count * object_chunks] visible objects per (view, chunk)
    uint16_t* vis_list;       // [view_count * object_chunks * kBatchChunk] per (view, chunk): its
                              // visible objects in object order, slot | LOD << 8
    uint32_t* chunk_offs;     // [view_count * object_chunks + 1]
    uint32_t* seg_totals;     // [gridDim.x]
    uint32_t* view_span_start;  // [view_count + 1] first span of each view (views padded to 32)
    ActiveSpan* spans;        // [span_capacity]
    uint32_t span_capacity;   // multiple of 32
    uint32_t* group_counts;   // [span_capacity / 32] visible meshlets per group of 32 spans
    uint32_t* group_offs;     // [span_capacity / 32 + 1]
    uint32_t* group_bits;     // [span_capacity / 32 * kWindowsPerWarp] window ballots
    uint32_t* span_vis;       // [span_capacity * 2] per-span visibility words, or null
    unsigned long long* phase_ns;  // [kBatchPhaseStamps] %globaltimer at launch and after each phase
    // An attached per-face shadow cull (helio_batch_attach_shadow): its test stage runs
    // as the first shadow_blocks units of phase 1, its scan in phase 2 and its placement
    // in phase 3. shadow_blocks = 0: none.
    ShadowDev shadow;
    uint32_t shadow_blocks;
    uint32_t* shadow_work;    // [1] placement queue head of the shadow cull, zero before the launch
};

// [0..7] phase boundaries, [8] / [9] largest per-CTA time spent on Hi-Z tiles /
// object chunks in phase 1 (ns).
constexpr uint32_t kBatchPhaseStamps = 10;

// Bounds over the valid objects of a scene (an object with lod_count > 0, an
// instance in range and a valid transform), as float bits, for the per-view reject
// boxes: bounds[0] = largest world radius max(local_radius * max_scale, 0),
// bounds[1] = largest |c.x| + |c.y| + |c.z| of a world centre c (computed exactly as
// the select computes them). `bounds` must be zero before the launch.
cudaError_t launch_scene_bounds(const VgSceneDev& scene, uint32_t* bounds, cudaStream_t stream);

// Packs the published draws of every view (min(counters[0], capacity) each) into
// one pair of arrays, view after view; offsets[v] = first draw of view v, offsets[V] =
// the total (entries past `capacity` are not written).
cudaError_t launch_pack_draws(const BatchViewDev* views, uint32_t view_count, HelioDrawIndexedIndirectArgs* indirect,
                              HelioGpuVgDraw* draws, uint32_t* offsets, uint64_t capacity, cudaStream_t stream);

// Dynamic shared memory of the persistent kernel (bytes).
size_t batch_dynamic_smem();
// Launches the two cooperative kernels of a batch on `stream`: phases 0..3 with
// `grid` CTAs, then phases 4..6 with `cull_grid` CTAs (each grid all co-resident).
cudaError_t launch_batch(const BatchParams& p, uint32_t grid, uint32_t cull_grid, cudaStream_t stream);
// Largest co-resident grids for this device (phases 0..3, phases 4..6).
uint32_t batch_max_grid();
uint32_t batch_cull_max_grid();

}  // namespace helio
