// vg.h — launch parameters of the virtual-geometry kernels.
#pragma once

#include "common.cuh"

namespace helio {

// Device-resident scene in the layout the cull kernels read. Meshlet descriptors
// are split into four 16-byte streams so each warp load is one contiguous 512 B.
struct VgSceneDev {
    const float4* m_bounds;  // center.xyz, radius
    const float4* m_cone;    // cone_apex.xyz, cone_cutoff
    const float4* m_axis;    // cone_axis.xyz, lod_error
    const uint4* m_draw;     // first_index, index_count, vertex_offset, instance_index
    HelioGpuVgObject* objects;
    const HelioGpuInstanceData* instances;
    const HelioInstanceCullData* cull;
    const HelioGpuVgWorkItem* items;
    uint32_t meshlet_count;
    uint32_t object_count;
    uint32_t instance_count;
    uint32_t work_item_count;
};

// View constants shared by every CTA of the select / cull kernels, computed once
// per launch by vg_view_setup_kernel from the device camera (vg_cull.wgsl:266-280
// planes; fields of GpuCameraUniforms) and the Hi-Z pyramid descriptor.
struct CullView {
    Planes planes;
    Mat4 vp;
    float4 pos_near;
    float p00, p11;
    float focal;      // |proj[1][1]| * screen_height * 0.5 (vg_cull.wgsl:321-322)
    float lod_threshold_px;
    HizView hiz;
    uint32_t screen_height;
    uint32_t hiz_mip_count;
    uint32_t pad[2];
};
static_assert(sizeof(CullView) % 16 == 0, "CullView is copied as 16-byte words");

// Per-object result of the select stage: selected LOD range of the object.
// x = first meshlet of the LOD, y = meshlets in it, z = instance index, w = LOD + 1 (0 = culled).
using SelRecord = uint4;

// Inputs of vg_view_setup_kernel: computes *out from the device camera.
struct ViewSetupParams {
    const HelioGpuCameraUniforms* camera;
    CullView* out;
    HizView hiz;
    uint32_t screen_height;
    uint32_t hiz_mip_count;
    float lod_threshold_px;
};

struct VgSelectParams {
    VgSceneDev scene;
    const CullView* view;
    SelRecord* sel;     // [object_count]
    uint32_t* counters; // [counter_count]
    uint32_t counter_count;
    uint32_t write_reserved;  // also store LOD + 1 into objects[i].reserved
    // compute_view = 1: every block builds the view constants from `setup` itself (the
    // view-setup launch folded in) and block 0 publishes them to setup.out (== view) for
    // the later kernels; 0: the blocks read them from `view`.
    uint32_t compute_view;
    ViewSetupParams setup;
};

constexpr uint32_t kCullWarps = 8;                       // warps per CTA tile
constexpr uint32_t kWindowsPerWarp = 64;                 // 32 items x 64 meshlets / 32 lanes
constexpr uint32_t kCullTargetWarps = 148u * 32u;        // warps that keep every SM busy

// Scratch of one cull launch. tile_counts must be zero before the test kernel
// (it accumulates per-warp counts); warp_counts and bits are written before
// they are read.
struct VgCullScratch {
    uint32_t* tile_counts;  // [num_tiles] visible meshlets per tile
    uint32_t* warp_counts;  // [num_tiles * kCullWarps]
    uint32_t* bits;         // [num_tiles * kCullWarps * kWindowsPerWarp] window ballots
};

inline size_t vg_cull_scratch_words(uint32_t tiles) {
    return (size_t)tiles * (1 + kCullWarps + (size_t)kCullWarps * kWindowsPerWarp);
}

struct VgCullParams {
    VgSceneDev scene;
    const CullView* view;
    const SelRecord* sel;
    HelioDrawIndexedIndirectArgs* indirect;
    HelioGpuVgDraw* draws;
    uint32_t* counters;
    uint32_t* visibility;  // [2 * work_item_count] or null
    VgCullScratch scratch;
    uint32_t capacity;
    uint32_t num_tiles;
    uint32_t items_per_warp;  // 1, 2, 4, ..., 32: warp w takes work items [w * ipw, (w + 1) * ipw)
};

// Work items per warp of the single-view cull: 32 (one per lane) when the scene has
// enough items to fill every SM with warps, fewer for small scenes, so that their
// windows spread over more warps instead of running in series on few. The draw order
// is the item order for every choice.
inline uint32_t vg_cull_items_per_warp(uint32_t work_items) {
    uint32_t ipw = 32;
    while (ipw > 1 && (uint64_t)work_items < (uint64_t)kCullTargetWarps * ipw) ipw >>= 1;
    return ipw;
}
inline uint32_t vg_cull_tiles(uint32_t work_items, uint32_t items_per_warp) {
    const uint32_t per_tile = kCullWarps * items_per_warp;
    return (work_items + per_tile - 1) / per_tile;
}

void launch_pack_meshlets(const HelioGpuMeshletEntry* aos, uint32_t n, float4* bounds, float4* cone, float4* axis,
                          uint4* draw, cudaStream_t stream);
void launch_instance_cull_data(const HelioGpuInstanceData* inst, uint32_t n, HelioInstanceCullData* out,
                               cudaStream_t stream);
void launch_vg_view_setup(const ViewSetupParams& p, cudaStream_t stream);
void launch_vg_select(const VgSelectParams& p, cudaStream_t stream);
// Test kernel then emit kernel on `stream`.
cudaError_t launch_vg_cull(const VgCullParams& p, cudaStream_t stream);

}  // namespace helio
