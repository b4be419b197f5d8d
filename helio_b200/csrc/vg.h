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

// Per-object result of the select stage: selected LOD range of the object.
// x = first meshlet of the LOD, y = meshlets in it, z = instance index, w = LOD + 1 (0 = culled).
using SelRecord = uint4;

struct VgSelectParams {
    VgSceneDev scene;
    const HelioGpuCameraUniforms* camera;
    SelRecord* sel;     // [object_count]
    uint32_t* counters; // [counter_count]
    uint32_t counter_count;
    uint32_t screen_height;
    float lod_threshold_px;
    uint32_t write_reserved;  // also store LOD + 1 into objects[i].reserved
};

// Scratch of one cull launch, cleared before it: [counters..][tile ticket][error][look-back states].
struct VgCullScratch {
    uint32_t* tile_counter;
    uint32_t* error_word;
    unsigned long long* lookback;  // [num_tiles]
};

struct VgCullParams {
    VgSceneDev scene;
    const HelioGpuCameraUniforms* camera;
    const SelRecord* sel;
    HelioDrawIndexedIndirectArgs* indirect;
    HelioGpuVgDraw* draws;
    uint32_t* counters;
    uint32_t* visibility;  // [2 * work_item_count] or null
    VgCullScratch scratch;
    HizView hiz;
    uint32_t capacity;
    uint32_t screen_height;
    uint32_t hiz_mip_count;  // mip_levels(width, height), unclamped (rendering.rs:828-829)
    uint32_t num_tiles;
};

constexpr uint32_t kCullWarps = 4;
constexpr uint32_t kCullItemsPerTile = kCullWarps * 32;

inline uint32_t vg_cull_tiles(uint32_t work_items) { return (work_items + kCullItemsPerTile - 1) / kCullItemsPerTile; }

void launch_pack_meshlets(const HelioGpuMeshletEntry* aos, uint32_t n, float4* bounds, float4* cone, float4* axis,
                          uint4* draw, cudaStream_t stream);
void launch_instance_cull_data(const HelioGpuInstanceData* inst, uint32_t n, HelioInstanceCullData* out,
                               cudaStream_t stream);
void launch_vg_select(const VgSelectParams& p, cudaStream_t stream);
void launch_vg_cull(const VgCullParams& p, cudaStream_t stream);

}  // namespace helio
