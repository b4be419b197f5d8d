// instance_cull.h — launch parameters of the per-draw culls.
#pragma once

#include "common.cuh"

namespace helio {

struct InstanceCullParams {
    const HelioGpuCameraUniforms* camera;  // device
    const HelioGpuInstanceData* instances;
    const HelioGpuDrawCall* draw_calls;
    const HelioGpuInstanceAabb* aabbs;
    uint32_t* indirect;  // draw_count x 5
    uint32_t* stats;     // 8
    float planes[24];    // CPU-extracted (crates/helio-pass-indirect-dispatch/src/lib.rs:271-300)
    HizView hiz;
    uint32_t draw_count;
    uint32_t instance_count;  // draws whose first_instance >= instance_count are frustum-culled
    uint32_t screen_w, screen_h;
    uint32_t hiz_mip_count;  // mip_levels(screen_w, screen_h), unclamped (occlusion-cull lib.rs:303)
    // Static Hi-Z (occlusion_cull.wgsl:222-259); off when static_texels is null.
    const float* static_texels;  // level 0: dims[0] x dims[1] x (dims[2] * 6), x fastest
    uint32_t static_dims[3];
    float static_min[3], static_max[3];
};

void launch_instance_cull(const InstanceCullParams& p, bool frustum, bool occlusion, cudaStream_t stream);

}  // namespace helio
