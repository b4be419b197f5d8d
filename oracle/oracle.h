/*
 * oracle.h — CPU restatement of Helio's GPU visibility path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is what the CUDA path is compared with: it
 * may be loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU
 * baseline / reference arm, and by nothing else. The product library
 * (helio_b200/lib/libhelio_cull.so) never links, loads or calls it.
 *
 * Every function restates one reference shader entry point or Rust helper, in
 * the WGSL operation order, with IEEE binary32 arithmetic and no contraction
 * (built with -O2 -ffp-contract=off). Citations are per function in oracle.cpp.
 *
 * Parity status: the reference's shaders cannot execute on either machine
 * (no Rust toolchain, browser-only wgpu, no graphics stack). The restatement is
 * pinned against every known-answer test that the reference's own test files
 * hold for this path (tests/golden/reference_kats.json); end-to-end execution of
 * the WGSL itself is unpinned.
 */
#ifndef HELIO_ORACLE_H
#define HELIO_ORACLE_H

#include <stdint.h>
#include "../include/helio_cull.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Decision statistics gathered while culling (for the 1e-6 relative margin band
 * and for the algorithmic byte count). */
typedef struct oracle_stats {
    uint64_t objects_tested;
    uint64_t objects_visible;
    uint64_t meshlets_tested;      /* meshlets of a selected LOD of a visible object */
    uint64_t meshlets_cone_loaded; /* passed frustum (cone inputs needed) */
    uint64_t meshlets_visible;
    uint64_t marginal_decisions;   /* comparisons whose operands lie within 1e-6 relative */
    uint64_t marginal_meshlets;    /* meshlets with at least one marginal decision */
    uint64_t marginal_objects;
} oracle_stats;

uint32_t oracle_mip_levels(uint32_t w, uint32_t h);
uint32_t oracle_ceil_log2(float d);
void oracle_extract_frustum_planes(const float vp[16], float planes[24]);
void oracle_instance_cull_data(const HelioGpuInstanceData* inst, uint32_t n,
                               HelioInstanceCullData* out);

/* Builds every level of the pyramid. levels[l] must hold width[l]*height[l]
 * floats (dense); level 0 receives the copy of depth. Returns mip count. */
uint32_t oracle_hiz_build(const float* depth, uint32_t w, uint32_t h, uint32_t pitch,
                          float* const* levels);

void oracle_indirect_dispatch(const HelioGpuCameraUniforms* cam, const float planes[24],
                              const HelioGpuInstanceData* inst, const HelioGpuDrawCall* dc,
                              const HelioGpuInstanceAabb* aabb, uint32_t draw_count,
                              uint32_t instance_count, uint32_t* indirect, uint32_t* stats);

void oracle_occlusion_cull(const HelioGpuCameraUniforms* cam, uint32_t screen_w,
                           uint32_t screen_h, const helio_hiz_pyramid* hiz,
                           const HelioGpuInstanceData* inst, const HelioGpuDrawCall* dc,
                           uint32_t draw_count, uint32_t instance_count, uint32_t* indirect,
                           uint32_t* stats, oracle_stats* st);

/* oracle_occlusion_cull with the static Hi-Z branch (occlusion_cull.wgsl:222-259) when
 * static_hiz is non-null (its texels are host memory here); the library's filter rule
 * (helio_occlusion_cull_set_static_hiz) is restated exactly. */
void oracle_occlusion_cull_static(const HelioGpuCameraUniforms* cam, uint32_t screen_w,
                                  uint32_t screen_h, const helio_hiz_pyramid* hiz,
                                  const HelioGpuInstanceData* inst, const HelioGpuDrawCall* dc,
                                  uint32_t draw_count, uint32_t instance_count, uint32_t* indirect,
                                  uint32_t* stats, oracle_stats* st, const helio_static_hiz* static_hiz);

/* Uniforms of the VG cull (CullUniforms, rendering.rs:828-859). */
typedef struct oracle_vg_uniforms {
    uint32_t object_count;
    uint32_t screen_width;
    uint32_t screen_height;
    uint32_t hiz_mip_count;
    uint32_t draw_capacity;
    float lod_error_threshold_px;
    uint32_t work_item_count;
    uint32_t meshlet_count;
    uint32_t instance_count;
    uint32_t counter_count;
} oracle_vg_uniforms;

/* cs_select_objects: writes selected[i] = LOD + 1 (0 = culled) and the LOD
 * histogram / max-LOD counters when counter_count >= 11. */
void oracle_vg_select(const HelioGpuCameraUniforms* cam, const oracle_vg_uniforms* u,
                      const HelioGpuVgObject* objects, const HelioGpuInstanceData* inst,
                      const HelioInstanceCullData* cull, uint32_t* selected, uint32_t* counters,
                      oracle_stats* st, int threads);

/* cs_cull_meshlets in the canonical (work item, lane) order. visibility receives
 * 2 words per work item. counters[0] = attempted, counters[1] = rejected. */
void oracle_vg_cull(const HelioGpuCameraUniforms* cam, const oracle_vg_uniforms* u,
                    const HelioGpuMeshletEntry* meshlets, const HelioGpuVgObject* objects,
                    const uint32_t* selected, const HelioGpuInstanceData* inst,
                    const HelioInstanceCullData* cull, const HelioGpuVgWorkItem* items,
                    const helio_hiz_pyramid* hiz, HelioDrawIndexedIndirectArgs* indirect,
                    HelioGpuVgDraw* draws, uint32_t* counters, uint32_t* visibility,
                    oracle_stats* st, int threads);

/* rebuild_vg_buffers (crates/helio/src/scene/virtual_geometry/rebuild.rs:18-58,
 * 98-172) over a mesh library and dense object slots, sequentially in the reference's
 * order. counts receives {descriptors, objects, work items, max_draw_count}; null
 * output arrays skip the writes (a counting pass). Returns 0, or 1 where the
 * reference panics (a count, max_draw_count or an LOD offset beyond u32) or a used
 * mesh's descriptors leave the pool. */
int oracle_vg_rebuild(const HelioGpuMeshletEntry* pool, uint32_t pool_count, const HelioVgMeshRecord* meshes,
                      uint32_t mesh_count, const uint32_t* slot_mesh, const HelioGpuInstanceData* slot_instances,
                      uint32_t slot_count, HelioGpuMeshletEntry* out_meshlets, HelioGpuVgObject* out_objects,
                      HelioGpuInstanceData* out_instances, HelioGpuVgWorkItem* out_items, uint64_t counts[4]);

/* ShadowCullPass::execute + shadow_cull.wgsl (crates/helio-pass-shadow-cull/src/lib.rs:
 * 257-328, shaders/shadow_cull.wgsl:49-96) over 256 faces: for every face whose dirty
 * word is non-zero, the draws whose instance sphere passes the face's six column-built
 * planes, in draw order (the reference appends with atomics, so its order is not
 * defined), copied to dst[face * max_per_face + i] for i < max_per_face;
 * face_counts[face] counts them all. A draw whose first_instance is not below
 * instance_count is skipped. Returns 0 without touching anything when face_count or
 * draw_count is zero (the reference returns before clearing the counts), else 1. */
int oracle_shadow_cull(const float* matrices, const HelioGpuInstanceData* instances, uint32_t instance_count,
                       const HelioDrawIndexedIndirectArgs* src, uint32_t draw_count, const uint32_t* face_dirty,
                       uint32_t face_count, uint32_t max_per_face, HelioDrawIndexedIndirectArgs* dst,
                       uint32_t* face_counts);

/* Single decisions, for the reference's known-answer tests. */
/* sphere_visible (vg_cull.wgsl:126-133) against six given planes. */
int oracle_sphere_visible(const float planes[24], const float center[3], float radius);
/* select_object_lod (crates/helio-pass-virtual-geometry/src/lib.rs:205-234 / vg_cull.wgsl:323-337). */
uint32_t oracle_select_lod(const float errors[8], uint32_t lod_count, float max_scale, float focal_px,
                           float closest, float max_error_px);
/* Cone rejection of cull_meshlet (vg_cull.wgsl:174-181) with a world-space axis. */
int oracle_cone_reject(const float camera[3], const float apex[3], const float axis_ws[3], float cutoff);
/* Hi-Z occlusion decision: near_z > hiz + 1/65536 (occlusion_cull.wgsl:207-208). */
int oracle_hiz_occludes(float near_z, float hiz);

#ifdef __cplusplus
}
#endif

#endif
