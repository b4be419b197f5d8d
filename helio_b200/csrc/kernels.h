// kernels.h — host-side launch interface of the CUDA kernels (no torch types).
#pragma once

#include <cstdint>
#include <cuda.h>  // CUtensorMap
#include <cuda_runtime.h>

#include "../../include/helio_cull.h"

namespace helio {

// ── Hi-Z ─────────────────────────────────────────────────────────────────────
// One pyramid build job (one view). Level l is lw[l] x lh[l] floats with row
// pitch lpitch[l]; levels[0] may be the depth buffer itself (copy_mip0 = 0).
struct HizJob {
    const float* depth;
    float* levels[HELIO_HIZ_MAX_MIPS];
    uint32_t lw[HELIO_HIZ_MAX_MIPS];
    uint32_t lh[HELIO_HIZ_MAX_MIPS];
    uint32_t lpitch[HELIO_HIZ_MAX_MIPS];
    uint32_t depth_pitch;
    uint32_t mip_count;
    uint32_t tiles_x;
    uint32_t tiles_y;
    uint32_t tile_begin;  // first flat tile of this job in a multi-job launch
    uint32_t copy_mip0;
    uint32_t pad[2];
};

constexpr uint32_t kHizTile = 64;  // mip-0 pixels per CTA tile side (levels 1..6 per tile)

// Fills the level geometry of a job for a width x height pyramid. `levels_base`
// receives levels 1.. (and level 0 when copy_mip0); returns floats needed.
size_t hiz_layout(uint32_t width, uint32_t height, uint32_t depth_pitch, bool copy_mip0,
                  HizJob* job);
void hiz_assign(HizJob* job, const float* depth, float* levels_base);

// jobs_dev: n_jobs jobs in device memory, tile_begin ascending; tickets_dev:
// n_jobs zero-initialised counters (left zero after the launch).
void launch_hiz_build(const HizJob* jobs_dev, uint32_t n_jobs, uint32_t total_tiles,
                      uint32_t* tickets_dev, cudaStream_t stream);
// One view, job passed by value (tile_begin must be 0).
void launch_hiz_build_single(const HizJob& job, uint32_t* ticket_dev, cudaStream_t stream);

// Tensor map of a 2-D float array (width x height, row pitch in floats) read in boxes of
// box_w x box_h; false when TMA cannot address it (base not 16-byte aligned, pitch not a
// multiple of 4 floats) or the driver offers no encoder.
bool encode_float_tile_map(CUtensorMap* map, const float* base, uint32_t width, uint32_t height, uint32_t pitch,
                           uint32_t box_w, uint32_t box_h);
// One view whose level 0 is addressed by `src` (encode_float_tile_map of job.depth,
// 64x64 boxes): a persistent grid with TMA tile loads. error_dev[0] gets kDevTimeout if
// a tile never lands (bounded wait).
void launch_hiz_build_tma(const CUtensorMap& src, const HizJob& job, uint32_t* ticket_dev, uint32_t* error_dev,
                          cudaStream_t stream);

}  // namespace helio
