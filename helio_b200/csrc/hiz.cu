// hiz.cu — fused multi-level Hi-Z pyramid build (HiZBuildPass).
//
// The reference runs one depth-copy dispatch and then mip_count-1 dispatches
// separated by barriers (crates/helio-pass-hiz/src/lib.rs:503-531). Here one launch
// builds every level of one or several views: one CTA per 64x64 tile of level 0
// (hiz_tile.cuh), and the last CTA of each view finishes the levels above 6.

#include "common.cuh"
#include "hiz_tile.cuh"
#include "kernels.h"

namespace helio {

namespace {

// `single` is used when jobs == nullptr (one view, job passed by value);
// otherwise jobs[] holds n_jobs views. The job is copied to shared memory so
// that its level arrays can be indexed at run time.
__global__ void __launch_bounds__(256) hiz_build_kernel(HizJob single, const HizJob* __restrict__ jobs,
                                                        uint32_t n_jobs, uint32_t* tickets) {
    __shared__ float s_m3[8][9];
    __shared__ HizJob s_J;
    __shared__ uint32_t s_job;
    const uint32_t tile = blockIdx.x;
    if (threadIdx.x == 0) {
        uint32_t lo = 0;
        if (jobs) {
            uint32_t hi = n_jobs - 1;
            while (lo < hi) {  // last job with tile_begin <= tile
                uint32_t mid = (lo + hi + 1) >> 1;
                if (jobs[mid].tile_begin <= tile) lo = mid;
                else hi = mid - 1;
            }
            s_J = jobs[lo];
        } else {
            s_J = single;
        }
        s_job = lo;
    }
    __syncthreads();
    hiz_tile(s_J, s_job, tile - s_J.tile_begin, tickets, s_m3);
}

}  // namespace

size_t hiz_layout(uint32_t width, uint32_t height, uint32_t depth_pitch, bool copy_mip0, HizJob* job) {
    uint32_t m = width > height ? width : height, bits = 0;
    while (m) {
        ++bits;
        m >>= 1;
    }
    uint32_t mips = bits < 1 ? 1 : bits;
    if (mips > HELIO_HIZ_MAX_MIPS) mips = HELIO_HIZ_MAX_MIPS;
    *job = HizJob{};
    job->mip_count = mips;
    job->depth_pitch = depth_pitch ? depth_pitch : width;
    job->copy_mip0 = copy_mip0 ? 1u : 0u;
    job->tiles_x = (width + kHizTile - 1) / kHizTile;
    job->tiles_y = (height + kHizTile - 1) / kHizTile;
    size_t total = 0;
    for (uint32_t l = 0; l < mips; ++l) {
        uint32_t w = width >> l, h = height >> l;
        job->lw[l] = w ? w : 1;
        job->lh[l] = h ? h : 1;
        job->lpitch[l] = (job->lw[l] + 3u) & ~3u;  // 16-byte rows
        if (l == 0 && !copy_mip0) {
            job->lpitch[0] = job->depth_pitch;
            continue;
        }
        total += (size_t)job->lpitch[l] * job->lh[l];
    }
    return total;
}

void hiz_assign(HizJob* job, const float* depth, float* levels_base) {
    job->depth = depth;
    size_t off = 0;
    for (uint32_t l = 0; l < job->mip_count; ++l) {
        if (l == 0 && !job->copy_mip0) {
            job->levels[0] = const_cast<float*>(depth);
            continue;
        }
        job->levels[l] = levels_base + off;
        off += (size_t)job->lpitch[l] * job->lh[l];
    }
}

void launch_hiz_build(const HizJob* jobs_dev, uint32_t n_jobs, uint32_t total_tiles, uint32_t* tickets_dev,
                      cudaStream_t stream) {
    if (total_tiles == 0 || n_jobs == 0) return;
    helio_launch_begin("hiz_build", stream);
    hiz_build_kernel<<<total_tiles, 256, 0, stream>>>(HizJob{}, jobs_dev, n_jobs, tickets_dev);
    helio_launch_end(stream);
}

void launch_hiz_build_single(const HizJob& job, uint32_t* ticket_dev, cudaStream_t stream) {
    const uint32_t tiles = job.tiles_x * job.tiles_y;
    if (tiles == 0) return;
    helio_launch_begin("hiz_build", stream);
    hiz_build_kernel<<<tiles, 256, 0, stream>>>(job, nullptr, 1u, ticket_dev);
    helio_launch_end(stream);
}

}  // namespace helio
