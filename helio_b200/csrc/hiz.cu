// hiz.cu — fused multi-level Hi-Z pyramid build (HiZBuildPass).
//
// The reference runs one depth-copy dispatch and then mip_count-1 dispatches
// separated by barriers (crates/helio-pass-hiz/src/lib.rs:503-531). Here one launch
// builds every level of one or several views: each 64x64 tile of level 0 is reduced
// by one CTA to levels 1..6 (hiz_tile.cuh), and the CTA of the last tile of each view
// finishes the levels above 6. A single view whose depth TMA can address (16-byte
// aligned, row pitch a multiple of 4 floats) runs the persistent form below, which
// streams the tiles into shared memory with TMA loads; other inputs and multi-view
// launches read the tile with 128-bit loads.

#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled

#include <algorithm>
#include <mutex>

#include "common.cuh"
#include "hiz_tile.cuh"
#include "kernels.h"
#include "tma.cuh"

namespace helio {

namespace {

// `single` is used when jobs == nullptr (one view, job passed by value);
// otherwise jobs[] holds n_jobs views. The job is copied to shared memory so
// that its level arrays can be indexed at run time.
__global__ void __launch_bounds__(256, 3) hiz_build_kernel(HizJob single, const HizJob* __restrict__ jobs,
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

// Persistent form for one view whose level 0 TMA can address (4 CTAs per SM): CTA b takes
// tiles b, b + G, b + 2G, ... Thread 0 keeps kHizStages 64x64 tiles in flight (TMA loads into
// shared memory, one mbarrier per stage), so each SM keeps several hundred KB of
// depth reads outstanding while its warps reduce the tile that has landed. The
// reduction of a tile is the same as in hiz_build_kernel (hiz_tile.cuh), reading the
// thread's 4x4 block from shared memory instead of global memory.
constexpr int kHizStages = 3;
constexpr uint32_t kHizTileBytes = kHizTile * kHizTile * 4u;
constexpr uint32_t kHizWaitPolls = 1u << 20;  // bounded wait for a landed tile
static_assert(2 * kHizTailBuf <= kHizStages * kHizTile * kHizTile, "the tail's two level buffers fit the staging");

__global__ void __launch_bounds__(256, 4) hiz_build_tma_kernel(const __grid_constant__ CUtensorMap src,
                                                               const __grid_constant__ HizJob J, uint32_t* ticket,
                                                               uint32_t* error) {
    extern __shared__ __align__(128) unsigned char s_raw[];  // kHizStages x 64 x 64 floats (+128 B)
    __shared__ __align__(8) uint64_t s_full[kHizStages];
    // TMA writes its boxes at 128-byte aligned shared addresses.
    float* s_stage = reinterpret_cast<float*>(s_raw + ((128u - (smem_u32(s_raw) & 127u)) & 127u));
    __shared__ float s_m3[8][9];
    const uint32_t tiles = J.tiles_x * J.tiles_y, G = gridDim.x;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    auto issue = [&](uint32_t t, int s) {
        const uint32_t ty = t / J.tiles_x, tx = t - ty * J.tiles_x;
        mbar_arrive_expect_tx(&s_full[s], kHizTileBytes);
        tma_load_2d(s_stage + s * (kHizTile * kHizTile), &src, &s_full[s], (int32_t)(tx * kHizTile),
                    (int32_t)(ty * kHizTile));
    };
    if (tid == 0) {
        for (int s = 0; s < kHizStages; ++s) mbar_init(&s_full[s], 1u);
        mbar_init_fence();
        for (int s = 0; s < kHizStages; ++s)
            if (blockIdx.x + s * G < tiles) issue(blockIdx.x + s * G, s);
    }
    __syncthreads();
    const int tx4 = lane & 15, ty4 = warp * 2 + (lane >> 4);
    uint32_t k = 0;
    for (;; ++k) {
        const uint32_t t = blockIdx.x + k * G;
        if (t >= tiles) break;
        const int s = (int)(k % kHizStages);
        const bool landed = mbar_wait_bounded(&s_full[s], (k / kHizStages) & 1u, kHizWaitPolls);
        if (__syncthreads_or(!landed)) {
            if (tid == 0) atomicOr(error, kDevTimeout);
            break;
        }
        float v[4][4];
        const float* tile = s_stage + s * (kHizTile * kHizTile) + (4 * ty4) * kHizTile + 4 * tx4;
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            const float4 q = *reinterpret_cast<const float4*>(tile + r * kHizTile);
            v[r][0] = q.x;
            v[r][1] = q.y;
            v[r][2] = q.z;
            v[r][3] = q.w;
        }
        __syncthreads();  // stage s is read (and warp 0 is done with the last tile's s_m3)
        if (tid == 0 && t + kHizStages * G < tiles) issue(t + kHizStages * G, s);
        hiz_tile_copy0(J, t, v);
        if (J.mip_count <= 1) continue;
        hiz_tile_levels123(J, t, v, s_m3);
        if (J.mip_count <= 3) continue;
        __syncthreads();
        if (warp == 0) hiz_tile_levels456(J, t, s_m3);
    }
    // A wait that gave up leaves later loads in flight: wait for them (bounded) before
    // the tail reuses the staging buffers or the CTA's shared memory is released.
    if (tid == 0) {
        for (uint32_t j = k; j < k + kHizStages; ++j)
            if (blockIdx.x + j * G < tiles)
                mbar_wait_bounded(&s_full[j % kHizStages], (j / kHizStages) & 1u, kHizWaitPolls);
    }
    // Levels 7..: every CTA takes one ticket after its last tile (one fence per CTA,
    // not per tile: warp 0 wrote all of this CTA's level-6 texels); the CTA that takes
    // the last ticket builds the tail with all 8 warps.
    if (J.mip_count > 7) {
        __shared__ uint32_t s_last;
        if (tid == 0) {
            __threadfence();
            const uint32_t last = (atomicAdd(ticket, 1u) + 1u == G) ? 1u : 0u;
            if (last) *ticket = 0u;  // every other CTA has taken its ticket
            s_last = last;
        }
        __syncthreads();
        if (s_last) {
            __threadfence();
            // Every tile has landed and been read: the staging buffers hold the tail's levels.
            hiz_tail_in<8, 2>(J, s_stage, s_stage + kHizTailBuf);
        }
    }
}

PFN_cuTensorMapEncodeTiled tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

}  // namespace

bool encode_float_tile_map(CUtensorMap* map, const float* base, uint32_t width, uint32_t height, uint32_t pitch,
                           uint32_t box_w, uint32_t box_h) {
    if (!base || ((reinterpret_cast<uintptr_t>(base) & 15u) != 0u) || (pitch & 3u) != 0u || width == 0 ||
        height == 0 || box_w == 0 || box_w > 256 || box_h == 0 || box_h > 256 || (box_w & 3u) != 0u)
        return false;
    PFN_cuTensorMapEncodeTiled enc = tensor_map_encoder();
    if (!enc) return false;
    const cuuint64_t dims[2] = {width, height};
    const cuuint64_t strides[1] = {(cuuint64_t)pitch * 4u};
    const cuuint32_t box[2] = {box_w, box_h};
    const cuuint32_t elem[2] = {1u, 1u};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, elem,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

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

void launch_hiz_build_tma(const CUtensorMap& src, const HizJob& job, uint32_t* ticket_dev, uint32_t* error_dev,
                          cudaStream_t stream) {
    const uint32_t tiles = job.tiles_x * job.tiles_y;
    if (tiles == 0) return;
    // Per device, once: the kernel's shared-memory limit (a per-device attribute) and its
    // co-resident grid.
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static int grid_of[kMaxDevices] = {0};
    const size_t smem = kHizStages * kHizTileBytes + 128;
    int dev = 0;
    cudaGetDevice(&dev);
    int full = 0;
    {
        std::lock_guard<std::mutex> lk(mu);
        if (dev < 0 || dev >= kMaxDevices || grid_of[dev] == 0) {
            int sms = 0, per_sm = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaFuncSetAttribute(hiz_build_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hiz_build_tma_kernel, 256, smem);
            full = std::max(1, sms) * std::max(1, per_sm);
            if (dev >= 0 && dev < kMaxDevices) grid_of[dev] = full;
        } else {
            full = grid_of[dev];
        }
    }
    const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)full);
    helio_launch_begin("hiz_build_tma", stream);
    hiz_build_tma_kernel<<<grid, 256, smem, stream>>>(src, job, ticket_dev, error_dev);
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
