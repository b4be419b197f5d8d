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

// Persistent form for one view whose level 0 TMA can address: CTA b takes tiles b, b + G,
// b + 2G, ... Thread 0 keeps kHizStages 64x64 tiles in flight per CTA (TMA loads into
// shared memory, one mbarrier per stage). A CTA is 4 warps and warp q reduces quadrant q
// (32x32 texels; q = 2 * row + column) of a landed tile on its own: each lane holds an
// 8-row x 4-column block, registers give levels 1 and 2, warp shuffles levels 3..5. The
// quadrants' level-5 texels meet in shared memory and thread 0 forms the tile's level-6
// texel after the next tile's barrier, so a tile costs one barrier of 4 warps. Every 2x2
// step takes its four texels in the order of hiz_build_kernel (top-left, top-right,
// bottom-left, bottom-right) through hiz_red4, so both forms give identical pyramids.
constexpr int kHizStages = 2;
constexpr int kHizTmaThreads = 128;
constexpr int kHizTmaCtasPerSm = 6;
constexpr uint32_t kHizTileBytes = kHizTile * kHizTile * 4u;
constexpr uint32_t kHizWaitPolls = 1u << 20;  // bounded wait for a landed tile
static_assert(2 * kHizTailBuf <= kHizStages * kHizTile * kHizTile, "the tail's two level buffers fit the staging");

__global__ void __launch_bounds__(kHizTmaThreads, kHizTmaCtasPerSm)
    hiz_build_tma_kernel(const __grid_constant__ CUtensorMap src, const __grid_constant__ HizJob J, uint32_t* ticket,
                         uint32_t* error) {
    extern __shared__ __align__(128) unsigned char s_raw[];  // kHizStages x 64 x 64 floats (+128 B)
    __shared__ __align__(8) uint64_t s_full[kHizStages];
    __shared__ float s_l5[2][4];  // level-5 texels of the quadrants, double-buffered by tile
    // The job in shared memory for the tail, whose fields of levels 7.. the tiles never read
    // (read from the parameter space, each level would wait for a cold constant-cache line).
    __shared__ __align__(16) HizJob s_J;
    // TMA writes its boxes at 128-byte aligned shared addresses.
    float* s_stage = reinterpret_cast<float*>(s_raw + ((128u - (smem_u32(s_raw) & 127u)) & 127u));
    const uint32_t tiles = J.tiles_x * J.tiles_y, G = gridDim.x;
    const int tid = threadIdx.x, lane = tid & 31, q = tid >> 5;
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
    for (int i = tid; i < (int)(sizeof(HizJob) / 4); i += kHizTmaThreads)
        reinterpret_cast<uint32_t*>(&s_J)[i] = reinterpret_cast<const uint32_t*>(&J)[i];
    __syncthreads();
    // The lane's 8x4 block within a staged tile.
    const int block = (32 * (q >> 1) + 8 * (lane >> 3)) * (int)kHizTile + 32 * (q & 1) + 4 * (lane & 7);
    uint32_t k = 0, prev = 0;
    bool failed = false;
    // The level-0 copy of the CTA's last tile waits until the CTA has taken its ticket, so
    // that the ticket's release does not wait for those stores.
    bool deferred = false;
    uint32_t dX0 = 0, dY0 = 0;
    float v[8][4];
    for (;; ++k) {
        const uint32_t t = blockIdx.x + k * G;
        if (t >= tiles) break;
        const int s = (int)(k % kHizStages);
        const bool landed = mbar_wait_bounded(&s_full[s], (k / kHizStages) & 1u, kHizWaitPolls);
        const float* tile = s_stage + s * (kHizTile * kHizTile) + block;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            const float4 x = *reinterpret_cast<const float4*>(tile + r * kHizTile);
            v[r][0] = x.x;
            v[r][1] = x.y;
            v[r][2] = x.z;
            v[r][3] = x.w;
        }
        // Stage s is read by every warp (and the previous tile's level-5 texels are in s_l5).
        if (__syncthreads_or(!landed)) {
            if (tid == 0) atomicOr(error, kDevTimeout);
            failed = true;
            break;
        }
        const uint32_t ty = t / J.tiles_x, tx = t - ty * J.tiles_x;
        const uint32_t X0 = tx * kHizTile, Y0 = ty * kHizTile;
        if (tid == 0) {
            if (t + kHizStages * G < tiles) issue(t + kHizStages * G, s);
            if (k > 0 && J.mip_count > 6) hiz_quad_level6(J, prev, s_l5[(k - 1) & 1]);
        }
        if (J.mip_count > 1) {
            const float m5 = hiz_quad_levels(J, X0, Y0, q, v);
            if (lane == 0) s_l5[k & 1][q] = m5;
        }
        if (t + G >= tiles && J.mip_count > 7) {
            deferred = true;
            dX0 = X0;
            dY0 = Y0;
        } else {
            hiz_quad_copy0(J, X0, Y0, q, v);
        }
        prev = t;
    }
    // A wait that gave up leaves later loads in flight: wait for them (bounded) before
    // the tail reuses the staging buffers or the CTA's shared memory is released.
    if (tid == 0) {
        for (uint32_t j = k; j < k + kHizStages; ++j)
            if (blockIdx.x + j * G < tiles)
                mbar_wait_bounded(&s_full[j % kHizStages], (j / kHizStages) & 1u, kHizWaitPolls);
    }
    __syncthreads();  // the last tile's level-5 texels
    if (tid == 0 && !failed && k > 0 && J.mip_count > 6) hiz_quad_level6(J, prev, s_l5[(k - 1) & 1]);
    // Levels 7..: every CTA takes one ticket after its last tile; thread 0 wrote all of this
    // CTA's level-6 texels, and its acquire-release add publishes them and, in the CTA with
    // the last ticket, sees every other CTA's. That CTA builds the tail with all 4 warps.
    if (J.mip_count > 7) {
        __shared__ uint32_t s_last;
        if (tid == 0) {
            uint32_t old;
            asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;" : "=r"(old) : "l"(ticket) : "memory");
            const uint32_t last = (old + 1u == G) ? 1u : 0u;
            if (last) *ticket = 0u;  // every other CTA has taken its ticket
            s_last = last;
        }
        __syncthreads();
        if (deferred) hiz_quad_copy0(J, dX0, dY0, q, v);
        // Every tile has landed and been read: the staging buffers hold the tail's levels.
        if (s_last) hiz_tail_body<4, 4>(s_J, s_stage, s_stage + kHizTailBuf);
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
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hiz_build_tma_kernel, kHizTmaThreads, smem);
            full = std::max(1, sms) * std::max(1, per_sm);
            if (dev >= 0 && dev < kMaxDevices) grid_of[dev] = full;
        } else {
            full = grid_of[dev];
        }
    }
    const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)full);
    helio_launch_begin("hiz_build_tma", stream);
    hiz_build_tma_kernel<<<grid, kHizTmaThreads, smem, stream>>>(src, job, ticket_dev, error_dev);
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
