// noalloc.cu — Hi-Z pyramid build for callers that cannot allocate device memory.
//
// Some hosts cannot call cudaMalloc at the point where they build the pyramid: an
// engine that owns every device allocation through its own pre-sized pools and
// forbids new allocations once a frame loop runs, a plugin loaded into a process
// whose device-memory accounting must stay fixed, or a frame loop that cannot take
// the implicit device synchronisation an allocation may cause. HiZBuildPass owns a
// small device allocation for its scratch (the completion ticket of the last-tile
// hand-off); this entry point instead keeps that scratch — one ticket per view — in
// the fixed array below, defined at file scope in device memory. The view
// descriptors travel by value as the kernel's parameter, so no host-to-device copy
// is made either. The caller passes the depth buffers and one output buffer for all
// levels, 16-byte aligned.
//
// Properties of the fixed array:
//   * at most kNoAllocMaxViews views per call (128 bytes of tickets); every GPU that
//     loads this library holds the array until the process exits;
//   * every call uses the same array and leaves its last contents there, so the
//     tickets are cleared on the stream at the start of each call; two calls whose
//     GPU work overlaps (different streams, or different host threads) race on it
//     and must be ordered by the caller;
//   * host code may not use the array's name as a device address: the first call on
//     each device looks the address up with cudaGetSymbolAddress (with that device
//     current) and caches it, so that first call on a device should come before any
//     stream capture.
// No cudaMalloc, cudaFree or allocating library routine is called here.

#include <cstring>
#include <mutex>

#include "common.cuh"
#include "hiz_tile.cuh"
#include "kernels.h"

namespace {

constexpr uint32_t kNoAllocMaxViews = 32;

struct NoAllocScratch {
    uint32_t tickets[kNoAllocMaxViews];
};

// Every view's job, passed by value as the kernel's parameter (32 x 280 bytes, within
// the 32 KB parameter space of sm_70 and later).
struct NoAllocJobs {
    helio::HizJob jobs[kNoAllocMaxViews];
};

static __device__ __align__(256) unsigned char g_noalloc_hiz_scratch[sizeof(NoAllocScratch)];

// The multi-view Hi-Z build of hiz.cu, reading its job table from the parameter
// instead of device memory: one CTA per 64x64 tile, the job found by a binary search
// over tile_begin, the last CTA of each view building levels 7.. (tickets[view]).
__global__ void __launch_bounds__(256) hiz_build_noalloc_kernel(const __grid_constant__ NoAllocJobs table,
                                                                uint32_t n_jobs, uint32_t* tickets) {
    __shared__ float s_m3[8][9];
    __shared__ helio::HizJob s_J;
    __shared__ uint32_t s_job;
    const uint32_t tile = blockIdx.x;
    if (threadIdx.x == 0) {
        uint32_t lo = 0, hi = n_jobs - 1;
        while (lo < hi) {  // last job with tile_begin <= tile
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (table.jobs[mid].tile_begin <= tile) lo = mid;
            else hi = mid - 1;
        }
        s_J = table.jobs[lo];
        s_job = lo;
    }
    __syncthreads();
    helio::hiz_tile(s_J, s_job, tile - s_J.tile_begin, tickets, s_m3);
}

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {nullptr};

// Errors go to the same per-thread message as every other entry point (helio_last_error).
int32_t noalloc_fail(int32_t code, const char* msg) { return helio_report_error(code, msg); }

}  // namespace

extern "C" int32_t helio_hiz_build_noalloc(uint32_t view_count, const helio_hiz_view_input* views, float* levels,
                                           size_t levels_floats, helio_hiz_pyramid* pyramids_out, void* stream) {
    if (view_count == 0 || !views || !levels || !pyramids_out)
        return noalloc_fail(HELIO_ERR_INVALID_ARG, "helio_hiz_build_noalloc: null pointer or no view");
    if (view_count > kNoAllocMaxViews)
        return noalloc_fail(HELIO_ERR_INVALID_ARG,
                            "helio_hiz_build_noalloc: at most 32 views per call (fixed scratch array)");
    // Level 1 is stored as float2 pairs and level 0 (when copied) as float4 rows; every
    // view's levels start on a 4-float boundary of `levels`, so `levels` itself must be
    // 16-byte aligned.
    if ((reinterpret_cast<uintptr_t>(levels) & 15u) != 0u)
        return noalloc_fail(HELIO_ERR_INVALID_ARG, "helio_hiz_build_noalloc: levels must be 16-byte aligned");

    // Device set-up: the scratch array's device address, once per device.
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
        return noalloc_fail(HELIO_ERR_CUDA, "helio_hiz_build_noalloc: no current CUDA device");
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_hiz_scratch);
            if (e != cudaSuccess || !p)
                return noalloc_fail(HELIO_ERR_CUDA, "helio_hiz_build_noalloc: cudaGetSymbolAddress failed");
            g_noalloc_ptr[dev] = p;
        }
        scratch = g_noalloc_ptr[dev];
    }

    // Jobs and pyramid descriptors: views are laid out one after another in `levels`.
    NoAllocJobs table{};
    helio::HizJob* jobs = table.jobs;
    size_t offset = 0;
    uint32_t tiles = 0;
    for (uint32_t v = 0; v < view_count; ++v) {
        const helio_hiz_view_input& in = views[v];
        if (!in.depth || in.width == 0 || in.height == 0 || in.width > 32768 || in.height > 32768)
            return noalloc_fail(HELIO_ERR_INVALID_ARG, "helio_hiz_build_noalloc: view size must be 1..32768");
        const uint32_t pitch = in.pitch ? in.pitch : in.width;
        if (pitch < in.width) return noalloc_fail(HELIO_ERR_INVALID_ARG, "helio_hiz_build_noalloc: pitch < width");
        const bool copy = (in.flags & HELIO_HIZ_ALIAS_MIP0) == 0u;
        const size_t need = helio::hiz_layout(in.width, in.height, pitch, copy, &jobs[v]);
        offset = (offset + 3u) & ~(size_t)3u;  // every view starts on a 16-byte boundary
        if (offset + need > levels_floats)
            return noalloc_fail(HELIO_ERR_INVALID_ARG, "helio_hiz_build_noalloc: levels buffer too small");
        helio::hiz_assign(&jobs[v], in.depth, levels + offset);
        offset += need;
        jobs[v].tile_begin = tiles;
        tiles += jobs[v].tiles_x * jobs[v].tiles_y;
        helio_hiz_pyramid& out = pyramids_out[v];
        std::memset(&out, 0, sizeof(out));
        out.mip_count = jobs[v].mip_count;
        for (uint32_t l = 0; l < jobs[v].mip_count; ++l) {
            out.width[l] = jobs[v].lw[l];
            out.height[l] = jobs[v].lh[l];
            out.pitch[l] = jobs[v].lpitch[l];
            out.levels[l] = jobs[v].levels[l];
        }
    }

    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    NoAllocScratch* dev_scratch = reinterpret_cast<NoAllocScratch*>(scratch);
    // An error left by an earlier call on this thread would otherwise be reported as
    // this call's launch failure below; it is reported (and left pending) instead.
    if (cudaPeekAtLastError() != cudaSuccess)
        return noalloc_fail(HELIO_ERR_CUDA, "helio_hiz_build_noalloc: a CUDA error from an earlier call is pending");
    // The tickets must start at zero; the previous call's contents are still there.
    if (cudaMemsetAsync(dev_scratch->tickets, 0, view_count * sizeof(uint32_t), s) != cudaSuccess)
        return noalloc_fail(HELIO_ERR_CUDA, "helio_hiz_build_noalloc: clearing the tickets failed");
    if (tiles == 0) return HELIO_OK;
    helio_launch_begin("hiz_build_noalloc", s);
    hiz_build_noalloc_kernel<<<tiles, 256, 0, s>>>(table, view_count, dev_scratch->tickets);
    helio_launch_end(s);
    if (cudaGetLastError() != cudaSuccess)
        return noalloc_fail(HELIO_ERR_CUDA, "helio_hiz_build_noalloc: kernel launch failed");
    return HELIO_OK;
}
