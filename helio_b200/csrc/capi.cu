// capi.cu — host side of the visibility passes behind the C-ABI of include/helio_cull.h.
//
// Each pass mirrors the reference RenderPass lifecycle (crates/helio-core/src/
// traits.rs:276-470): create ~ new(), prepare ~ prepare(&PrepareContext), execute ~
// execute(&mut PassContext), resize ~ on_resize(), publish ~ publish(). Buffers grow
// in prepare (x2 policy, crates/helio-pass-virtual-geometry/src/rendering.rs:729-764);
// execute never allocates.

#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>

#include "common.cuh"
#include "host_util.h"
#include "instance_cull.h"
#include "kernels.h"
#include "vg.h"

#include <map>
#include <mutex>
#include <vector>

static std::atomic<uint64_t> g_launches{0};

namespace {

// Event profiler state: pending (name, start, end) records until collected.
struct ProfRecord {
    const char* name;
    cudaEvent_t start, end;
};
struct Profiler {
    std::mutex mu;
    std::atomic<bool> enabled{false};
    std::vector<ProfRecord> pending;
    std::vector<cudaEvent_t> free_events;
    std::map<std::string, std::pair<uint64_t, double>> totals;
    thread_local static cudaEvent_t open_start;
    thread_local static const char* open_name;
    cudaEvent_t take() {
        if (!free_events.empty()) {
            cudaEvent_t e = free_events.back();
            free_events.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
};
thread_local cudaEvent_t Profiler::open_start = nullptr;
thread_local const char* Profiler::open_name = nullptr;
Profiler g_prof;

bool capturing(cudaStream_t s) {
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(s, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone;
}

}  // namespace

void helio_launch_begin(const char* kernel, cudaStream_t stream) {
    if (!g_prof.enabled.load(std::memory_order_relaxed) || capturing(stream)) return;
    std::lock_guard<std::mutex> lk(g_prof.mu);
    Profiler::open_start = g_prof.take();
    Profiler::open_name = kernel;
    cudaEventRecord(Profiler::open_start, stream);
}

void helio_launch_note(void) { g_launches.fetch_add(1, std::memory_order_relaxed); }

void helio_launch_end(cudaStream_t stream) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    if (!Profiler::open_start) return;
    std::lock_guard<std::mutex> lk(g_prof.mu);
    cudaEvent_t end = g_prof.take();
    cudaEventRecord(end, stream);
    g_prof.pending.push_back({Profiler::open_name, Profiler::open_start, end});
    Profiler::open_start = nullptr;
    Profiler::open_name = nullptr;
}

namespace {

thread_local std::string t_last_error;

int32_t fail(int32_t code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return code;
}

}  // namespace

int32_t helio_report_error(int32_t code, const char* message) { return fail(code, "%s", message); }

int32_t helio_fail(int32_t code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return fail(code, "%s", buf);
}

using helio::as_stream;
using helio::DevBuf;

namespace {

uint32_t mip_levels(uint32_t w, uint32_t h) { return helio::host_mip_levels(w, h); }

helio::HizView to_view(const helio_hiz_pyramid& p) {
    helio::HizView v{};
    for (int l = 0; l < HELIO_HIZ_MAX_MIPS; ++l) {
        v.levels[l] = p.levels[l];
        v.width[l] = p.width[l];
        v.height[l] = p.height[l];
        v.pitch[l] = p.pitch[l];
    }
    v.mip_count = p.mip_count;
    return v;
}

int32_t check_pyramid(const helio_hiz_pyramid* hiz) {
    if (!hiz) return fail(HELIO_ERR_RESOURCE, "Hi-Z pyramid not available (is the Hi-Z pass executed?)");
    if (hiz->mip_count == 0 || hiz->mip_count > HELIO_HIZ_MAX_MIPS)
        return fail(HELIO_ERR_INVALID_ARG, "Hi-Z pyramid mip_count %u out of range", hiz->mip_count);
    for (uint32_t l = 0; l < hiz->mip_count; ++l)
        if (!hiz->levels[l] || hiz->width[l] == 0 || hiz->height[l] == 0 || hiz->pitch[l] < hiz->width[l])
            return fail(HELIO_ERR_INVALID_ARG, "Hi-Z pyramid level %u malformed", l);
    return HELIO_OK;
}

}  // namespace

// ════════════════════════════════════════════════════════════════════════════
// Pass state
// ════════════════════════════════════════════════════════════════════════════

struct helio_hiz_pass {
    uint32_t width = 0, height = 0, flags = 0;
    DevBuf levels;
    DevBuf ticket;  // [0] last-tile ticket, [1] device error word (kDevTimeout, sticky)
    helio::HizJob job{};
    alignas(64) CUtensorMap depth_map{};  // level 0 in 64x64 boxes, when use_tma
    bool use_tma = false;
    const float* depth = nullptr;
    uint32_t depth_pitch = 0;
    uint64_t camera_generation = 0, prev_generation = 0;
    bool first_frame = true;
    bool prepared = false;
};

struct helio_indirect_dispatch_pass {
    uint32_t* stats = nullptr;
    float planes[24] = {0};
    uint32_t draw_count = 0;
};

struct helio_occlusion_cull_pass {
    uint32_t width = 0, height = 0;
    uint32_t* stats = nullptr;
    uint32_t draw_count = 0;
    helio_static_hiz static_hiz{};  // texels null = no static Hi-Z
};

struct helio_vg_pass {
    helio_vg_config cfg{};
    float lod_threshold = 2.0f;
    uint32_t publication_limit = HELIO_VG_DEFAULT_PUBLICATION_LIMIT;
    uint32_t counter_count = HELIO_VG_COUNTER_COUNT;
    // Scene (device resident).
    DevBuf m_bounds, m_cone, m_axis, m_draw, objects, instances, cull, items, staging;
    // Outputs and scratch.
    DevBuf indirect, draws, visibility, sel, scratch;
    uint32_t capacity = 0;
    uint32_t meshlet_count = 0, object_count = 0, work_item_count = 0, max_draw_count = 0;
    uint64_t last_version = 0, last_instance_version = 0;
    bool have_version = false;
    uint32_t num_tiles = 0;
    uint32_t items_per_warp = 32;
    size_t scratch_clear_bytes = 0;
    size_t view_offset = 0;
};

// ════════════════════════════════════════════════════════════════════════════
// Library-wide
// ════════════════════════════════════════════════════════════════════════════

extern "C" {

int32_t helio_abi_version(void) { return HELIO_ABI_VERSION; }
const char* helio_last_error(void) { return t_last_error.c_str(); }
uint64_t helio_kernel_launch_count(void) { return g_launches.load(); }

int32_t helio_profiler_enable(int32_t enabled) {
    g_prof.enabled.store(enabled != 0);
    return HELIO_OK;
}

int32_t helio_profiler_collect(helio_kernel_timing* out, uint32_t capacity, uint32_t* count) {
    HELIO_ARG(count && (capacity == 0 || out), "null pointer");
    std::lock_guard<std::mutex> lk(g_prof.mu);
    for (const ProfRecord& r : g_prof.pending) {
        HELIO_CK(cudaEventSynchronize(r.end));
        float ms = 0.0f;
        HELIO_CK(cudaEventElapsedTime(&ms, r.start, r.end));
        auto& t = g_prof.totals[r.name];
        t.first += 1;
        t.second += ms;
        g_prof.free_events.push_back(r.start);
        g_prof.free_events.push_back(r.end);
    }
    g_prof.pending.clear();
    uint32_t n = 0;
    for (const auto& kv : g_prof.totals) {
        if (n < capacity) {
            std::memset(&out[n], 0, sizeof(out[n]));
            std::strncpy(out[n].name, kv.first.c_str(), sizeof(out[n].name) - 1);
            out[n].launches = kv.second.first;
            out[n].total_ms = kv.second.second;
        }
        ++n;
    }
    *count = n;
    return HELIO_OK;
}

void helio_profiler_reset(void) {
    std::lock_guard<std::mutex> lk(g_prof.mu);
    for (const ProfRecord& r : g_prof.pending) {
        cudaEventSynchronize(r.end);
        g_prof.free_events.push_back(r.start);
        g_prof.free_events.push_back(r.end);
    }
    g_prof.pending.clear();
    g_prof.totals.clear();
}

const char* helio_status_string(int32_t status) {
    switch (status) {
        case HELIO_OK: return "ok";
        case HELIO_ERR_CUDA: return "cuda error";
        case HELIO_ERR_INVALID_ARG: return "invalid argument";
        case HELIO_ERR_RESOURCE: return "resource not found";
        case HELIO_ERR_CAPACITY: return "capacity exceeded";
        case HELIO_ERR_TIMEOUT: return "device wait timed out";
        case HELIO_ERR_BUDGET: return "memory budget exceeded";
        case HELIO_ERR_NOT_READY: return "not ready";
        default: return "unknown status";
    }
}

uint32_t helio_mip_levels(uint32_t width, uint32_t height) { return mip_levels(width, height); }

void helio_extract_frustum_planes(const float vp[16], float planes_out[24]) {
    // crates/helio-pass-indirect-dispatch/src/lib.rs:271-300. Host binary32 with
    // the same left-to-right order as the reference (no contraction: the host
    // compiler is invoked with -ffp-contract=off).
    float r[4][4];
    for (int i = 0; i < 4; ++i)
        for (int c = 0; c < 4; ++c) r[i][c] = vp[c * 4 + i];
    float p[6][4];
    for (int c = 0; c < 4; ++c) {
        p[0][c] = r[3][c] + r[0][c];
        p[1][c] = r[3][c] - r[0][c];
        p[2][c] = r[3][c] + r[1][c];
        p[3][c] = r[3][c] - r[1][c];
        p[4][c] = r[2][c];
        p[5][c] = r[3][c] - r[2][c];
    }
    for (int k = 0; k < 6; ++k) {
        float len = std::sqrt((p[k][0] * p[k][0] + p[k][1] * p[k][1]) + p[k][2] * p[k][2]);
        for (int c = 0; c < 4; ++c) planes_out[k * 4 + c] = (len > 1e-10f) ? p[k][c] / len : p[k][c];
    }
}

float helio_lod_max_error_pixels(uint32_t q) {
    switch (q) {  // crates/helio-pass-virtual-geometry/src/lib.rs:195-202
        case HELIO_LOD_LOW: return 4.0f;
        case HELIO_LOD_HIGH: return 1.0f;
        case HELIO_LOD_ULTRA: return 0.5f;
        default: return 2.0f;
    }
}

int32_t helio_instance_cull_data(const HelioGpuInstanceData* instances_dev, uint32_t count,
                                 HelioInstanceCullData* out_dev, void* stream) {
    HELIO_ARG(count == 0 || (instances_dev && out_dev), "null pointer");
    helio::launch_instance_cull_data(instances_dev, count, out_dev, as_stream(stream));
    HELIO_CK(cudaGetLastError());
    return HELIO_OK;
}

// ════════════════════════════════════════════════════════════════════════════
// Hi-Z
// ════════════════════════════════════════════════════════════════════════════

static int32_t hiz_configure(helio_hiz_pass* p, uint32_t w, uint32_t h) {
    HELIO_ARG(w > 0 && h > 0 && w <= 32768 && h <= 32768, "Hi-Z size must be 1..32768");
    p->width = w;
    p->height = h;
    p->prepared = false;
    p->first_frame = true;
    return HELIO_OK;
}

int32_t helio_hiz_create(const helio_hiz_config* config, helio_hiz_pass** out) {
    HELIO_ARG(config && out, "null pointer");
    *out = nullptr;
    helio_hiz_pass* p = new (std::nothrow) helio_hiz_pass();
    if (!p) return fail(HELIO_ERR_RESOURCE, "out of host memory");
    p->flags = config->flags;
    int32_t st = hiz_configure(p, config->width, config->height);
    if (st != HELIO_OK) {
        delete p;
        return st;
    }
    cudaError_t e = p->ticket.ensure(16);
    if (e == cudaSuccess) e = cudaMemset(p->ticket.ptr, 0, 16);
    if (e != cudaSuccess) {
        delete p;
        return fail(HELIO_ERR_CUDA, "Hi-Z scratch: %s", cudaGetErrorString(e));
    }
    *out = p;
    return HELIO_OK;
}

int32_t helio_hiz_prepare(helio_hiz_pass* p, const float* depth_dev, uint32_t depth_pitch,
                          uint64_t camera_generation) {
    HELIO_ARG(p && depth_dev, "null pointer");
    uint32_t pitch = depth_pitch ? depth_pitch : p->width;
    HELIO_ARG(pitch >= p->width, "depth pitch smaller than width");
    const bool copy = (p->flags & HELIO_HIZ_ALIAS_MIP0) == 0u;
    size_t floats = helio::hiz_layout(p->width, p->height, pitch, copy, &p->job);
    HELIO_CK(p->levels.ensure(floats * sizeof(float)));
    helio::hiz_assign(&p->job, depth_dev, p->levels.as<float>());
    p->use_tma = (p->flags & HELIO_HIZ_NO_TMA) == 0u &&
                 helio::encode_float_tile_map(&p->depth_map, depth_dev, p->width, p->height, pitch, helio::kHizTile,
                                              helio::kHizTile);
    p->depth = depth_dev;
    p->depth_pitch = pitch;
    p->camera_generation = camera_generation;
    p->prepared = true;
    return HELIO_OK;
}

int32_t helio_hiz_execute(helio_hiz_pass* p, void* stream) {
    HELIO_ARG(p, "null pointer");
    if (!p->prepared) return fail(HELIO_ERR_RESOURCE, "Hi-Z pass executed before prepare");
    // Reuse the previous pyramid when the camera is unchanged (crates/helio-pass-hiz/src/lib.rs:472-478).
    if (!p->first_frame && p->camera_generation != UINT64_MAX && p->camera_generation == p->prev_generation)
        return HELIO_OK;
    p->first_frame = false;
    p->prev_generation = p->camera_generation;
    if (p->use_tma)
        helio::launch_hiz_build_tma(p->depth_map, p->job, p->ticket.as<uint32_t>(), p->ticket.as<uint32_t>() + 1,
                                    as_stream(stream));
    else
        helio::launch_hiz_build_single(p->job, p->ticket.as<uint32_t>(), as_stream(stream));
    HELIO_CK(cudaGetLastError());
    return HELIO_OK;
}

int32_t helio_hiz_device_status(const helio_hiz_pass* p, void* stream) {
    HELIO_ARG(p, "null pointer");
    uint32_t err = 0;
    HELIO_CK(cudaMemcpyAsync(&err, p->ticket.as<uint32_t>() + 1, 4, cudaMemcpyDeviceToHost, as_stream(stream)));
    HELIO_CK(cudaStreamSynchronize(as_stream(stream)));
    if (err & helio::kDevTimeout) return fail(HELIO_ERR_TIMEOUT, "a Hi-Z tile load never completed (bounded wait)");
    return HELIO_OK;
}

int32_t helio_hiz_resize(helio_hiz_pass* p, uint32_t w, uint32_t h) {
    HELIO_ARG(p, "null pointer");
    return hiz_configure(p, w, h);
}

int32_t helio_hiz_publish(const helio_hiz_pass* p, helio_hiz_pyramid* out) {
    HELIO_ARG(p && out, "null pointer");
    if (!p->prepared) return fail(HELIO_ERR_RESOURCE, "Hi-Z pyramid not built yet");
    std::memset(out, 0, sizeof(*out));
    out->mip_count = p->job.mip_count;
    for (uint32_t l = 0; l < p->job.mip_count; ++l) {
        out->width[l] = p->job.lw[l];
        out->height[l] = p->job.lh[l];
        out->pitch[l] = p->job.lpitch[l];
        out->levels[l] = p->job.levels[l];
    }
    return HELIO_OK;
}

void helio_hiz_destroy(helio_hiz_pass* p) { delete p; }

// ════════════════════════════════════════════════════════════════════════════
// Instance passes
// ════════════════════════════════════════════════════════════════════════════

int32_t helio_indirect_dispatch_create(uint32_t* stats_dev, helio_indirect_dispatch_pass** out) {
    HELIO_ARG(stats_dev && out, "null pointer");
    helio_indirect_dispatch_pass* p = new (std::nothrow) helio_indirect_dispatch_pass();
    if (!p) return fail(HELIO_ERR_RESOURCE, "out of host memory");
    p->stats = stats_dev;
    *out = p;
    return HELIO_OK;
}

int32_t helio_indirect_dispatch_prepare(helio_indirect_dispatch_pass* p, const HelioGpuCameraUniforms* camera_host,
                                        uint32_t draw_count) {
    HELIO_ARG(p && camera_host, "null pointer");
    helio_extract_frustum_planes(camera_host->view_proj, p->planes);
    p->draw_count = draw_count;
    return HELIO_OK;
}

static int32_t check_scene(const helio_scene_buffers* s, uint32_t draw_count, bool need_aabb) {
    HELIO_ARG(s, "null scene");
    if (draw_count == 0) return HELIO_OK;
    HELIO_ARG(s->camera && s->instances && s->draw_calls && s->indirect, "scene buffer missing");
    HELIO_ARG(!need_aabb || s->aabbs, "AABB buffer missing");
    HELIO_ARG(draw_count <= s->draw_count, "draw_count exceeds the scene's draw-call buffer");
    return HELIO_OK;
}

int32_t helio_indirect_dispatch_execute(helio_indirect_dispatch_pass* p, const helio_scene_buffers* scene,
                                        void* stream) {
    HELIO_ARG(p, "null pointer");
    int32_t st = check_scene(scene, p->draw_count, true);
    if (st != HELIO_OK) return st;
    if (p->draw_count == 0) return HELIO_OK;
    helio::InstanceCullParams prm{};
    prm.camera = scene->camera;
    prm.instances = scene->instances;
    prm.draw_calls = scene->draw_calls;
    prm.instance_count = scene->instance_count;
    prm.aabbs = scene->aabbs;
    prm.indirect = scene->indirect;
    prm.stats = p->stats;
    std::memcpy(prm.planes, p->planes, sizeof(prm.planes));
    prm.draw_count = p->draw_count;
    helio::launch_instance_cull(prm, true, false, as_stream(stream));
    HELIO_CK(cudaGetLastError());
    return HELIO_OK;
}

void helio_indirect_dispatch_destroy(helio_indirect_dispatch_pass* p) { delete p; }

int32_t helio_occlusion_cull_create(uint32_t w, uint32_t h, uint32_t* stats_dev, helio_occlusion_cull_pass** out) {
    HELIO_ARG(stats_dev && out, "null pointer");
    helio_occlusion_cull_pass* p = new (std::nothrow) helio_occlusion_cull_pass();
    if (!p) return fail(HELIO_ERR_RESOURCE, "out of host memory");
    p->width = w;
    p->height = h;
    p->stats = stats_dev;
    *out = p;
    return HELIO_OK;
}

int32_t helio_occlusion_cull_prepare(helio_occlusion_cull_pass* p, uint32_t draw_count) {
    HELIO_ARG(p, "null pointer");
    p->draw_count = draw_count;
    return HELIO_OK;
}

static void fill_occlusion(helio::InstanceCullParams& prm, const helio_occlusion_cull_pass* p,
                           const helio_hiz_pyramid* hiz) {
    prm.hiz = to_view(*hiz);
    prm.screen_w = p->width;
    prm.screen_h = p->height;
    prm.hiz_mip_count = mip_levels(p->width, p->height);
    prm.static_texels = p->static_hiz.texels;
    for (int k = 0; k < 3; ++k) {
        prm.static_dims[k] = p->static_hiz.grid_resolution[k];
        prm.static_min[k] = p->static_hiz.world_bounds_min[k];
        prm.static_max[k] = p->static_hiz.world_bounds_max[k];
    }
}

int32_t helio_occlusion_cull_set_static_hiz(helio_occlusion_cull_pass* p, const helio_static_hiz* hiz) {
    HELIO_ARG(p, "null pointer");
    if (!hiz) {
        p->static_hiz = helio_static_hiz{};
        return HELIO_OK;
    }
    HELIO_ARG(hiz->texels, "static Hi-Z texels missing");
    for (int k = 0; k < 3; ++k) HELIO_ARG(hiz->grid_resolution[k] > 0, "static Hi-Z grid must be non-empty");
    HELIO_ARG((uint64_t)hiz->grid_resolution[2] * 6u <= 0x7FFFFFFFull &&
                  (uint64_t)hiz->grid_resolution[0] <= 0x7FFFFFFFull && (uint64_t)hiz->grid_resolution[1] <= 0x7FFFFFFFull,
              "static Hi-Z grid too large");
    p->static_hiz = *hiz;
    return HELIO_OK;
}

int32_t helio_occlusion_cull_execute(helio_occlusion_cull_pass* p, const helio_scene_buffers* scene,
                                     const helio_hiz_pyramid* hiz, uint64_t frame_num, void* stream) {
    HELIO_ARG(p, "null pointer");
    if (frame_num == 0) return HELIO_OK;  // occlusion-cull/src/lib.rs:321
    int32_t st = check_scene(scene, p->draw_count, false);
    if (st != HELIO_OK) return st;
    if (p->draw_count == 0) return HELIO_OK;
    st = check_pyramid(hiz);
    if (st != HELIO_OK) return st;
    helio::InstanceCullParams prm{};
    prm.camera = scene->camera;
    prm.instances = scene->instances;
    prm.draw_calls = scene->draw_calls;
    prm.instance_count = scene->instance_count;
    prm.indirect = scene->indirect;
    prm.stats = p->stats;
    prm.draw_count = p->draw_count;
    fill_occlusion(prm, p, hiz);
    helio::launch_instance_cull(prm, false, true, as_stream(stream));
    HELIO_CK(cudaGetLastError());
    return HELIO_OK;
}

int32_t helio_occlusion_cull_resize(helio_occlusion_cull_pass* p, uint32_t w, uint32_t h) {
    HELIO_ARG(p, "null pointer");
    p->width = w;
    p->height = h;
    return HELIO_OK;
}

void helio_occlusion_cull_destroy(helio_occlusion_cull_pass* p) { delete p; }

int32_t helio_instance_cull_fused_execute(helio_indirect_dispatch_pass* f, helio_occlusion_cull_pass* o,
                                          const helio_scene_buffers* scene, const helio_hiz_pyramid* hiz,
                                          uint64_t frame_num, void* stream) {
    HELIO_ARG(f && o, "null pointer");
    if (frame_num == 0) return helio_indirect_dispatch_execute(f, scene, stream);
    HELIO_ARG(f->draw_count == o->draw_count, "frustum and occlusion passes prepared with different draw counts");
    HELIO_ARG(f->stats == o->stats, "fused execution needs one shared statistics buffer");
    int32_t st = check_scene(scene, f->draw_count, true);
    if (st != HELIO_OK) return st;
    if (f->draw_count == 0) return HELIO_OK;
    st = check_pyramid(hiz);
    if (st != HELIO_OK) return st;
    helio::InstanceCullParams prm{};
    prm.camera = scene->camera;
    prm.instances = scene->instances;
    prm.draw_calls = scene->draw_calls;
    prm.instance_count = scene->instance_count;
    prm.aabbs = scene->aabbs;
    prm.indirect = scene->indirect;
    prm.stats = f->stats;
    std::memcpy(prm.planes, f->planes, sizeof(prm.planes));
    prm.draw_count = f->draw_count;
    fill_occlusion(prm, o, hiz);
    helio::launch_instance_cull(prm, true, true, as_stream(stream));
    HELIO_CK(cudaGetLastError());
    return HELIO_OK;
}

// ════════════════════════════════════════════════════════════════════════════
// Virtual geometry
// ════════════════════════════════════════════════════════════════════════════

int32_t helio_vg_create(const helio_vg_config* config, helio_vg_pass** out) {
    HELIO_ARG(config && out, "null pointer");
    HELIO_ARG(config->width > 0 && config->height > 0, "render size must be non-zero");
    HELIO_ARG(config->counter_count == 0 || config->counter_count == 2 || config->counter_count == 11,
              "counter_count must be 2 or 11");
    HELIO_ARG((config->flags & ~HELIO_VG_CLEAR_INDIRECT) == 0, "unknown VG pass flags");
    helio_vg_pass* p = new (std::nothrow) helio_vg_pass();
    if (!p) return fail(HELIO_ERR_RESOURCE, "out of host memory");
    p->cfg = *config;
    p->lod_threshold = helio_lod_max_error_pixels(config->lod_quality);
    p->publication_limit = config->publication_limit ? config->publication_limit : HELIO_VG_DEFAULT_PUBLICATION_LIMIT;
    p->counter_count = config->counter_count ? config->counter_count : HELIO_VG_COUNTER_COUNT;
    *out = p;
    return HELIO_OK;
}

static int32_t vg_copy(void* dst, const void* src, size_t bytes, uint32_t memory, cudaStream_t s) {
    if (!bytes) return HELIO_OK;
    HELIO_ARG(src, "frame data array missing");
    HELIO_CK(cudaMemcpyAsync(dst, src, bytes,
                             memory == HELIO_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    return HELIO_OK;
}

int32_t helio_vg_prepare(helio_vg_pass* p, const helio_vg_frame_data* f, void* stream) {
    HELIO_ARG(p && f, "null pointer");
    HELIO_ARG(f->memory == HELIO_MEM_HOST || f->memory == HELIO_MEM_DEVICE, "unknown memory space");
    cudaStream_t s = as_stream(stream);
    int32_t st;
    if (!p->have_version || f->buffer_version != p->last_version) {
        // Full upload (rendering.rs:715-786).
        const size_t M = f->meshlet_count, O = f->object_count, W = f->work_item_count;
        HELIO_CK(p->m_bounds.ensure(M * 16));
        HELIO_CK(p->m_cone.ensure(M * 16));
        HELIO_CK(p->m_axis.ensure(M * 16));
        HELIO_CK(p->m_draw.ensure(M * 16));
        HELIO_CK(p->objects.ensure(O * sizeof(HelioGpuVgObject)));
        HELIO_CK(p->instances.ensure(O * sizeof(HelioGpuInstanceData)));
        HELIO_CK(p->cull.ensure(O * sizeof(HelioInstanceCullData)));
        HELIO_CK(p->items.ensure(W * sizeof(HelioGpuVgWorkItem)));
        HELIO_CK(p->sel.ensure(O * sizeof(helio::SelRecord)));
        HELIO_CK(p->visibility.ensure(W * 8));
        const HelioGpuMeshletEntry* aos = f->meshlets;
        if (M) {
            if (f->memory == HELIO_MEM_HOST) {
                HELIO_CK(p->staging.ensure(M * sizeof(HelioGpuMeshletEntry)));
                if ((st = vg_copy(p->staging.ptr, f->meshlets, M * sizeof(HelioGpuMeshletEntry), f->memory, s))) return st;
                aos = p->staging.as<HelioGpuMeshletEntry>();
            }
            HELIO_ARG(aos, "meshlet array missing");
            helio::launch_pack_meshlets(aos, (uint32_t)M, p->m_bounds.as<float4>(), p->m_cone.as<float4>(),
                                        p->m_axis.as<float4>(), p->m_draw.as<uint4>(), s);
            HELIO_CK(cudaGetLastError());
        }
        if ((st = vg_copy(p->objects.ptr, f->objects, O * sizeof(HelioGpuVgObject), f->memory, s))) return st;
        if ((st = vg_copy(p->instances.ptr, f->instances, O * sizeof(HelioGpuInstanceData), f->memory, s))) return st;
        if ((st = vg_copy(p->items.ptr, f->work_items, W * sizeof(HelioGpuVgWorkItem), f->memory, s))) return st;
        helio::launch_instance_cull_data(p->instances.as<HelioGpuInstanceData>(), (uint32_t)O,
                                         p->cull.as<HelioInstanceCullData>(), s);
        HELIO_CK(cudaGetLastError());
        if (f->memory == HELIO_MEM_HOST && M) {
            // The staging copy is consumed by the pack kernel; release it once it ran.
            HELIO_CK(cudaStreamSynchronize(s));
            p->staging.release();
        }
        p->meshlet_count = f->meshlet_count;
        p->object_count = f->object_count;
        p->work_item_count = f->work_item_count;
        uint32_t bounded = f->max_draw_count < p->publication_limit ? f->max_draw_count : p->publication_limit;
        if (bounded > p->capacity) {
            uint64_t grown = (uint64_t)bounded * 2u;
            uint32_t cap = (uint32_t)(grown < p->publication_limit ? grown : p->publication_limit);
            HELIO_CK(p->indirect.ensure((size_t)cap * sizeof(HelioDrawIndexedIndirectArgs)));
            HELIO_CK(p->draws.ensure((size_t)cap * sizeof(HelioGpuVgDraw)));
            p->capacity = cap;
        }
        p->max_draw_count = bounded;
        p->items_per_warp = helio::vg_cull_items_per_warp(p->work_item_count);
        p->num_tiles = helio::vg_cull_tiles(p->work_item_count, p->items_per_warp);
        // scratch: counters (16 words) | tile counts (both cleared per execute) | warp counts |
        //          window bits | view constants (16-byte aligned)
        p->scratch_clear_bytes = 64 + (size_t)p->num_tiles * 4;
        p->view_offset = (64 + helio::vg_cull_scratch_words(p->num_tiles) * 4 + 15) & ~(size_t)15;
        HELIO_CK(p->scratch.ensure(p->view_offset + sizeof(helio::CullView)));
        HELIO_CK(cudaMemsetAsync(p->scratch.ptr, 0, p->scratch_clear_bytes, s));
        p->last_version = f->buffer_version;
        p->last_instance_version = f->instance_version;
        p->have_version = true;
    } else if (f->instance_version != p->last_instance_version) {
        // Dirty-instance patch (rendering.rs:787-819).
        const uint64_t start = f->instance_dirty_start, count = f->instance_dirty_count;
        HELIO_ARG(count > 0 && start + count <= p->object_count, "invalid dirty instance range");
        const HelioGpuInstanceData* src = f->instances + start;
        int32_t st2 = vg_copy(p->instances.as<HelioGpuInstanceData>() + start, src,
                              count * sizeof(HelioGpuInstanceData), f->memory, s);
        if (st2) return st2;
        helio::launch_instance_cull_data(p->instances.as<HelioGpuInstanceData>() + start, (uint32_t)count,
                                         p->cull.as<HelioInstanceCullData>() + start, s);
        HELIO_CK(cudaGetLastError());
        p->last_instance_version = f->instance_version;
    }
    return HELIO_OK;
}

int32_t helio_vg_execute(helio_vg_pass* p, const HelioGpuCameraUniforms* camera_dev, const helio_hiz_pyramid* hiz,
                         void* stream) {
    HELIO_ARG(p, "null pointer");
    if (!p->have_version || p->object_count == 0 || p->work_item_count == 0 || p->max_draw_count == 0)
        return HELIO_OK;  // rendering.rs:1032-1038
    HELIO_ARG(camera_dev, "camera missing");
    int32_t st = check_pyramid(hiz);
    if (st != HELIO_OK) return st;
    cudaStream_t s = as_stream(stream);
    uint32_t* scratch = p->scratch.as<uint32_t>();
    HELIO_CK(cudaMemsetAsync(p->scratch.ptr, 0, p->scratch_clear_bytes, s));
    if (p->cfg.flags & HELIO_VG_CLEAR_INDIRECT)  // rendering.rs:1128-1130
        HELIO_CK(cudaMemsetAsync(p->indirect.ptr, 0, (size_t)p->capacity * sizeof(HelioDrawIndexedIndirectArgs), s));

    helio::VgSceneDev scene{};
    scene.m_bounds = p->m_bounds.as<float4>();
    scene.m_cone = p->m_cone.as<float4>();
    scene.m_axis = p->m_axis.as<float4>();
    scene.m_draw = p->m_draw.as<uint4>();
    scene.objects = p->objects.as<HelioGpuVgObject>();
    scene.instances = p->instances.as<HelioGpuInstanceData>();
    scene.cull = p->cull.as<HelioInstanceCullData>();
    scene.items = p->items.as<HelioGpuVgWorkItem>();
    scene.meshlet_count = p->meshlet_count;
    scene.object_count = p->object_count;
    scene.instance_count = p->object_count;
    scene.work_item_count = p->work_item_count;

    helio::CullView* view =
        reinterpret_cast<helio::CullView*>(reinterpret_cast<char*>(p->scratch.ptr) + p->view_offset);
    helio::ViewSetupParams vs{};
    vs.camera = camera_dev;
    vs.out = view;
    vs.hiz = to_view(*hiz);
    vs.screen_height = p->cfg.height;
    vs.hiz_mip_count = mip_levels(p->cfg.width, p->cfg.height);  // unclamped, rendering.rs:828-829
    vs.lod_threshold_px = p->lod_threshold;

    helio::VgSelectParams sp{};
    // The select blocks build the view constants themselves (block 0 publishes them for
    // the meshlet kernels); only an empty scene, with no select launch, needs the setup launch.
    if (p->object_count) {
        sp.compute_view = 1u;
        sp.setup = vs;
    } else {
        helio::launch_vg_view_setup(vs, s);
    }
    sp.scene = scene;
    sp.view = view;
    sp.sel = p->sel.as<helio::SelRecord>();
    sp.counters = scratch;
    sp.counter_count = p->counter_count;
    sp.write_reserved = 1u;
    helio::launch_vg_select(sp, s);

    helio::VgCullParams cp{};
    cp.scene = scene;
    cp.view = view;
    cp.sel = p->sel.as<helio::SelRecord>();
    cp.indirect = p->indirect.as<HelioDrawIndexedIndirectArgs>();
    cp.draws = p->draws.as<HelioGpuVgDraw>();
    cp.counters = scratch;
    cp.visibility = p->visibility.as<uint32_t>();
    cp.scratch.tile_counts = scratch + 16;
    cp.scratch.warp_counts = cp.scratch.tile_counts + p->num_tiles;
    cp.scratch.bits = cp.scratch.warp_counts + (size_t)p->num_tiles * helio::kCullWarps;
    cp.capacity = p->max_draw_count;  // min(draw_capacity, buffer lengths), vg_cull.wgsl:248-251
    cp.num_tiles = p->num_tiles;
    cp.items_per_warp = p->items_per_warp;
    HELIO_CK(helio::launch_vg_cull(cp, s));
    HELIO_CK(cudaGetLastError());
    return HELIO_OK;
}

int32_t helio_vg_resize(helio_vg_pass* p, uint32_t w, uint32_t h) {
    HELIO_ARG(p && w > 0 && h > 0, "invalid size");
    p->cfg.width = w;
    p->cfg.height = h;
    return HELIO_OK;
}

int32_t helio_vg_set_lod_quality(helio_vg_pass* p, uint32_t q) {
    HELIO_ARG(p && q <= HELIO_LOD_ULTRA, "invalid LOD quality");
    p->cfg.lod_quality = q;
    p->lod_threshold = helio_lod_max_error_pixels(q);
    return HELIO_OK;
}

int32_t helio_vg_publish(const helio_vg_pass* p, helio_vg_outputs* out) {
    HELIO_ARG(p && out, "null pointer");
    std::memset(out, 0, sizeof(*out));
    out->indirect = p->indirect.as<HelioDrawIndexedIndirectArgs>();
    out->draws = p->draws.as<HelioGpuVgDraw>();
    out->counters = p->scratch.as<uint32_t>();
    out->visibility = p->visibility.as<uint32_t>();
    out->objects = p->objects.as<HelioGpuVgObject>();
    out->capacity = p->max_draw_count;
    out->counter_count = p->counter_count;
    out->work_item_count = p->work_item_count;
    out->object_count = p->object_count;
    return HELIO_OK;
}

int32_t helio_vg_device_status(helio_vg_pass* p, void* stream) {
    HELIO_ARG(p, "null pointer");
    // The VG kernels never wait on one another inside a launch; this reports any
    // asynchronous CUDA error of the work queued so far.
    HELIO_CK(cudaStreamSynchronize(as_stream(stream)));
    HELIO_CK(cudaGetLastError());
    return HELIO_OK;
}

void helio_vg_destroy(helio_vg_pass* p) { delete p; }

}  // extern "C"
