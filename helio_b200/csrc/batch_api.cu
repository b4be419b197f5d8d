// batch_api.cu — host side of the device-resident scene and of the batched
// multi-view cull (include/helio_cull.h, "Batched multi-view culling").

#include <cstddef>
#include <cstring>
#include <new>
#include <algorithm>
#include <vector>

#include "batch.h"
#include "host_util.h"
#include "kernels.h"
#include "shadow_host.h"
#include "vg.h"

using helio::as_stream;
using helio::DevBuf;

struct helio_vg_scene {
    DevBuf m_bounds, m_cone, m_axis, m_draw, objects, instances, cull, staging;
    DevBuf bounds;  // [2] launch_scene_bounds of the current objects and instances
    uint32_t meshlet_count = 0, object_count = 0;
    uint64_t lod0_meshlets = 0, max_spans = 0, max_draw_count = 0;
    uint64_t version = 0, instance_version = 0;
    bool have = false;

    helio::VgSceneDev dev() const {
        helio::VgSceneDev s{};
        s.m_bounds = m_bounds.as<float4>();
        s.m_cone = m_cone.as<float4>();
        s.m_axis = m_axis.as<float4>();
        s.m_draw = m_draw.as<uint4>();
        s.objects = objects.as<HelioGpuVgObject>();
        s.instances = instances.as<HelioGpuInstanceData>();
        s.cull = cull.as<HelioInstanceCullData>();
        s.items = nullptr;
        s.meshlet_count = meshlet_count;
        s.object_count = object_count;
        s.instance_count = object_count;
        s.work_item_count = 0;
        return s;
    }
};

struct helio_batch {
    helio_batch_config cfg{};
    const helio_vg_scene* scene = nullptr;
    uint32_t view_count = 0;
    std::vector<helio::BatchViewDev> host_views;
    DevBuf views, cviews, lod, levels, out_indirect, out_draws, clear, chunk_counts, chunk_vis, vis_list, chunk_offs, seg_totals,
        view_span_start, spans, group_counts, group_offs, group_bits, span_vis;
    size_t clear_bytes = 0;
    uint32_t grid = 0, object_chunks = 0, hiz_tiles = 0, span_capacity = 0, lod_pitch = 0;
    std::vector<size_t> out_offset;  // first draw of each view in out_indirect / out_draws
    bool prepared = false;
    helio_shadow_cull_pass* shadow = nullptr;  // attached per-face shadow cull, or null
    uint32_t spin_limit = helio::kSpinLimit;  // helio_batch_set_wait_limit
    uint32_t barrier_extra = 0;

    // Buffer k of the plan's order (kBuf* below).
    DevBuf& buf(int k) {
        DevBuf* all[] = {&levels, &out_indirect, &out_draws, &clear, &views, &cviews, &lod, &chunk_counts,
                         &chunk_vis, &vis_list, &chunk_offs, &seg_totals, &view_span_start, &spans,
                         &group_counts, &group_offs, &group_bits, &span_vis};
        return *all[k];
    }

    // Cleared region: counters (16 words per view) | barrier (2) | error (1) |
    // work queue (1) | phase stamps (u64, 8-byte aligned).
    uint32_t* counters(uint32_t v) const { return clear.as<uint32_t>() + 16u * v; }
    uint32_t* barrier() const { return clear.as<uint32_t>() + 16u * view_count; }
    uint32_t* error() const { return barrier() + 2; }
    uint32_t* work() const { return barrier() + 3; }
    uint32_t* setup_done() const { return barrier() + 4; }
    uint32_t* expand_work() const { return barrier() + 5; }
    uint32_t* test_work() const { return barrier() + 6; }
    uint32_t* shadow_work() const { return barrier() + 7; }
    size_t stamps_offset() const { return ((16u * view_count + 8u) * 4u + 7u) & ~(size_t)7u; }
    unsigned long long* stamps() const {
        return reinterpret_cast<unsigned long long*>(clear.as<char>() + stamps_offset());
    }
};

namespace {

int32_t copy_in(void* dst, const void* src, size_t bytes, uint32_t memory, cudaStream_t s) {
    if (!bytes) return HELIO_OK;
    HELIO_ARG(src, "frame data array missing");
    HELIO_CK(cudaMemcpyAsync(dst, src, bytes,
                             memory == HELIO_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, s));
    return HELIO_OK;
}

int32_t refresh_bounds(helio_vg_scene* sc, cudaStream_t s) {
    HELIO_CK(sc->bounds.ensure(8));
    HELIO_CK(cudaMemsetAsync(sc->bounds.ptr, 0, 8, s));
    HELIO_CK(helio::launch_scene_bounds(sc->dev(), sc->bounds.as<uint32_t>(), s));
    return HELIO_OK;
}

// Device buffers of a batch, in helio_batch::buf order.
enum {
    kBufLevels, kBufIndirect, kBufDraws, kBufClear, kBufViews, kBufCViews, kBufLod, kBufChunkCounts, kBufChunkVis,
    kBufVisList, kBufChunkOffs, kBufSegTotals, kBufViewSpanStart, kBufSpans, kBufGroupCounts, kBufGroupOffs,
    kBufGroupBits, kBufSpanVis, kBatchBufs
};

// Everything helio_batch_prepare sizes for a set of views: per-buffer bytes, the
// pyramid layout of each view (written into `dev` when given), output capacities.
struct BatchPlan {
    size_t need[kBatchBufs] = {};
    std::vector<size_t> level_off, out_offset;
    std::vector<uint32_t> capacity;
    uint32_t tiles = 0, pairs = 0, grid = 0, object_chunks = 0, span_capacity = 0, lod_pitch = 0;
};

// CTAs of the meshlet-test launch: the configured count (at most what fits), else the
// same share of the device as the first launch's `grid` CTAs.
uint32_t cull_grid_of(const helio_batch_config& cfg, uint32_t grid) {
    const uint32_t full = helio::batch_max_grid(), cull_full = helio::batch_cull_max_grid();
    if (cfg.cull_ctas) return std::min(cfg.cull_ctas, std::max(1u, cull_full));
    return std::max(1u, (uint32_t)((uint64_t)cull_full * grid / std::max(1u, full)));
}

int32_t plan_batch(const helio_batch_config& cfg, const helio_vg_scene* sc, uint32_t n, const helio_batch_view* views,
                   BatchPlan& p, helio::BatchViewDev* dev) {
    p.level_off.assign(n, 0);
    p.out_offset.assign(n + 1, 0);
    p.capacity.assign(n, 0);
    size_t level_floats = 0;
    const uint64_t default_cap = sc->max_draw_count < HELIO_VG_DEFAULT_PUBLICATION_LIMIT
                                     ? sc->max_draw_count
                                     : (uint64_t)HELIO_VG_DEFAULT_PUBLICATION_LIMIT;
    for (uint32_t v = 0; v < n; ++v) {
        const helio_batch_view& in = views[v];
        HELIO_ARG(in.width > 0 && in.height > 0 && in.width <= 32768 && in.height <= 32768,
                  "view size out of 1..32768");
        const uint32_t pitch = in.depth_pitch ? in.depth_pitch : in.width;
        HELIO_ARG(pitch >= in.width, "depth pitch smaller than width");
        helio::HizJob job{};
        helio::HizJob& J = dev ? dev[v].hiz : job;
        const size_t need = helio::hiz_layout(in.width, in.height, pitch, (in.flags & HELIO_HIZ_ALIAS_MIP0) == 0u, &J);
        p.level_off[v] = level_floats;
        level_floats += (need + 3u) & ~(size_t)3u;
        J.tile_begin = p.tiles;
        if (dev) dev[v].hiz_pair_begin = p.pairs;
        p.tiles += J.tiles_x * J.tiles_y;
        p.pairs += (J.tiles_x * J.tiles_y + 1u) / 2u;
        const uint32_t cap = in.draw_capacity ? in.draw_capacity : (uint32_t)default_cap;
        p.capacity[v] = cap;
        p.out_offset[v + 1] = p.out_offset[v] + (cap ? cap : 1);
    }
    const uint32_t O = sc->object_count;
    p.object_chunks = (O + helio::kBatchChunk - 1) / helio::kBatchChunk;
    uint64_t span_cap = cfg.max_spans ? cfg.max_spans : (uint64_t)n * sc->max_spans + 32ull * n;
    span_cap = (span_cap + 31u) & ~31ull;
    HELIO_ARG(span_cap <= 0x7FFFFFE0ull, "span capacity exceeds 2^31");
    p.span_capacity = (uint32_t)span_cap;
    p.grid = helio::batch_max_grid();
    HELIO_ARG(p.grid > 0, "the batch kernel does not fit on this device");
    if (cfg.max_ctas && cfg.max_ctas < p.grid) p.grid = cfg.max_ctas;
    p.lod_pitch = p.object_chunks * helio::kBatchChunk;
    const size_t units = (size_t)n * p.object_chunks, groups = p.span_capacity / 32u;
    p.need[kBufLevels] = level_floats * sizeof(float);
    p.need[kBufIndirect] = p.out_offset[n] * sizeof(HelioDrawIndexedIndirectArgs);
    p.need[kBufDraws] = p.out_offset[n] * sizeof(HelioGpuVgDraw);
    p.need[kBufClear] = (((16u * n + 8u) * 4u + 7u) & ~(size_t)7u) + helio::kBatchPhaseStamps * 8u;
    p.need[kBufViews] = n * sizeof(helio::BatchViewDev);
    p.need[kBufCViews] = n * sizeof(helio::CullView);
    p.need[kBufLod] = (size_t)n * (p.lod_pitch ? p.lod_pitch : helio::kBatchChunk);
    p.need[kBufChunkCounts] = (units + 1) * 4;
    p.need[kBufChunkVis] = (units + 1) * 4;
    p.need[kBufVisList] = std::max<size_t>(1, units) * helio::kBatchChunk * sizeof(uint16_t);
    p.need[kBufChunkOffs] = (units + 1) * 4;
    p.need[kBufSegTotals] = (size_t)std::max(p.grid, helio::batch_cull_max_grid()) * 4;
    p.need[kBufViewSpanStart] = (size_t)(n + 1) * 4;
    p.need[kBufSpans] = (size_t)p.span_capacity * sizeof(helio::ActiveSpan);
    p.need[kBufGroupCounts] = (groups + 1) * 4;
    p.need[kBufGroupOffs] = (groups + 1) * 4;
    p.need[kBufGroupBits] = (groups + 1) * helio::kWindowsPerWarp * 4;
    p.need[kBufSpanVis] = (cfg.flags & HELIO_BATCH_SPAN_VISIBILITY) ? (size_t)p.span_capacity * 8 : 0;
    for (size_t& x : p.need) x = x ? x : 16;  // DevBuf::ensure allocates at least 16 bytes
    return HELIO_OK;
}

}  // namespace

extern "C" {

int32_t helio_vg_scene_create(helio_vg_scene** out) {
    HELIO_ARG(out, "null pointer");
    *out = new (std::nothrow) helio_vg_scene();
    return *out ? HELIO_OK : helio_fail(HELIO_ERR_RESOURCE, "out of host memory");
}

int32_t helio_vg_scene_upload(helio_vg_scene* sc, const helio_vg_frame_data* f, void* stream) {
    HELIO_ARG(sc && f, "null pointer");
    HELIO_ARG(f->memory == HELIO_MEM_HOST || f->memory == HELIO_MEM_DEVICE, "unknown memory space");
    cudaStream_t s = as_stream(stream);
    int32_t st;
    if (!sc->have || f->buffer_version != sc->version) {
        const size_t M = f->meshlet_count, O = f->object_count;
        HELIO_CK(sc->m_bounds.ensure(M * 16));
        HELIO_CK(sc->m_cone.ensure(M * 16));
        HELIO_CK(sc->m_axis.ensure(M * 16));
        HELIO_CK(sc->m_draw.ensure(M * 16));
        HELIO_CK(sc->objects.ensure(O * sizeof(HelioGpuVgObject)));
        HELIO_CK(sc->instances.ensure(O * sizeof(HelioGpuInstanceData)));
        HELIO_CK(sc->cull.ensure(O * sizeof(HelioInstanceCullData)));
        const HelioGpuMeshletEntry* aos = f->meshlets;
        if (M) {
            if (f->memory == HELIO_MEM_HOST) {
                HELIO_CK(sc->staging.ensure(M * sizeof(HelioGpuMeshletEntry)));
                if ((st = copy_in(sc->staging.ptr, f->meshlets, M * sizeof(HelioGpuMeshletEntry), f->memory, s)))
                    return st;
                aos = sc->staging.as<HelioGpuMeshletEntry>();
            }
            HELIO_ARG(aos, "meshlet array missing");
            helio::launch_pack_meshlets(aos, (uint32_t)M, sc->m_bounds.as<float4>(), sc->m_cone.as<float4>(),
                                        sc->m_axis.as<float4>(), sc->m_draw.as<uint4>(), s);
            HELIO_CK(cudaGetLastError());
        }
        if ((st = copy_in(sc->objects.ptr, f->objects, O * sizeof(HelioGpuVgObject), f->memory, s))) return st;
        if ((st = copy_in(sc->instances.ptr, f->instances, O * sizeof(HelioGpuInstanceData), f->memory, s)))
            return st;
        helio::launch_instance_cull_data(sc->instances.as<HelioGpuInstanceData>(), (uint32_t)O,
                                         sc->cull.as<HelioInstanceCullData>(), s);
        HELIO_CK(cudaGetLastError());
        // Per-object span bound and LOD0 size, for capacities and the metric.
        std::vector<HelioGpuVgObject> objs(O);
        if (O) {
            HELIO_CK(cudaMemcpyAsync(objs.data(), sc->objects.ptr, O * sizeof(HelioGpuVgObject),
                                     cudaMemcpyDeviceToHost, s));
        }
        HELIO_CK(cudaStreamSynchronize(s));
        if (f->memory == HELIO_MEM_HOST) sc->staging.release();
        uint64_t lod0 = 0, spans = 0, maxd = 0;
        for (const HelioGpuVgObject& o : objs) {
            lod0 += o.lod_meshlet_counts[0];
            uint32_t mx = 0;
            for (uint32_t l = 0; l < HELIO_VG_LOD_LEVELS && l < o.lod_count; ++l)
                mx = o.lod_meshlet_counts[l] > mx ? o.lod_meshlet_counts[l] : mx;
            spans += (mx + 63u) / 64u;
            maxd += mx;
        }
        sc->meshlet_count = f->meshlet_count;
        sc->object_count = f->object_count;
        sc->lod0_meshlets = lod0;
        sc->max_spans = spans;
        sc->max_draw_count = maxd;
        sc->version = f->buffer_version;
        sc->instance_version = f->instance_version;
        sc->have = true;
        if ((st = refresh_bounds(sc, s))) return st;
    } else if (f->instance_version != sc->instance_version) {
        const uint64_t start = f->instance_dirty_start, count = f->instance_dirty_count;
        HELIO_ARG(count > 0 && start + count <= sc->object_count, "invalid dirty instance range");
        if ((st = copy_in(sc->instances.as<HelioGpuInstanceData>() + start, f->instances + start,
                          count * sizeof(HelioGpuInstanceData), f->memory, s)))
            return st;
        helio::launch_instance_cull_data(sc->instances.as<HelioGpuInstanceData>() + start, (uint32_t)count,
                                         sc->cull.as<HelioInstanceCullData>() + start, s);
        HELIO_CK(cudaGetLastError());
        sc->instance_version = f->instance_version;
        if ((st = refresh_bounds(sc, s))) return st;
    }
    return HELIO_OK;
}

int32_t helio_vg_scene_info_get(const helio_vg_scene* sc, helio_vg_scene_info* out) {
    HELIO_ARG(sc && out, "null pointer");
    out->meshlet_count = sc->meshlet_count;
    out->object_count = sc->object_count;
    out->lod0_meshlets = sc->lod0_meshlets;
    out->max_spans = sc->max_spans;
    out->device_bytes = sc->m_bounds.bytes + sc->m_cone.bytes + sc->m_axis.bytes + sc->m_draw.bytes +
                        sc->objects.bytes + sc->instances.bytes + sc->cull.bytes;
    return HELIO_OK;
}

void helio_vg_scene_destroy(helio_vg_scene* sc) { delete sc; }

int32_t helio_batch_create(const helio_batch_config* cfg, helio_batch** out) {
    HELIO_ARG(cfg && out, "null pointer");
    HELIO_ARG(cfg->max_views >= 1 && cfg->max_views <= HELIO_BATCH_MAX_VIEWS, "max_views must be 1..128");
    helio_batch* b = new (std::nothrow) helio_batch();
    if (!b) return helio_fail(HELIO_ERR_RESOURCE, "out of host memory");
    b->cfg = *cfg;
    *out = b;
    return HELIO_OK;
}

int32_t helio_batch_prepare(helio_batch* b, const helio_vg_scene* sc, uint32_t n, const helio_batch_view* views,
                            void* stream) {
    HELIO_ARG(b && sc && views, "null pointer");
    HELIO_ARG(sc->have, "scene not uploaded");
    HELIO_ARG(n >= 1 && n <= b->cfg.max_views, "view count must be 1..max_views");
    cudaStream_t s = as_stream(stream);
    b->prepared = false;
    b->scene = sc;
    b->view_count = n;
    b->host_views.assign(n, helio::BatchViewDev{});
    for (uint32_t v = 0; v < n; ++v) HELIO_ARG(views[v].depth, "view depth missing");

    BatchPlan plan;
    int32_t st;
    if ((st = plan_batch(b->cfg, sc, n, views, plan, b->host_views.data()))) return st;
    b->grid = plan.grid;
    b->object_chunks = plan.object_chunks;
    b->hiz_tiles = plan.pairs;
    b->span_capacity = plan.span_capacity;
    b->lod_pitch = plan.lod_pitch;
    b->out_offset = plan.out_offset;
    for (uint32_t v = 0; v < n; ++v) b->host_views[v].capacity = plan.capacity[v];
    for (int k = 0; k < kBatchBufs; ++k) HELIO_CK(b->buf(k).ensure(plan.need[k]));
    b->clear_bytes = plan.need[kBufClear];
    HELIO_CK(cudaMemsetAsync(b->clear.ptr, 0, b->clear_bytes, s));
    std::vector<size_t>& level_off = plan.level_off;
    // View table.
    for (uint32_t v = 0; v < n; ++v) {
        const helio_batch_view& in = views[v];
        helio::BatchViewDev& d = b->host_views[v];
        d.camera = in.camera;
        helio::hiz_assign(&d.hiz, in.depth, b->levels.as<float>() + level_off[v]);
        d.width = in.width;
        d.height = in.height;
        d.hiz_mip_count = helio::host_mip_levels(in.width, in.height);
        d.lod_threshold_px = in.lod_error_threshold_px > 0.0f ? in.lod_error_threshold_px : 2.0f;
        d.indirect = b->out_indirect.as<HelioDrawIndexedIndirectArgs>() + b->out_offset[v];
        d.draws = b->out_draws.as<HelioGpuVgDraw>() + b->out_offset[v];
        d.counters = b->counters(v);
    }
    HELIO_CK(cudaMemcpyAsync(b->views.ptr, b->host_views.data(), n * sizeof(helio::BatchViewDev),
                             cudaMemcpyHostToDevice, s));
    HELIO_CK(cudaStreamSynchronize(s));
    b->prepared = true;
    return HELIO_OK;
}

int32_t helio_batch_autotune(helio_batch* b, uint32_t repeats, helio_batch_tuning* out, void* stream) {
    HELIO_ARG(b && out, "null pointer");
    if (!b->prepared) return helio_fail(HELIO_ERR_RESOURCE, "autotune before prepare");
    cudaStream_t s = as_stream(stream);
    repeats = repeats ? repeats : 3u;
    int dev = 0, sms = 0;
    HELIO_CK(cudaGetDevice(&dev));
    HELIO_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    cudaEvent_t e0, e1;
    HELIO_CK(cudaEventCreate(&e0));
    HELIO_CK(cudaEventCreate(&e1));
    const helio_batch_config saved = b->cfg;
    auto time_cfg = [&](uint32_t views, uint32_t ctas, uint32_t cull_ctas, double& ms) -> int32_t {
        b->cfg.select_views = views;
        b->cfg.max_ctas = ctas;
        b->cfg.cull_ctas = cull_ctas;
        std::vector<float> t(repeats);
        int32_t st = helio_batch_execute(b, s);  // warm-up
        if (st) return st;
        for (uint32_t r = 0; r < repeats; ++r) {
            HELIO_CK(cudaEventRecord(e0, s));
            if ((st = helio_batch_execute(b, s))) return st;
            HELIO_CK(cudaEventRecord(e1, s));
            HELIO_CK(cudaEventSynchronize(e1));
            HELIO_CK(cudaEventElapsedTime(&t[r], e0, e1));
        }
        std::sort(t.begin(), t.end());
        ms = t[repeats / 2];
        return HELIO_OK;
    };
    double base = 0.0, best = 1e30;
    uint32_t best_v = 32, best_c = b->grid, best_cc = 0, n = 0;
    int32_t st = time_cfg(saved.select_views, saved.max_ctas, saved.cull_ctas, base);
    // Stage 1: the first launch's shape, the meshlet-test launch at its proportional share.
    for (uint32_t v = 8; !st && v <= 32; v += 8) {
        for (uint32_t k = 1; !st && k <= 3; ++k) {
            const uint32_t ctas = std::min<uint32_t>((uint32_t)sms * k, b->grid);
            double ms = 0.0;
            if ((st = time_cfg(v, ctas, 0, ms))) break;
            ++n;
            if (ms < best) {
                best = ms;
                best_v = v;
                best_c = ctas;
            }
        }
    }
    // Stage 2: the meshlet-test launch's CTAs per SM at the chosen first launch.
    const uint32_t cull_full = helio::batch_cull_max_grid();
    for (uint32_t k = 1; !st && (uint64_t)sms * k <= cull_full; ++k) {
        double ms = 0.0;
        if ((st = time_cfg(best_v, best_c, (uint32_t)sms * k, ms))) break;
        ++n;
        if (ms < best) {
            best = ms;
            best_cc = (uint32_t)sms * k;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->cfg = saved;
    if (st) return st;
    b->cfg.select_views = best_v;
    b->cfg.max_ctas = best_c;
    b->cfg.cull_ctas = best_cc;
    // Leave the outputs of the chosen configuration in the buffers.
    if ((st = helio_batch_execute(b, s))) return st;
    HELIO_CK(cudaStreamSynchronize(s));
    std::memset(out, 0, sizeof(*out));
    out->select_views = best_v;
    out->ctas = best_c;
    out->cull_ctas = best_cc ? best_cc : cull_grid_of(b->cfg, best_c);
    out->candidates = n;
    out->best_ms = best;
    out->default_ms = base;
    return HELIO_OK;
}

int32_t helio_batch_estimate_bytes(const helio_batch_config* cfg, const helio_vg_scene* sc, uint32_t n,
                                   const helio_batch_view* views, uint64_t* bytes) {
    HELIO_ARG(cfg && sc && views && bytes, "null pointer");
    HELIO_ARG(sc->have, "scene not uploaded");
    HELIO_ARG(n >= 1 && n <= HELIO_BATCH_MAX_VIEWS, "view count must be 1..128");
    BatchPlan plan;
    int32_t st;
    if ((st = plan_batch(*cfg, sc, n, views, plan, nullptr))) return st;
    uint64_t total = 0;
    for (size_t x : plan.need) total += x;
    *bytes = total;
    return HELIO_OK;
}

int32_t helio_batch_growth_bytes(const helio_batch* b, const helio_batch_config* cfg, const helio_vg_scene* sc,
                                 uint32_t n, const helio_batch_view* views, uint64_t* bytes) {
    HELIO_ARG(b && cfg && sc && views && bytes, "null pointer");
    HELIO_ARG(sc->have, "scene not uploaded");
    HELIO_ARG(n >= 1 && n <= HELIO_BATCH_MAX_VIEWS, "view count must be 1..128");
    BatchPlan plan;
    int32_t st;
    if ((st = plan_batch(*cfg, sc, n, views, plan, nullptr))) return st;
    uint64_t grow = 0;
    helio_batch* mb = const_cast<helio_batch*>(b);
    for (int k = 0; k < kBatchBufs; ++k) {
        const DevBuf& d = mb->buf(k);
        const size_t held = d.ptr ? d.bytes : 0;
        if (!d.ptr || plan.need[k] > d.bytes) grow += helio::grow_capacity(plan.need[k], held) - held;
    }
    *bytes = grow;
    return HELIO_OK;
}

int32_t helio_batch_reconfigure(helio_batch* b, const helio_batch_config* cfg) {
    HELIO_ARG(b && cfg, "null pointer");
    HELIO_ARG(cfg->max_views >= 1 && cfg->max_views <= HELIO_BATCH_MAX_VIEWS, "max_views must be 1..128");
    b->cfg = *cfg;
    b->prepared = false;
    return HELIO_OK;
}

int32_t helio_batch_device_bytes(const helio_batch* b, uint64_t* bytes) {
    HELIO_ARG(b && bytes, "null pointer");
    *bytes = b->views.bytes + b->cviews.bytes + b->lod.bytes + b->levels.bytes + b->out_indirect.bytes +
             b->out_draws.bytes + b->clear.bytes + b->chunk_counts.bytes + b->chunk_vis.bytes + b->vis_list.bytes +
             b->chunk_offs.bytes + b->seg_totals.bytes + b->view_span_start.bytes + b->spans.bytes +
             b->group_counts.bytes + b->group_offs.bytes + b->group_bits.bytes + b->span_vis.bytes;
    return HELIO_OK;
}

int32_t helio_batch_set_cameras(helio_batch* b, uint32_t n, const HelioGpuCameraUniforms* cams, void* stream) {
    HELIO_ARG(b && cams, "null pointer");
    HELIO_ARG(b->prepared && n == b->view_count, "camera count differs from the prepared views");
    cudaStream_t s = as_stream(stream);
    for (uint32_t v = 0; v < n; ++v) b->host_views[v].camera = cams[v];
    // One strided copy: the camera leads every entry of the view table.
    static_assert(offsetof(helio::BatchViewDev, camera) == 0, "camera leads the view table entry");
    HELIO_CK(cudaMemcpy2DAsync(b->views.ptr, sizeof(helio::BatchViewDev), b->host_views.data(),
                               sizeof(helio::BatchViewDev), sizeof(HelioGpuCameraUniforms), n, cudaMemcpyHostToDevice,
                               s));
    return HELIO_OK;
}

int32_t helio_batch_set_cameras_device(helio_batch* b, uint32_t n, const HelioGpuCameraUniforms* cams, void* stream) {
    HELIO_ARG(b && cams, "null pointer");
    HELIO_ARG(b->prepared && n == b->view_count, "camera count differs from the prepared views");
    HELIO_CK(cudaMemcpy2DAsync(b->views.ptr, sizeof(helio::BatchViewDev), cams, sizeof(HelioGpuCameraUniforms),
                               sizeof(HelioGpuCameraUniforms), n, cudaMemcpyDeviceToDevice, as_stream(stream)));
    return HELIO_OK;
}

int32_t helio_batch_pack_draws(const helio_batch* b, HelioDrawIndexedIndirectArgs* indirect, HelioGpuVgDraw* draws,
                               uint32_t* offsets, uint64_t capacity, void* stream) {
    HELIO_ARG(b && indirect && draws && offsets, "null pointer");
    HELIO_ARG(b->prepared, "batch not prepared");
    HELIO_CK(helio::launch_pack_draws(b->views.as<helio::BatchViewDev>(), b->view_count, indirect, draws, offsets,
                                      capacity, as_stream(stream)));
    return HELIO_OK;
}

int32_t helio_batch_attach_shadow(helio_batch* b, helio_shadow_cull_pass* pass) {
    HELIO_ARG(b, "null pointer");
    b->shadow = pass;
    return HELIO_OK;
}

int32_t helio_batch_execute(helio_batch* b, void* stream) {
    HELIO_ARG(b, "null pointer");
    if (!b->prepared) return helio_fail(HELIO_ERR_RESOURCE, "batch executed before prepare");
    cudaStream_t s = as_stream(stream);
    HELIO_CK(cudaMemsetAsync(b->clear.ptr, 0, b->clear_bytes, s));
    // No launch for an empty scene: an attached shadow cull then runs on its own.
    if (b->scene->object_count == 0) return b->shadow ? helio_shadow_cull_execute(b->shadow, stream) : HELIO_OK;
    helio::BatchParams P{};
    P.scene = b->scene->dev();
    P.views = b->views.as<helio::BatchViewDev>();
    P.cviews = b->cviews.as<helio::CullView>();
    P.lod = b->lod.as<uint8_t>();
    P.lod_pitch = b->lod_pitch;
    P.scene_bounds = b->scene->bounds.as<uint32_t>();
    P.view_count = b->view_count;
    P.select_views = b->cfg.select_views ? b->cfg.select_views : 32u;
    P.object_chunks = b->object_chunks;
    P.hiz_tiles = b->hiz_tiles;
    P.barrier = b->barrier();
    P.spin_limit = b->spin_limit;
    P.barrier_extra = b->barrier_extra;
    P.error = b->error();
    P.work = b->work();
    P.setup_done = b->setup_done();
    P.expand_work = b->expand_work();
    P.test_work = b->test_work();
    P.chunk_counts = b->chunk_counts.as<uint32_t>();
    P.chunk_vis = b->chunk_vis.as<uint32_t>();
    P.vis_list = b->vis_list.as<uint16_t>();
    P.chunk_offs = b->chunk_offs.as<uint32_t>();
    P.seg_totals = b->seg_totals.as<uint32_t>();
    P.view_span_start = b->view_span_start.as<uint32_t>();
    P.spans = b->spans.as<helio::ActiveSpan>();
    P.span_capacity = b->span_capacity;
    P.group_counts = b->group_counts.as<uint32_t>();
    P.group_offs = b->group_offs.as<uint32_t>();
    P.group_bits = b->group_bits.as<uint32_t>();
    P.span_vis = (b->cfg.flags & HELIO_BATCH_SPAN_VISIBILITY) ? b->span_vis.as<uint32_t>() : nullptr;
    P.phase_ns = b->stamps();
    P.shadow_blocks = 0;
    P.shadow_work = b->shadow_work();
    if (b->shadow && helio::shadow_dev(b->shadow, &P.shadow)) P.shadow_blocks = P.shadow.blocks;
    const uint32_t grid = (b->cfg.max_ctas && b->cfg.max_ctas < b->grid) ? b->cfg.max_ctas : b->grid;
    HELIO_CK(helio::launch_batch(P, grid, cull_grid_of(b->cfg, grid), s));
    return HELIO_OK;
}

int32_t helio_batch_get_phase_times(helio_batch* b, double* us_out, uint32_t capacity, uint32_t* count,
                                    void* stream) {
    HELIO_ARG(b && count && (capacity == 0 || us_out), "null pointer");
    HELIO_ARG(b->prepared, "batch not prepared");
    unsigned long long t[helio::kBatchPhaseStamps] = {0};
    HELIO_CK(cudaMemcpyAsync(t, b->stamps(), sizeof(t), cudaMemcpyDeviceToHost, as_stream(stream)));
    HELIO_CK(cudaStreamSynchronize(as_stream(stream)));
    const uint32_t n = 9;
    for (uint32_t k = 0; k < 7 && k < capacity; ++k)
        us_out[k] = (t[k + 1] >= t[k] && t[k] != 0) ? (double)(t[k + 1] - t[k]) * 1e-3 : 0.0;
    for (uint32_t k = 7; k < n && k < capacity; ++k) us_out[k] = (double)t[k + 1] * 1e-3;
    *count = n;
    return HELIO_OK;
}

int32_t helio_batch_get_view_outputs(const helio_batch* b, uint32_t v, helio_batch_view_outputs* out) {
    HELIO_ARG(b && out, "null pointer");
    HELIO_ARG(b->prepared && v < b->view_count, "view index out of range");
    const helio::BatchViewDev& d = b->host_views[v];
    std::memset(out, 0, sizeof(*out));
    out->indirect = d.indirect;
    out->draws = d.draws;
    out->counters = d.counters;
    out->lod = b->lod.as<uint8_t>() + (size_t)v * b->lod_pitch;
    out->capacity = d.capacity;
    out->object_count = b->scene->object_count;
    out->pyramid.mip_count = d.hiz.mip_count;
    for (uint32_t l = 0; l < d.hiz.mip_count; ++l) {
        out->pyramid.width[l] = d.hiz.lw[l];
        out->pyramid.height[l] = d.hiz.lh[l];
        out->pyramid.pitch[l] = d.hiz.lpitch[l];
        out->pyramid.levels[l] = d.hiz.levels[l];
    }
    return HELIO_OK;
}

int32_t helio_batch_get_spans(const helio_batch* b, helio_batch_span_list* out) {
    HELIO_ARG(b && out, "null pointer");
    HELIO_ARG(b->prepared, "batch not prepared");
    out->spans = b->spans.as<uint32_t>();
    out->visibility = (b->cfg.flags & HELIO_BATCH_SPAN_VISIBILITY) ? b->span_vis.as<uint32_t>() : nullptr;
    out->view_span_start = b->view_span_start.as<uint32_t>();
    out->span_capacity = b->span_capacity;
    out->view_count = b->view_count;
    return HELIO_OK;
}

int32_t helio_batch_set_wait_limit(helio_batch* b, uint32_t max_polls, uint32_t extra_arrivals) {
    HELIO_ARG(b, "null pointer");
    b->spin_limit = max_polls ? max_polls : helio::kSpinLimit;
    b->barrier_extra = extra_arrivals;
    return HELIO_OK;
}

int32_t helio_batch_status(helio_batch* b, void* stream) {
    HELIO_ARG(b, "null pointer");
    if (!b->prepared) return HELIO_OK;
    uint32_t err = 0;
    HELIO_CK(cudaMemcpyAsync(&err, b->error(), 4, cudaMemcpyDeviceToHost, as_stream(stream)));
    HELIO_CK(cudaStreamSynchronize(as_stream(stream)));
    if (err & helio::kBatchErrTimeout) return helio_fail(HELIO_ERR_TIMEOUT, "a grid barrier of the batch timed out");
    if (err & helio::kBatchErrSpanCapacity)
        return helio_fail(HELIO_ERR_CAPACITY, "active spans exceeded the batch's max_spans; outputs incomplete");
    return HELIO_OK;
}

void helio_batch_destroy(helio_batch* b) { delete b; }

}  // extern "C"
