// serve.cu — continuous batching of cull requests over device-resident scenes.
//
// A request names a scene and carries 1..max_views views. The server keeps a FIFO of
// pending requests and `slots` batch contexts, each with its own stream and a
// cooperative launch of `ctas_per_slot` CTAs, so that batches of different slots run
// on the device at the same time. Each pump():
//   1. retires the slots whose launch has finished (event query, no blocking) and
//      records a completion per request;
//   2. while a slot is free, forms the next batch (helio_serve_plan_batch: the oldest
//      request, then later requests of the same scene that still fit max_views) and
//      admits it if the scenes' bytes plus every slot's scratch, grown to what this
//      batch needs (helio_batch_growth_bytes), stay within the HBM budget; then
//      prepares and launches it on the slot's stream.
// Requests that arrive while batches run join the queue and start as soon as a slot
// and memory are free: continuous batching, not a queue in front of one launch.
// A request's outputs stay in its batch's buffers until helio_serve_release; a slot
// is reused once all of its requests are released.
//
// There is no counterpart in the reference (its passes cull one view per frame); the
// per-view results are those of the batched kernel, hence of the single-view passes.

#include <algorithm>
#include <cstring>
#include <deque>
#include <new>
#include <unordered_map>
#include <vector>

#include "batch.h"
#include "host_util.h"

using helio::as_stream;

namespace {

struct ServeRequest {
    uint64_t id = 0, tag = 0;
    uint32_t scene = 0;
    std::vector<helio_batch_view> views;
    double arrival = 0.0, launch = 0.0, done = 0.0;
    int32_t status = HELIO_OK;
    int slot = -1;
    uint32_t first_view = 0, batch_requests = 0;
    bool complete = false;
    double device_ms = 0.0, device_start = 0.0, device_end = 0.0;
};

struct Slot {
    helio_batch* batch = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr, done = nullptr;
    std::vector<uint64_t> requests;  // of the current (or last) launch
    bool running = false;
    uint32_t unreleased = 0;
    uint64_t bytes = 0;  // device bytes the slot's batch holds
};

}  // namespace

struct helio_serve {
    helio_serve_config cfg{};
    std::vector<const helio_vg_scene*> scenes;
    uint64_t scene_bytes = 0;
    std::deque<uint64_t> pending;
    std::unordered_map<uint64_t, ServeRequest> reqs;
    std::vector<Slot> slots;
    std::vector<helio_serve_completion> completions;
    uint64_t next_id = 1, batches = 0;
    uint32_t grid = 0;
    cudaEvent_t origin = nullptr;  // device time origin of the completions' device times

    uint64_t used() const {
        uint64_t u = scene_bytes;
        for (const Slot& s : slots) u += s.bytes;
        return u;
    }
    ~helio_serve() {
        for (Slot& s : slots) {
            if (s.stream) cudaStreamSynchronize(s.stream);
            if (s.batch) helio_batch_destroy(s.batch);
            if (s.start) cudaEventDestroy(s.start);
            if (s.done) cudaEventDestroy(s.done);
            if (s.stream) cudaStreamDestroy(s.stream);
        }
        if (origin) cudaEventDestroy(origin);
    }
};

namespace {

helio_batch_config slot_config(const helio_serve* sv, uint32_t views, const helio_vg_scene* sc) {
    helio_batch_config c{};
    c.max_views = sv->cfg.max_views;
    c.flags = 0;
    const uint64_t per_view = sv->cfg.spans_per_view ? sv->cfg.spans_per_view : 0;
    helio_vg_scene_info info{};
    helio_vg_scene_info_get(sc, &info);
    c.max_spans = (per_view ? per_view : info.max_spans) * (uint64_t)views + 32ull * views;
    c.max_ctas = sv->grid;
    return c;
}

// Retires finished launches (non-blocking).
int32_t retire(helio_serve* sv, double now) {
    for (Slot& s : sv->slots) {
        if (!s.running) continue;
        const cudaError_t q = cudaEventQuery(s.done);
        if (q == cudaErrorNotReady) continue;
        if (q != cudaSuccess) return helio_fail(HELIO_ERR_CUDA, cudaGetErrorString(q));
        float ms = 0.0f, t0 = 0.0f, t1 = 0.0f;
        cudaEventElapsedTime(&ms, s.start, s.done);
        cudaEventElapsedTime(&t0, sv->origin, s.start);
        cudaEventElapsedTime(&t1, sv->origin, s.done);
        const int32_t st = helio_batch_status(s.batch, s.stream);
        s.running = false;
        for (uint64_t id : s.requests) {
            ServeRequest& r = sv->reqs[id];
            r.complete = true;
            r.done = now;
            r.status = st;
            r.device_ms = ms;
            helio_serve_completion c{};
            c.request = r.id;
            c.tag = r.tag;
            c.status = st;
            c.batch_requests = r.batch_requests;
            c.view_count = (uint32_t)r.views.size();
            c.arrival_s = r.arrival;
            c.launch_s = r.launch;
            c.done_s = now;
            c.batch_device_ms = ms;
            c.device_start_ms = t0;
            c.device_end_ms = t1;
            sv->completions.push_back(c);
        }
    }
    return HELIO_OK;
}

// Launches the requests at queue positions `chosen` on slot `k` with batch config `c`.
int32_t launch(helio_serve* sv, int k, const std::vector<uint32_t>& chosen, const helio_batch_config& c, double now) {
    Slot& s = sv->slots[(size_t)k];
    std::vector<uint64_t> ids;
    std::vector<helio_batch_view> views;
    for (uint32_t pos : chosen) ids.push_back(sv->pending[pos]);
    const uint32_t scene = sv->reqs[ids[0]].scene;
    for (uint64_t id : ids) {
        ServeRequest& r = sv->reqs[id];
        r.first_view = (uint32_t)views.size();
        views.insert(views.end(), r.views.begin(), r.views.end());
    }
    const helio_vg_scene* sc = sv->scenes[scene];
    int32_t st;
    if (!s.batch && (st = helio_batch_create(&c, &s.batch))) return st;
    if ((st = helio_batch_reconfigure(s.batch, &c))) return st;
    if ((st = helio_batch_prepare(s.batch, sc, (uint32_t)views.size(), views.data(), s.stream))) return st;
    helio_batch_device_bytes(s.batch, &s.bytes);
    HELIO_CK(cudaEventRecord(s.start, s.stream));
    if ((st = helio_batch_execute(s.batch, s.stream))) return st;
    HELIO_CK(cudaEventRecord(s.done, s.stream));
    // Remove the launched requests from the queue (positions are ascending).
    for (size_t i = chosen.size(); i-- > 0;) sv->pending.erase(sv->pending.begin() + chosen[i]);
    for (uint64_t id : ids) {
        ServeRequest& r = sv->reqs[id];
        r.slot = k;
        r.launch = now;
        r.batch_requests = (uint32_t)ids.size();
    }
    s.requests = ids;
    s.running = true;
    s.unreleased = (uint32_t)ids.size();
    ++sv->batches;
    return HELIO_OK;
}

}  // namespace

extern "C" {

int32_t helio_serve_plan_batch(const helio_serve_pending* queue, uint32_t n, uint32_t max_views, uint32_t max_requests,
                               uint32_t* chosen, uint32_t* count) {
    HELIO_ARG(count && (n == 0 || (queue && chosen)), "null pointer");
    *count = 0;
    if (n == 0) return HELIO_OK;
    HELIO_ARG(max_views >= 1, "max_views must be at least 1");
    const uint32_t scene = queue[0].scene;
    uint32_t views = 0;
    for (uint32_t i = 0; i < n; ++i) {
        if (queue[i].scene != scene) continue;
        if (max_requests && *count >= max_requests) break;
        if (i == 0) {
            HELIO_ARG(queue[0].view_count >= 1 && queue[0].view_count <= max_views, "request view count out of range");
        } else if (views + queue[i].view_count > max_views) {
            continue;  // a later, smaller request of the scene may still fit
        }
        views += queue[i].view_count;
        chosen[(*count)++] = i;
    }
    return HELIO_OK;
}

int32_t helio_serve_create(const helio_serve_config* cfg, helio_serve** out) {
    HELIO_ARG(cfg && out, "null pointer");
    HELIO_ARG(cfg->slots >= 1 && cfg->slots <= 16, "slots must be 1..16");
    HELIO_ARG(cfg->max_views >= 1 && cfg->max_views <= HELIO_BATCH_MAX_VIEWS, "max_views must be 1..128");
    helio_serve* sv = new (std::nothrow) helio_serve();
    if (!sv) return helio_fail(HELIO_ERR_RESOURCE, "out of host memory");
    sv->cfg = *cfg;
    const uint32_t full = helio::batch_max_grid();
    if (full == 0) {
        delete sv;
        return helio_fail(HELIO_ERR_RESOURCE, "the batch kernel does not fit on this device");
    }
    sv->grid = cfg->ctas_per_slot ? std::min(cfg->ctas_per_slot, full) : std::max(1u, full / cfg->slots);
    sv->slots.resize(cfg->slots);
    bool ok = cudaEventCreate(&sv->origin) == cudaSuccess;
    for (Slot& s : sv->slots) {
        ok = ok && cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreate(&s.start) == cudaSuccess && cudaEventCreate(&s.done) == cudaSuccess;
    }
    // The origin of the device times: recorded before any launch of this server.
    ok = ok && cudaEventRecord(sv->origin, sv->slots[0].stream) == cudaSuccess;
    if (!ok) {
        delete sv;
        return helio_fail(HELIO_ERR_CUDA, "stream or event creation failed");
    }
    *out = sv;
    return HELIO_OK;
}

int32_t helio_serve_add_scene(helio_serve* sv, const helio_vg_scene* scene, uint32_t* id) {
    HELIO_ARG(sv && scene && id, "null pointer");
    helio_vg_scene_info info{};
    int32_t st;
    if ((st = helio_vg_scene_info_get(scene, &info))) return st;
    if (sv->cfg.hbm_budget_bytes && sv->used() + info.device_bytes > sv->cfg.hbm_budget_bytes)
        return helio_fail(HELIO_ERR_CAPACITY, "the scene does not fit in the HBM budget");
    sv->scene_bytes += info.device_bytes;
    *id = (uint32_t)sv->scenes.size();
    sv->scenes.push_back(scene);
    return HELIO_OK;
}

int32_t helio_serve_submit(helio_serve* sv, const helio_serve_request* rq, uint64_t* id) {
    HELIO_ARG(sv && rq && id, "null pointer");
    HELIO_ARG(rq->scene < sv->scenes.size(), "unknown scene");
    HELIO_ARG(rq->view_count >= 1 && rq->view_count <= sv->cfg.max_views && rq->views, "view count out of range");
    ServeRequest r;
    r.id = sv->next_id++;
    r.tag = rq->tag;
    r.scene = rq->scene;
    r.views.assign(rq->views, rq->views + rq->view_count);
    r.arrival = rq->arrival_s;
    sv->reqs.emplace(r.id, std::move(r));
    sv->pending.push_back(sv->next_id - 1);
    *id = sv->next_id - 1;
    return HELIO_OK;
}

int32_t helio_serve_pump(helio_serve* sv, double now_s, uint32_t* ready) {
    HELIO_ARG(sv, "null pointer");
    int32_t st;
    if ((st = retire(sv, now_s))) return st;
    while (!sv->pending.empty()) {
        int k = -1;
        for (size_t i = 0; i < sv->slots.size(); ++i)
            if (!sv->slots[i].running && sv->slots[i].unreleased == 0) {
                // Prefer a free slot that already holds the most memory (the least growth).
                if (k < 0 || sv->slots[i].bytes > sv->slots[(size_t)k].bytes) k = (int)i;
            }
        if (k < 0) break;
        std::vector<helio_serve_pending> q;
        q.reserve(sv->pending.size());
        for (uint64_t id : sv->pending) {
            const ServeRequest& r = sv->reqs[id];
            q.push_back(helio_serve_pending{r.scene, (uint32_t)r.views.size()});
        }
        std::vector<uint32_t> chosen(q.size());
        uint32_t n = 0;
        if ((st = helio_serve_plan_batch(q.data(), (uint32_t)q.size(), sv->cfg.max_views,
                                         sv->cfg.max_requests_per_batch, chosen.data(), &n)))
            return st;
        chosen.resize(n);
        std::vector<helio_batch_view> views;
        for (uint32_t pos : chosen) {
            const ServeRequest& r = sv->reqs[sv->pending[pos]];
            views.insert(views.end(), r.views.begin(), r.views.end());
        }
        const helio_vg_scene* sc = sv->scenes[q[0].scene];
        const helio_batch_config c = slot_config(sv, (uint32_t)views.size(), sc);
        const uint32_t nv = (uint32_t)views.size();
        Slot& s = sv->slots[(size_t)k];
        auto growth = [&](uint64_t& g) -> int32_t {
            return s.batch ? helio_batch_growth_bytes(s.batch, &c, sc, nv, views.data(), &g)
                           : helio_batch_estimate_bytes(&c, sc, nv, views.data(), &g);
        };
        uint64_t grow = 0;
        if ((st = growth(grow))) return st;
        if (sv->cfg.hbm_budget_bytes && sv->used() + grow > sv->cfg.hbm_budget_bytes) {
            // Free the memory of the other idle slots before waiting.
            bool freed = false;
            for (size_t i = 0; i < sv->slots.size(); ++i) {
                Slot& o = sv->slots[i];
                if ((int)i != k && !o.running && o.unreleased == 0 && o.batch) {
                    helio_batch_destroy(o.batch);
                    o.batch = nullptr;
                    o.bytes = 0;
                    freed = true;
                }
            }
            if (sv->used() + grow > sv->cfg.hbm_budget_bytes && s.batch) {
                // Start this slot afresh too: its old buffers may be the wrong shape.
                helio_batch_destroy(s.batch);
                s.batch = nullptr;
                s.bytes = 0;
                if ((st = growth(grow))) return st;
                freed = true;
            }
            if (sv->used() + grow > sv->cfg.hbm_budget_bytes) {
                bool busy = false;
                for (const Slot& o : sv->slots) busy = busy || o.running || o.unreleased;
                if (!busy && !freed) {
                    // Nothing else holds memory: this request can never be admitted.
                    const uint64_t id = sv->pending[chosen[0]];
                    ServeRequest& r = sv->reqs[id];
                    r.complete = true;
                    r.status = HELIO_ERR_CAPACITY;
                    r.done = now_s;
                    helio_serve_completion cpl{};
                    cpl.request = id;
                    cpl.tag = r.tag;
                    cpl.status = HELIO_ERR_CAPACITY;
                    cpl.view_count = (uint32_t)r.views.size();
                    cpl.arrival_s = r.arrival;
                    cpl.done_s = now_s;
                    sv->completions.push_back(cpl);
                    sv->pending.erase(sv->pending.begin() + chosen[0]);
                    continue;
                }
                if (!busy) continue;  // memory was freed: plan again
                break;                // wait for running batches to finish and be released
            }
        }
        if ((st = launch(sv, k, chosen, c, now_s))) return st;
    }
    if (ready) *ready = (uint32_t)sv->completions.size();
    return HELIO_OK;
}

int32_t helio_serve_completions(helio_serve* sv, helio_serve_completion* out, uint32_t capacity, uint32_t* count) {
    HELIO_ARG(sv && count && (capacity == 0 || out), "null pointer");
    const uint32_t n = (uint32_t)std::min<size_t>(capacity, sv->completions.size());
    if (n) std::memcpy(out, sv->completions.data(), n * sizeof(helio_serve_completion));
    sv->completions.erase(sv->completions.begin(), sv->completions.begin() + n);
    *count = n;
    return HELIO_OK;
}

int32_t helio_serve_outputs(const helio_serve* sv, uint64_t request, uint32_t view, helio_batch_view_outputs* out) {
    HELIO_ARG(sv && out, "null pointer");
    const auto it = sv->reqs.find(request);
    HELIO_ARG(it != sv->reqs.end(), "unknown or released request");
    const ServeRequest& r = it->second;
    HELIO_ARG(r.complete && r.slot >= 0, "request not complete");
    HELIO_ARG(view < r.views.size(), "view index out of range");
    return helio_batch_get_view_outputs(sv->slots[(size_t)r.slot].batch, r.first_view + view, out);
}

int32_t helio_serve_release(helio_serve* sv, uint64_t request) {
    HELIO_ARG(sv, "null pointer");
    const auto it = sv->reqs.find(request);
    HELIO_ARG(it != sv->reqs.end(), "unknown or released request");
    HELIO_ARG(it->second.complete, "request not complete");
    if (it->second.slot >= 0) {
        Slot& s = sv->slots[(size_t)it->second.slot];
        if (s.unreleased) --s.unreleased;
    }
    sv->reqs.erase(it);
    return HELIO_OK;
}

int32_t helio_serve_stats_get(const helio_serve* sv, helio_serve_stats* out) {
    HELIO_ARG(sv && out, "null pointer");
    std::memset(out, 0, sizeof(*out));
    out->pending = (uint32_t)sv->pending.size();
    for (const Slot& s : sv->slots) out->running += s.running ? 1u : 0u;
    out->batches = sv->batches;
    out->bytes_in_use = sv->used();
    out->scene_bytes = sv->scene_bytes;
    out->ctas_per_slot = sv->grid;
    return HELIO_OK;
}

void helio_serve_destroy(helio_serve* sv) { delete sv; }

}  // extern "C"
