// vg_cull.cu — virtual-geometry object select and meshlet cull (VirtualGeometryPass).
//
// References (crates/helio-pass-virtual-geometry/):
//   shaders/vg_cull.wgsl:282-352   cs_select_objects  -> vg_select_kernel
//   shaders/vg_cull.wgsl:135-264   cull_meshlet       -> meshlet_visible + emission
//   shaders/vg_cull.wgsl:354-405   cs_cull_meshlets   -> vg_cull_test_kernel + vg_cull_emit_kernel
//   src/lib.rs:132-167             InstanceCullData::from_instance -> instance_cull_data_kernel
//
// Layout and scheduling (B200 design, not a translation of the WGSL dispatches):
//   * meshlet descriptors are re-laid once per upload into four 16-byte streams;
//   * a warp owns 32 consecutive work items (one per lane); the lanes read their
//     item and the object's selected-LOD record, then the warp packs the active
//     meshlets of all 32 items densely into 32-lane windows, so a work item whose
//     LOD has 13 meshlets occupies 13 lanes instead of a 64-lane group;
//   * visible meshlets are compacted deterministically in two launches without
//     any device-side wait: the test kernel stores each warp's window ballots and
//     the per-tile / per-warp visible counts; the emit kernel runs only for tiles
//     with visible meshlets, sums the counts of the tiles before it, and writes
//     each draw at slot = (visible meshlets before it in (work item, lane) order).
//     The reference appends with atomicAdd (vg_cull.wgsl:247), so its order is
//     unspecified; this order is reproducible and first_instance = slot.

#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "vg.h"
#include "vg_device.cuh"

namespace helio {

namespace {

// ── Scene preparation ─────────────────────────────────────────────────────────

__global__ void pack_meshlets_kernel(const HelioGpuMeshletEntry* __restrict__ aos, uint32_t n,
                                     float4* __restrict__ bounds, float4* __restrict__ cone,
                                     float4* __restrict__ axis, uint4* __restrict__ draw) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4* src = reinterpret_cast<const float4*>(aos + i);
        bounds[i] = __ldcs(src + 0);
        cone[i] = __ldcs(src + 1);
        axis[i] = __ldcs(src + 2);
        draw[i] = __ldcs(reinterpret_cast<const uint4*>(src + 3));
    }
}

// InstanceCullData::from_instance (lib.rs:132-167), Rust f32 evaluation order.
__global__ void instance_cull_data_kernel(const HelioGpuInstanceData* __restrict__ inst, uint32_t n,
                                          HelioInstanceCullData* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float m[16];
        const float4* src = reinterpret_cast<const float4*>(inst[i].model);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            float4 q = __ldg(src + k);
            m[4 * k + 0] = q.x;
            m[4 * k + 1] = q.y;
            m[4 * k + 2] = q.z;
            m[4 * k + 3] = q.w;
        }
        const float sx = fsqrt(fadd(fadd(fmul(m[0], m[0]), fmul(m[1], m[1])), fmul(m[2], m[2])));
        const float sy = fsqrt(fadd(fadd(fmul(m[4], m[4]), fmul(m[5], m[5])), fmul(m[6], m[6])));
        const float sz = fsqrt(fadd(fadd(fmul(m[8], m[8]), fmul(m[9], m[9])), fmul(m[10], m[10])));
        const float max_scale = fmaxf(fmaxf(sx, sy), sz);
        const float min_scale = fminf(fminf(sx, sy), sz);
        const float dot_xy = fadd(fadd(fmul(m[0], m[4]), fmul(m[1], m[5])), fmul(m[2], m[6]));
        const float dot_xz = fadd(fadd(fmul(m[0], m[8]), fmul(m[1], m[9])), fmul(m[2], m[10]));
        const float dot_yz = fadd(fadd(fmul(m[4], m[8]), fmul(m[5], m[9])), fmul(m[6], m[10]));
        const float det = fadd(fsub(fmul(m[0], fsub(fmul(m[5], m[10]), fmul(m[6], m[9]))),
                                    fmul(m[4], fsub(fmul(m[1], m[10]), fmul(m[2], m[9])))),
                               fmul(m[8], fsub(fmul(m[1], m[6]), fmul(m[2], m[5]))));
        const bool affine = fabsf(m[3]) <= 1.0e-6f && fabsf(m[7]) <= 1.0e-6f && fabsf(m[11]) <= 1.0e-6f &&
                            fabsf(fsub(m[15], 1.0f)) <= 1.0e-4f;
        bool finite = true;
#pragma unroll
        for (int k = 0; k < 16; ++k) finite = finite && isfinite(m[k]);
        const bool valid = finite && isfinite(max_scale) && min_scale > 1.0e-8f && affine;
        const float ut = fmul(max_scale, 1.0e-4f);
        const float ot = fmul(fmul(max_scale, max_scale), 1.0e-4f);
        const bool ap = fsub(max_scale, min_scale) <= ut && fabsf(dot_xy) <= ot && fabsf(dot_xz) <= ot &&
                        fabsf(dot_yz) <= ot;
        const bool cone = valid && ap && det > 0.0f;
        HelioInstanceCullData r;
        r.max_scale = valid ? max_scale : 0.0f;
        r.min_scale = valid ? min_scale : 0.0f;
        r.cone_cull_enabled = cone ? 1u : 0u;
        r.valid_transform = valid ? 1u : 0u;
        out[i] = r;
    }
}

// ── View constants (one warp per launch) ──────────────────────────────────────

// The view constants of P's camera into v (shared memory), by one warp (every lane of
// the warp calls it; lanes 0..5 build the planes, lane 0 the rest).
__device__ __forceinline__ void view_setup_warp(const ViewSetupParams& P, CullView& v) {
    publish_planes_warp(P.camera->view_proj, v.planes);
    if ((threadIdx.x & 31) == 0) {
        const HelioGpuCameraUniforms* cam = P.camera;
        v.vp = ldg_mat4(cam->view_proj);
        v.pos_near = __ldg(reinterpret_cast<const float4*>(cam->position_near));
        v.p00 = __ldg(&cam->proj[0]);
        v.p11 = __ldg(&cam->proj[5]);
        v.focal = fmul(fmul(fabsf(v.p11), (float)P.screen_height), 0.5f);
        v.lod_threshold_px = P.lod_threshold_px;
        v.hiz = P.hiz;
        v.screen_height = P.screen_height;
        v.hiz_mip_count = P.hiz_mip_count;
        v.pad[0] = v.pad[1] = 0u;
    }
    __syncwarp();
}

__global__ void __launch_bounds__(32) vg_view_setup_kernel(ViewSetupParams P) {
    __shared__ CullView s_view;
    view_setup_warp(P, s_view);
    if (threadIdx.x == 0) *P.out = s_view;
}

// ── Object select: cs_select_objects (vg_cull.wgsl:282-352) ───────────────────

__global__ void __launch_bounds__(256) vg_select_kernel(VgSelectParams P) {
    __shared__ CullView s_view;
    pdl_launch_dependents();  // the meshlet tests may be scheduled (they wait for this grid)
    if (P.compute_view) {
        // The view setup folded in: warp 0 builds the constants; block 0 publishes them.
        if (threadIdx.x < 32) view_setup_warp(P.setup, s_view);
        __syncthreads();
        if (blockIdx.x == 0) {
            const uint4* src = reinterpret_cast<const uint4*>(&s_view);
            uint4* dst = reinterpret_cast<uint4*>(P.setup.out);
            for (uint32_t k = threadIdx.x; k < sizeof(CullView) / 16; k += blockDim.x) dst[k] = src[k];
        }
    } else {
        load_view(P.view, s_view, threadIdx.x, blockDim.x);
        __syncthreads();
    }
    const Planes& s_planes = s_view.planes;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const int lane = threadIdx.x & 31;
    const VgSceneDev& S = P.scene;
    bool vis = false;
    uint32_t selected = 0, lod_count = 0;
    if (i < S.object_count) {
        const HelioGpuVgObject* o = S.objects + i;
        // One round trip for the object fields, one for the instance fields.
        const uint4 head = __ldg(reinterpret_cast<const uint4*>(o));  // instance_index, lod_count, max_meshlet_count, reserved
        const float4 lb = __ldg(reinterpret_cast<const float4*>(o->local_bounds));
        const float4 e0 = __ldg(reinterpret_cast<const float4*>(o->lod_errors));
        const float4 e1 = __ldg(reinterpret_cast<const float4*>(o->lod_errors + 4));
        lod_count = min(head.y, 8u);
        const uint32_t ii = head.x;
        uint32_t sel = 0;
        if (lod_count > 0u && ii < S.instance_count) {
            const HelioInstanceCullData cd = load_cull(S.cull + ii);
            const Mat4 model = ldg_mat4(S.instances[ii].model);
            if (cd.valid_transform != 0u) {
                const F3 c = mat4_point3(model, f3(lb.x, lb.y, lb.z));
                const float wr = fmaxf(fmul(lb.w, cd.max_scale), 0.0f);
                if (sphere_visible_vg(s_planes, c, wr)) {
                    const float4 pn = s_view.pos_near;
                    const F3 d = sub3(c, f3(pn.x, pn.y, pn.z));
                    const float dist = fsqrt(dot3(d, d));
                    const float closest = fmaxf(fsub(dist, wr), fmaxf(pn.w, 1.0e-4f));
                    const float focal = s_view.focal;
                    const QuotientBound qb = quotient_bound(s_view.lod_threshold_px);
                    const float r = quotient_rcp(closest);
                    const float err[8] = {e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w};
                    uint32_t lod = 0;
#pragma unroll
                    for (uint32_t level = 1; level < 8; ++level) {
                        if (level >= lod_count) break;
                        // px = err * max_scale * focal / closest; px <= threshold keeps the level.
                        if (quotient_le(fmul(fmul(err[level], cd.max_scale), focal), closest, r, qb)) lod = level;
                        else break;
                    }
                    selected = lod;
                    sel = lod + 1;
                    vis = true;
                }
            }
        }
        SelRecord rec = make_uint4(0u, 0u, ii, sel);
        if (sel) {
            rec.x = __ldg(&o->lod_first_meshlets[sel - 1]);
            rec.y = __ldg(&o->lod_meshlet_counts[sel - 1]);
        }
        P.sel[i] = rec;
        if (P.write_reserved) S.objects[i].reserved = sel;
    }
    if (P.counter_count >= 11u) {
#pragma unroll
        for (uint32_t l = 0; l < 8; ++l) {
            const uint32_t n = __popc(__ballot_sync(0xffffffffu, vis && selected == l));
            if (lane == 0 && n) atomicAdd(P.counters + 2 + l, n);
        }
        uint32_t mx = vis ? lod_count - 1u : 0u;
        const bool any = __ballot_sync(0xffffffffu, vis) != 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (lane == 0 && any) atomicMax(P.counters + 10, mx);
    }
}

// ── Meshlet cull ──────────────────────────────────────────────────────────────

// The 32 work items of one warp (lane = item): active meshlet range and packing offsets.
struct WarpItems {
    uint32_t n, first, inst, lod, off, total;
};

__device__ __forceinline__ WarpItems load_warp_items(const VgSceneDev& S, const SelRecord* sel, uint32_t w_idx) {
    const int lane = threadIdx.x & 31;
    WarpItems w{0u, 0u, 0u, 0u, 0u, 0u};
    if (w_idx < S.work_item_count) {
        const HelioGpuVgWorkItem it = S.items[w_idx];
        if (it.object_index < S.object_count) {
            const SelRecord r = __ldg(sel + it.object_index);
            if (r.w != 0u && it.local_meshlet_base < r.y) {
                w.n = min(64u, r.y - it.local_meshlet_base);
                w.first = r.x + it.local_meshlet_base;
                w.inst = r.z;
                w.lod = r.w - 1u;
            }
        }
    }
    uint32_t incl = w.n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    w.off = incl - w.n;
    w.total = __shfl_sync(0xffffffffu, incl, 31);
    return w;
}

constexpr int kBitWordsPerWarp = kWindowsPerWarp + 2;  // +2 so bit-field reads stay in bounds

// kWide: the form for large scenes, whose warps each walk many windows (32 work items per
// warp) and whose launch has more tiles than fit at four CTAs per SM: they gain more from a
// fifth resident CTA than they lose to loading the cone inputs after the frustum test (10M
// meshlets at 3840x2160: 27.3 -> 25.0 us). With fewer items per warp each warp's latency
// dominates, and the loads stay together (1M meshlets: 43.6 against 45.5 us per step).
template <bool kWide>
__global__ void __launch_bounds__(kCullWarps * 32, kWide ? 5 : 4) vg_cull_test_kernel(VgCullParams P) {
    __shared__ CullView s_view;
    __shared__ uint32_t s_bits[kCullWarps][kBitWordsPerWarp];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const VgSceneDev& S = P.scene;
    const uint32_t tile = blockIdx.x;
    pdl_launch_dependents();  // the emission may be scheduled (it waits for this grid)
    for (int k = lane; k < kBitWordsPerWarp; k += 32) s_bits[warp][k] = 0u;
    pdl_wait();  // the select's records and view constants
    const bool mine = (uint32_t)lane < P.items_per_warp;
    const uint32_t w_idx = (tile * kCullWarps + warp) * P.items_per_warp + lane;
    const WarpItems it = load_warp_items(S, P.sel, mine ? w_idx : 0xFFFFFFFFu);

    // View constants are staged only when some warp of the tile has work.
    if (__syncthreads_or(it.total > 0u)) {
        load_view(P.view, s_view, tid, blockDim.x);
        __syncthreads();
    }

    uint32_t warp_count = 0;
    const uint32_t windows = (it.total + 31u) >> 5;
    for (uint32_t win = 0; win < windows; ++win) {
        const uint32_t s = win * 32u + lane;
        const int j = owner_lane(it.off, s);
        const uint32_t j_off = __shfl_sync(0xffffffffu, it.off, j);
        const uint32_t j_first = __shfl_sync(0xffffffffu, it.first, j);
        const uint32_t j_inst = __shfl_sync(0xffffffffu, it.inst, j);
        bool vis = false;
        if (s < it.total) {
            const uint32_t mi = j_first + (s - j_off);
            if (mi < S.meshlet_count) {
                const HelioGpuInstanceData* in = S.instances + j_inst;
                const HelioInstanceCullData cd = load_cull(S.cull + j_inst);
                const Mat4 model = ldg_mat4(in->model);
                vis = meshlet_visible<false, kWide>(S, s_view, mi, model, cd, in);
            }
        }
        const uint32_t bits = __ballot_sync(0xffffffffu, vis);
        if (lane == 0) s_bits[warp][win] = bits;
        warp_count += __popc(bits);
    }
    __syncwarp();
    const size_t wslot = (size_t)tile * kCullWarps + warp;
    if (lane == 0) {
        P.scratch.warp_counts[wslot] = warp_count;
        if (warp_count) {
            atomicAdd(P.scratch.tile_counts + tile, warp_count);
            atomicAdd(P.counters + 0, warp_count);
        }
    }
    if (warp_count) {
        for (uint32_t k = lane; k < windows; k += 32) P.scratch.bits[wslot * kWindowsPerWarp + k] = s_bits[warp][k];
    }
    // Per-work-item visibility words: bits [off, off + n) of the warp's window bits.
    if (P.visibility && mine && w_idx < S.work_item_count) {
        uint32_t lo = 0, hi = 0;
        if (it.n) {
            const uint32_t w0 = it.off >> 5, sh = it.off & 31u;
            const unsigned long long a = (unsigned long long)s_bits[warp][w0] |
                                         ((unsigned long long)s_bits[warp][w0 + 1] << 32);
            const unsigned long long c = s_bits[warp][w0 + 2];
            unsigned long long field = sh ? ((a >> sh) | (c << (64 - sh))) : a;
            if (it.n < 64) field &= (1ull << it.n) - 1ull;
            lo = (uint32_t)field;
            hi = (uint32_t)(field >> 32);
        }
        reinterpret_cast<uint2*>(P.visibility)[w_idx] = make_uint2(lo, hi);
    }
}

__global__ void __launch_bounds__(kCullWarps * 32) vg_cull_emit_kernel(VgCullParams P) {
    __shared__ uint32_t s_red[kCullWarps];
    __shared__ uint32_t s_prefix;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tile = blockIdx.x;
    pdl_wait();  // the meshlet tests' counts and window bits
    const uint32_t count = P.scratch.tile_counts[tile];
    if (count == 0u) return;  // uniform: the whole CTA leaves

    // Exclusive prefix: visible meshlets of all earlier tiles.
    uint32_t sum = 0;
    for (uint32_t i = tid; i < tile; i += blockDim.x) sum += P.scratch.tile_counts[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) s_red[warp] = sum;
    __syncthreads();
    if (tid == 0) {
        uint32_t p = 0;
#pragma unroll
        for (int w = 0; w < (int)kCullWarps; ++w) p += s_red[w];
        s_prefix = p;
        const unsigned long long end = (unsigned long long)p + count;
        const unsigned long long lo = p > P.capacity ? p : P.capacity;
        if (end > lo) atomicAdd(P.counters + 1, (uint32_t)(end - lo));
    }
    __syncthreads();

    const size_t wslot0 = (size_t)tile * kCullWarps;
    const uint32_t wc = P.scratch.warp_counts[wslot0 + warp];
    if (wc == 0u) return;  // uniform per warp; no block barrier follows
    uint32_t base = s_prefix;
    for (int w = 0; w < warp; ++w) base += P.scratch.warp_counts[wslot0 + w];

    const VgSceneDev& S = P.scene;
    const uint32_t w_idx = (tile * kCullWarps + warp) * P.items_per_warp + lane;
    const WarpItems it = load_warp_items(S, P.sel, (uint32_t)lane < P.items_per_warp ? w_idx : 0xFFFFFFFFu);
    const uint32_t windows = (it.total + 31u) >> 5;
    const uint32_t* wbits = P.scratch.bits + (wslot0 + warp) * kWindowsPerWarp;
    for (uint32_t win = 0; win < windows; ++win) {
        const uint32_t bits = wbits[win];
        if (bits == 0u) continue;
        const uint32_t s = win * 32u + lane;
        const int j = owner_lane(it.off, s);
        const uint32_t j_off = __shfl_sync(0xffffffffu, it.off, j);
        const uint32_t j_first = __shfl_sync(0xffffffffu, it.first, j);
        const uint32_t j_inst = __shfl_sync(0xffffffffu, it.inst, j);
        const uint32_t j_lod = __shfl_sync(0xffffffffu, it.lod, j);
        if ((bits >> lane) & 1u) {
            const uint32_t slot = base + __popc(bits & ((1u << lane) - 1u));
            if (slot < P.capacity) {
                const uint32_t mi = j_first + (s - j_off);
                const uint4 d = __ldg(S.m_draw + mi);
                uint32_t* o = reinterpret_cast<uint32_t*>(P.indirect + slot);
                o[0] = d.y;  // index_count
                o[1] = 1u;
                o[2] = d.x;  // first_index
                o[3] = d.z;  // vertex_offset
                o[4] = slot; // first_instance
                reinterpret_cast<uint4*>(P.draws)[slot] = make_uint4(j_inst, mi, j_lod, 0u);
            }
        }
        base += __popc(bits);
    }
}

}  // namespace

void launch_pack_meshlets(const HelioGpuMeshletEntry* aos, uint32_t n, float4* bounds, float4* cone, float4* axis,
                          uint4* draw, cudaStream_t stream) {
    if (!n) return;
    uint32_t blocks = (n + 255u) / 256u;
    if (blocks > 148u * 16u) blocks = 148u * 16u;
    helio_launch_begin("pack_meshlets", stream);
    pack_meshlets_kernel<<<blocks, 256, 0, stream>>>(aos, n, bounds, cone, axis, draw);
    helio_launch_end(stream);
}

void launch_instance_cull_data(const HelioGpuInstanceData* inst, uint32_t n, HelioInstanceCullData* out,
                               cudaStream_t stream) {
    if (!n) return;
    uint32_t blocks = (n + 255u) / 256u;
    if (blocks > 148u * 16u) blocks = 148u * 16u;
    helio_launch_begin("instance_cull_data", stream);
    instance_cull_data_kernel<<<blocks, 256, 0, stream>>>(inst, n, out);
    helio_launch_end(stream);
}

void launch_vg_view_setup(const ViewSetupParams& p, cudaStream_t stream) {
    helio_launch_begin("vg_view_setup", stream);
    vg_view_setup_kernel<<<1, 32, 0, stream>>>(p);
    helio_launch_end(stream);
}

void launch_vg_select(const VgSelectParams& p, cudaStream_t stream) {
    if (!p.scene.object_count) return;
    helio_launch_begin("vg_select", stream);
    vg_select_kernel<<<(p.scene.object_count + 255u) / 256u, 256, 0, stream>>>(p);
    helio_launch_end(stream);
}

namespace {

// The meshlet tests and the emission are launched with programmatic stream serialization:
// each may be scheduled while the kernel before it finishes (its CTAs wait in pdl_wait), which
// hides a launch gap per kernel.
cudaError_t launch_after(void (*kernel)(VgCullParams), uint32_t grid, const VgCullParams& p, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kCullWarps * 32);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, p);
}

}  // namespace

cudaError_t launch_vg_cull(const VgCullParams& p, cudaStream_t stream) {
    if (!p.num_tiles) return cudaSuccess;
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const bool wide = p.items_per_warp >= 32u && p.num_tiles > 4u * (uint32_t)std::max(sms, 1);
    helio_launch_begin("vg_cull_test", stream);
    cudaError_t e = launch_after(wide ? vg_cull_test_kernel<true> : vg_cull_test_kernel<false>, p.num_tiles, p, stream);
    helio_launch_end(stream);
    if (e != cudaSuccess) return e;
    helio_launch_begin("vg_cull_emit", stream);
    e = launch_after(vg_cull_emit_kernel, p.num_tiles, p, stream);
    helio_launch_end(stream);
    return e;
}

}  // namespace helio
