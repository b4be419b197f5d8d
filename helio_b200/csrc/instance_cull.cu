// instance_cull.cu — per-draw frustum + sub-pixel cull (IndirectDispatchPass) and
// per-draw Hi-Z occlusion cull (OcclusionCullPass), separately or fused.
//
// References:
//   crates/helio-pass-indirect-dispatch/shaders/indirect_dispatch.wgsl:79-176
//   crates/helio-pass-occlusion-cull/shaders/occlusion_cull.wgsl:101-259 (the static
//     Hi-Z branch, :222-259, when the pass has a baked grid: static_hiz_occludes)
// One thread per draw call, in a grid-stride loop over the draws. Statistics are
// aggregated per warp (ballot + popc) and per block before one atomic per block and
// slot; the totals equal the reference's per-thread atomics.

#include <algorithm>

#include "common.cuh"
#include "kernels.h"
#include "instance_cull.h"

namespace helio {

namespace {

// Linear-filtered fetch of level 0 of the static Hi-Z at normalised (x, y, z), clamp to
// edge: per axis t = x * n - 0.5, taps floor(t) and floor(t) + 1 clamped to [0, n - 1],
// weight frac(t) rounded to 8 fractional bits; x, then y, then z, each (1 - w) a + w b.
struct StaticTap {
    uint32_t i0, i1;
    float w;
};

__device__ __forceinline__ StaticTap static_tap(float x, uint32_t n) {
    const float t = fsub(fmul(x, (float)n), 0.5f);
    const float fl = floorf(t);
    const float w = fdiv(rintf(fmul(fsub(t, fl), 256.0f)), 256.0f);
    const int i = (int)fl;
    const int hi = (int)n - 1;
    return StaticTap{(uint32_t)min(max(i, 0), hi), (uint32_t)min(max(i + 1, 0), hi), w};
}

__device__ __forceinline__ float static_lerp(float a, float b, float w) {
    return fadd(fmul(fsub(1.0f, w), a), fmul(w, b));
}

__device__ float static_hiz_sample(const InstanceCullParams& P, float x, float y, float z) {
    const uint32_t W = P.static_dims[0], H = P.static_dims[1], D = P.static_dims[2] * 6u;
    const StaticTap tx = static_tap(x, W), ty = static_tap(y, H), tz = static_tap(z, D);
    const float* T = P.static_texels;
    auto at = [&](uint32_t i, uint32_t j, uint32_t k) { return __ldg(T + ((size_t)k * H + j) * W + i); };
    const float c00 = static_lerp(at(tx.i0, ty.i0, tz.i0), at(tx.i1, ty.i0, tz.i0), tx.w);
    const float c10 = static_lerp(at(tx.i0, ty.i1, tz.i0), at(tx.i1, ty.i1, tz.i0), tx.w);
    const float c01 = static_lerp(at(tx.i0, ty.i0, tz.i1), at(tx.i1, ty.i0, tz.i1), tx.w);
    const float c11 = static_lerp(at(tx.i0, ty.i1, tz.i1), at(tx.i1, ty.i1, tz.i1), tx.w);
    return static_lerp(static_lerp(c00, c10, ty.w), static_lerp(c01, c11, ty.w), tz.w);
}

// The static Hi-Z test (occlusion_cull.wgsl:222-259): true = occluded.
__device__ bool static_hiz_occludes(const InstanceCullParams& P, F3 center, F3 cam_pos) {
    const F3 d = sub3(center, cam_pos);
    const float dist = fsqrt(dot3(d, d));
    if (!(dist > 0.001f)) return false;
    const F3 v = f3(fdiv(d.x, dist), fdiv(d.y, dist), fdiv(d.z, dist));
    const float ax = fabsf(v.x), ay = fabsf(v.y), az = fabsf(v.z);
    uint32_t layer;
    if (ax >= ay && ax >= az) layer = v.x < 0.0f ? 1u : 0u;
    else if (ay >= az) layer = v.y < 0.0f ? 3u : 2u;
    else layer = v.z < 0.0f ? 5u : 4u;
    const float u = clampf(fdiv(fsub(center.x, P.static_min[0]), fsub(P.static_max[0], P.static_min[0])), 0.0f, 1.0f);
    const float vv = clampf(fdiv(fsub(center.y, P.static_min[1]), fsub(P.static_max[1], P.static_min[1])), 0.0f, 1.0f);
    const float w0 = clampf(fdiv(fsub(center.z, P.static_min[2]), fsub(P.static_max[2], P.static_min[2])), 0.0f, 1.0f);
    const float w = fdiv(fadd(w0, (float)layer), 6.0f);
    const float occ = static_hiz_sample(P, u, vv, w);
    return dist > fadd(occ, 0.1f);
}

// One draw (indirect_dispatch.wgsl:100-176 and / or occlusion_cull.wgsl:146-220):
// writes its indirect record and returns which statistics it adds to (bit s = slot s).
template <bool kFrustum, bool kOcclusion>
__device__ __forceinline__ uint32_t cull_draw(const InstanceCullParams& P, const HizView& s_hiz, uint32_t idx,
                                              bool active) {
    bool c_total = false, c_frustum = false, c_subpixel = false, c_visible = false, c_shadow = false,
         c_shadow_vis = false, c_occ = false, c_shadow_occ = false;

    if (active && P.draw_calls[idx].first_instance >= P.instance_count) {
        // A draw whose representative instance lies outside the instance buffer has
        // no bounds to test: it is written as frustum-culled and not occlusion-tested.
        if (kFrustum) {
            const HelioGpuDrawCall dc = P.draw_calls[idx];
            uint32_t* o = P.indirect + (size_t)idx * 5;
            o[0] = dc.index_count;
            o[1] = 0u;
            o[2] = dc.first_index;
            o[3] = (uint32_t)dc.vertex_offset;
            o[4] = dc.first_instance;
            c_frustum = true;
            c_total = true;
        }
    } else if (active) {
        const HelioGpuDrawCall dc = P.draw_calls[idx];
        const uint32_t ii = dc.first_instance;
        const float4 bounds = __ldg(reinterpret_cast<const float4*>(P.instances[ii].bounds));
        const uint32_t flags = __ldg(&P.instances[ii].flags);
        const HelioGpuCameraUniforms* cam = P.camera;
        const Mat4 vp = ldg_mat4(cam->view_proj);
        const F3 center = f3(bounds.x, bounds.y, bounds.z);
        const float radius = bounds.w;
        uint32_t instance_count_out = 0u;  // value of indirect[idx].instance_count after the frustum stage

        if (kFrustum) {
            const float4 amin = __ldg(reinterpret_cast<const float4*>(P.aabbs[ii].min));
            const float4 amax = __ldg(reinterpret_cast<const float4*>(P.aabbs[ii].max));
            // aabb_in_frustum (:88-98)
            bool aabb_visible = true;
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                const float* pl = P.planes + i * 4;
                float px = pl[0] >= 0.0f ? amax.x : amin.x;
                float py = pl[1] >= 0.0f ? amax.y : amin.y;
                float pz = pl[2] >= 0.0f ? amax.z : amin.z;
                float dist = fadd(dot3(f3(pl[0], pl[1], pl[2]), f3(px, py, pz)), pl[3]);
                aabb_visible = aabb_visible && !(dist < 0.0f);
            }
            const bool degenerate = amin.x == amax.x && amin.y == amax.y && amin.z == amax.z;
            // sphere_in_frustum (:79-86)
            bool sphere_visible = true;
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                const float* pl = P.planes + i * 4;
                float dist = fadd(dot3(f3(pl[0], pl[1], pl[2]), center), pl[3]);
                sphere_visible = sphere_visible && !(fadd(dist, radius) < 0.0f);
            }
            const bool visible = degenerate ? sphere_visible : aabb_visible;
            bool should_draw = visible;
            if (visible) {
                const float4 clip = mat4_point4(vp, center);
                if (clip.w > 0.0f) {
                    const float p11 = __ldg(&cam->proj[5]);
                    float r_ndc = fabsf(fdiv(fmul(radius, p11), clip.w));
                    if (r_ndc < 0.001f) should_draw = false;
                }
            }
            const bool shadow = (flags & 1u) != 0u;
            c_shadow = shadow;
            instance_count_out = should_draw ? dc.instance_count : 0u;
            uint32_t* o = P.indirect + (size_t)idx * 5;
            o[0] = dc.index_count;
            o[1] = instance_count_out;
            o[2] = dc.first_index;
            o[3] = (uint32_t)dc.vertex_offset;
            o[4] = dc.first_instance;
            if (should_draw) {
                c_visible = true;
                c_shadow_vis = shadow;
            } else if (!visible) {
                c_frustum = true;
            } else {
                c_subpixel = true;
            }
            c_total = true;
        }

        if (kOcclusion) {
            bool occluded = false;
            if (radius > 0.0f) {
                const float4 clip = mat4_point4(vp, center);
                if (clip.w > 0.0f) {
                    const float p00 = __ldg(&cam->proj[0]), p11 = __ldg(&cam->proj[5]);
                    const float ndc_x = fdiv(clip.x, clip.w), ndc_y = fdiv(clip.y, clip.w);
                    const float uv_x = fadd(fmul(ndc_x, 0.5f), 0.5f), uv_y = fadd(fmul(ndc_y, -0.5f), 0.5f);
                    const float ndc_r = fmaxf(fabsf(fdiv(fmul(radius, p00), clip.w)), fabsf(fdiv(fmul(radius, p11), clip.w)));
                    const bool off = fadd(ndc_x, ndc_r) < -1.0f || fsub(ndc_x, ndc_r) > 1.0f ||
                                     fadd(ndc_y, ndc_r) < -1.0f || fsub(ndc_y, ndc_r) > 1.0f;
                    if (!off) {
                        // sphere_near_depth (:124-140)
                        const float4 pn = __ldg(reinterpret_cast<const float4*>(cam->position_near));
                        const F3 tc = sub3(center, f3(pn.x, pn.y, pn.z));
                        const float dist_sq = dot3(tc, tc);
                        float near_z = 0.0f;
                        if (!(dist_sq <= fmul(radius, radius))) {
                            const F3 dir = muls3(tc, fdiv(1.0f, fsqrt(dist_sq)));
                            const F3 nws = sub3(center, muls3(dir, radius));
                            const float4 nc = mat4_point4(vp, nws);
                            near_z = nc.w <= 0.0f ? 0.0f : clampf(fdiv(nc.z, nc.w), 0.0f, 1.0f);
                        }
                        // screen_radius_px (:110-113), pick_mip (:116-120)
                        const float half_h = fmul((float)P.screen_h, 0.5f);
                        const float r_px = fabsf(fmul(fmul(fdiv(radius, clip.w), p11), half_h));
                        const float diameter = fmaxf(fmul(r_px, 2.0f), 1.0f);
                        const uint32_t mip = min(ceil_log2_exact(diameter), P.hiz_mip_count - 1u);
                        const float uv_half = fmul(ndc_r, 0.5f);
                        const float u0 = clampf(fsub(uv_x, uv_half), 0.0f, 1.0f), v0 = clampf(fsub(uv_y, uv_half), 0.0f, 1.0f);
                        const float u1 = clampf(fadd(uv_x, uv_half), 0.0f, 1.0f), v1 = clampf(fadd(uv_y, uv_half), 0.0f, 1.0f);
                        const float h00 = hiz_sample(s_hiz, u0, v0, mip);
                        const float h01 = hiz_sample(s_hiz, u1, v0, mip);
                        const float h10 = hiz_sample(s_hiz, u0, v1, mip);
                        const float h11 = hiz_sample(s_hiz, u1, v1, mip);
                        const float hz = fmaxf(fmaxf(h00, h01), fmaxf(h10, h11));
                        occluded = near_z > fadd(hz, 1.0f / 65536.0f);
                        if (!occluded && P.static_texels)
                            occluded = static_hiz_occludes(P, center, f3(pn.x, pn.y, pn.z));
                    }
                }
            }
            if (occluded) {
                uint32_t* ic = P.indirect + (size_t)idx * 5 + 1;
                const bool was_visible = kFrustum ? (instance_count_out != 0u) : (*ic != 0u);
                *ic = 0u;
                if (was_visible) {
                    c_occ = true;
                    c_shadow_occ = (flags & 1u) != 0u;
                }
            }
        }
    }

    const bool conds[8] = {c_total, c_frustum, c_subpixel, c_visible, c_occ, c_shadow, c_shadow_vis, c_shadow_occ};
    uint32_t bits = 0u;
#pragma unroll
    for (int k = 0; k < 8; ++k) bits |= conds[k] ? (1u << k) : 0u;
    return bits;
}

// Grid-stride over the draws, one thread per draw per round. The statistics are summed
// per warp (ballot + popc) in lane 0's registers, per block in shared memory, and added
// to the global counters once per block and slot: the totals equal the reference's
// one atomic per thread, without thousands of atomics on the same 8 words.
template <bool kFrustum, bool kOcclusion>
__global__ void __launch_bounds__(256) instance_cull_kernel(InstanceCullParams P) {
    __shared__ HizView s_hiz;
    __shared__ uint32_t s_stats[8];
    if (threadIdx.x < 8) s_stats[threadIdx.x] = 0u;
    if (kOcclusion && threadIdx.x == 0) copy_hiz(P.hiz, s_hiz);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    uint32_t acc[8] = {0u, 0u, 0u, 0u, 0u, 0u, 0u, 0u};
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x; base < P.draw_count; base += stride) {
        const uint32_t idx = base + threadIdx.x;
        const uint32_t bits = cull_draw<kFrustum, kOcclusion>(P, s_hiz, idx, idx < P.draw_count);
#pragma unroll
        for (int k = 0; k < 8; ++k) acc[k] += __popc(__ballot_sync(0xffffffffu, (bits >> k) & 1u));
    }
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const bool used = kFrustum ? (k != 4 && k != 7) : (k == 4 || k == 7);
            if ((used || (kFrustum && kOcclusion)) && acc[k]) atomicAdd(&s_stats[k], acc[k]);
        }
    }
    __syncthreads();
    if (threadIdx.x < 8 && s_stats[threadIdx.x]) atomicAdd(P.stats + threadIdx.x, s_stats[threadIdx.x]);
}

}  // namespace

void launch_instance_cull(const InstanceCullParams& p, bool frustum, bool occlusion, cudaStream_t stream) {
    if (p.draw_count == 0) return;
    if (!frustum && !occlusion) return;
    // Enough blocks to fill every SM 8 deep; each takes its share of the draws.
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);  // a cached attribute query
    if (sms < 1) sms = 1;
    const uint32_t blocks = std::min<uint32_t>((p.draw_count + 255u) / 256u, (uint32_t)sms * 8u);
    helio_launch_begin(frustum && occlusion ? "instance_cull_fused" : frustum ? "indirect_dispatch" : "occlusion_cull",
                       stream);
    if (frustum && occlusion) instance_cull_kernel<true, true><<<blocks, 256, 0, stream>>>(p);
    else if (frustum) instance_cull_kernel<true, false><<<blocks, 256, 0, stream>>>(p);
    else instance_cull_kernel<false, true><<<blocks, 256, 0, stream>>>(p);
    helio_launch_end(stream);
}

}  // namespace helio
