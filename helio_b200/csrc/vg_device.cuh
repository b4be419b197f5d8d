// vg_device.cuh — device functions of the meshlet cull shared by the single-view
// kernels (vg_cull.cu) and the persistent multi-view kernel (batch.cu).
#pragma once

#include "common.cuh"
#include "vg.h"

namespace helio {

__device__ __forceinline__ HelioInstanceCullData load_cull(const HelioInstanceCullData* p) {
    const uint4 q = __ldg(reinterpret_cast<const uint4*>(p));
    HelioInstanceCullData r;
    r.max_scale = __uint_as_float(q.x);
    r.min_scale = __uint_as_float(q.y);
    r.cone_cull_enabled = q.z;
    r.valid_transform = q.w;
    return r;
}

// Cooperative copy of view constants into shared memory (16-byte words).
__device__ __forceinline__ void load_view(const CullView* src, CullView& dst, int tid, int nthreads) {
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(&dst);
    for (int k = tid; k < (int)(sizeof(CullView) / 16); k += nthreads) d[k] = __ldg(s + k);
}

__device__ __forceinline__ float rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// The cone test's decision dot(cta / |cta|, a / |a|) >= cutoff (vg_cull.wgsl:172-180),
// bit-for-bit. The reference value E normalises both vectors with a correctly rounded
// square root and three divisions each, then takes the dot product; it lies within
// about 10 ulp(1) of the real cosine R (both vectors are unit length after
// normalisation, so every term is at most 1). D = fma-dot(cta, a) * rsqrt.approx(|cta|^2)
// * rsqrt.approx(|a|^2) lies within about 16 ulp(1) of R: 3 roundings in the dot
// (relative to sum |cta_i a_i| <= |cta||a|), at most 2^-22.9 relative error in each
// rsqrt.approx (PTX ISA) plus the squared norms' own rounding, and two products. So
// |D - E| < 2^-19, and D outside cutoff +- 2^-16 decides the comparison; everything
// else (and squared norms outside [1e-30, 1e30], non-finite values) takes the
// reference's own sequence.
__device__ __forceinline__ bool cone_rejects(F3 a, F3 cta, float ads, float cutoff) {
    const float da = dot3(a, a);
    if (da >= 1.0e-30f && da <= 1.0e30f && ads <= 1.0e30f) {
        const float t = fmaf(cta.z, a.z, fmaf(cta.y, a.y, cta.x * a.x));
        const float d = t * rsqrt_approx(ads) * rsqrt_approx(da);
        if (isfinite(d)) {
            if (d >= cutoff + 0x1p-16f) return true;
            if (d < cutoff - 0x1p-16f) return false;
        }
    }
    const F3 axis_ws = divs3(a, fsqrt(da));
    return dot3(divs3(cta, fsqrt(ads)), axis_ws) >= cutoff;
}

// World-space bounding sphere of meshlet mi of an instance (vg_cull.wgsl:150-152).
__device__ __forceinline__ void meshlet_sphere(const VgSceneDev& S, uint32_t mi, const Mat4& model,
                                               const HelioInstanceCullData& cd, F3& c, float& wr) {
    const float4 b = __ldg(S.m_bounds + mi);
    c = mat4_point3(model, f3(b.x, b.y, b.z));
    wr = fmaxf(fmul(b.w, cd.max_scale), 0.0f);
}

// Everything the frustum and cone tests read of one meshlet of one instance,
// loaded in one go (one memory round trip instead of one per test).
struct MeshletInputs {
    float4 bounds, cone, axis;
    float4 n0, n1, n2;  // the instance's normal matrix columns
};

__device__ __forceinline__ MeshletInputs load_meshlet(const VgSceneDev& S, uint32_t mi,
                                                      const HelioGpuInstanceData* inst) {
    MeshletInputs m;
    m.bounds = __ldg(S.m_bounds + mi);
    m.cone = __ldg(S.m_cone + mi);
    m.axis = __ldg(S.m_axis + mi);
    const float4* nm = reinterpret_cast<const float4*>(inst->normal_mat);
    m.n0 = __ldg(nm);
    m.n1 = __ldg(nm + 1);
    m.n2 = __ldg(nm + 2);
    return m;
}

// cull_meshlet, first part (vg_cull.wgsl:143-182): the frustum and normal-cone
// tests. True = the meshlet is still a candidate and the Hi-Z test decides it;
// (c, wr) is its world-space sphere.
__device__ __forceinline__ bool meshlet_frustum_cone(const CullView& C, const MeshletInputs& m, const Mat4& model,
                                                     const HelioInstanceCullData& cd, F3& c, float& wr) {
    if (cd.valid_transform == 0u) return false;
    c = mat4_point3(model, f3(m.bounds.x, m.bounds.y, m.bounds.z));
    wr = fmaxf(fmul(m.bounds.w, cd.max_scale), 0.0f);
    if (!sphere_visible_vg(C.planes, c, wr)) return false;
    // Perspective normal-cone test (:159-182).
    if (cd.cone_cull_enabled != 0u) {
        const F3 cam = f3(C.pos_near.x, C.pos_near.y, C.pos_near.z);
        const F3 ctc = sub3(c, cam);
        const float cam_dist_sq = dot3(ctc, ctc);
        const float guard = fmul(wr, 1.5f);
        if (cam_dist_sq > fmul(guard, guard) && m.cone.w <= 1.0f) {
            const F3 a = mat3_vec(m.n0, m.n1, m.n2, f3(m.axis.x, m.axis.y, m.axis.z));
            const F3 apex = mat4_point3(model, f3(m.cone.x, m.cone.y, m.cone.z));
            const F3 cta = sub3(apex, cam);
            const float ads = dot3(cta, cta);
            if (ads > 1.0e-12f && cone_rejects(a, cta, ads, m.cone.w)) return false;
        }
    }
    return true;
}

// The same tests with the cone inputs (apex, axis, the instance's normal matrix) loaded
// only for meshlets whose sphere passes the frustum: fewer registers live at a time, for
// kernels that run more warps per SM instead of more loads per warp.
__device__ __forceinline__ bool meshlet_frustum_cone_lazy(const CullView& C, const VgSceneDev& S, uint32_t mi,
                                                          const HelioGpuInstanceData* inst, const Mat4& model,
                                                          const HelioInstanceCullData& cd, F3& c, float& wr) {
    if (cd.valid_transform == 0u) return false;
    const float4 b = __ldg(S.m_bounds + mi);
    c = mat4_point3(model, f3(b.x, b.y, b.z));
    wr = fmaxf(fmul(b.w, cd.max_scale), 0.0f);
    if (!sphere_visible_vg(C.planes, c, wr)) return false;
    if (cd.cone_cull_enabled != 0u) {
        const F3 cam = f3(C.pos_near.x, C.pos_near.y, C.pos_near.z);
        const F3 ctc = sub3(c, cam);
        const float cam_dist_sq = dot3(ctc, ctc);
        const float guard = fmul(wr, 1.5f);
        const float4 cone = __ldg(S.m_cone + mi);
        if (cam_dist_sq > fmul(guard, guard) && cone.w <= 1.0f) {
            const float4 axis = __ldg(S.m_axis + mi);
            const float4* nm = reinterpret_cast<const float4*>(inst->normal_mat);
            const F3 a = mat3_vec(__ldg(nm), __ldg(nm + 1), __ldg(nm + 2), f3(axis.x, axis.y, axis.z));
            const F3 apex = mat4_point3(model, f3(cone.x, cone.y, cone.z));
            const F3 cta = sub3(apex, cam);
            const float ads = dot3(cta, cta);
            if (ads > 1.0e-12f && cone_rejects(a, cta, ads, cone.w)) return false;
        }
    }
    return true;
}

// cull_meshlet, second part (vg_cull.wgsl:184-240): the conservative Hi-Z test of
// the sphere (c, wr). True = visible. kCoherentHiz: the pyramid was written
// earlier in the same launch.
template <bool kCoherentHiz = false>
__device__ __forceinline__ bool meshlet_hiz_visible(const CullView& C, F3 c, float wr) {
    const HizView& hz = C.hiz;
    const F3 ctc = sub3(c, f3(C.pos_near.x, C.pos_near.y, C.pos_near.z));
    const float4 clip = mat4_point4(C.vp, c);
    if (clip.w > 0.0f) {
        const float ndc_x = fdiv(clip.x, clip.w), ndc_y = fdiv(clip.y, clip.w);
        const float uv_x = fadd(fmul(ndc_x, 0.5f), 0.5f), uv_y = fadd(fmul(ndc_y, -0.5f), 0.5f);
        const float nvd = fsub(clip.w, wr);
        if (nvd > C.pos_near.w) {
            const float ndc_r = fmaxf(fabsf(fdiv(fmul(wr, C.p00), nvd)), fabsf(fdiv(fmul(wr, C.p11), nvd)));
            const float uvr = fmul(ndc_r, 0.5f);
            const float u0 = fsub(uv_x, uvr), v0 = fsub(uv_y, uvr), u1 = fadd(uv_x, uvr), v1 = fadd(uv_y, uvr);
            if (u0 >= 0.0f && v0 >= 0.0f && u1 <= 1.0f && v1 <= 1.0f) {
                // The four texel loads first: the sphere's nearest depth below is computed
                // while they are in flight (neither depends on the other).
                const float half_h = fmul((float)C.screen_height, 0.5f);
                const float dpx = fmaxf(fmul(fmul(ndc_r, half_h), 2.0f), 1.0f);
                const uint32_t mip = min(ceil_log2_exact(dpx), C.hiz_mip_count - 1u);
                const float h00 = hiz_sample<kCoherentHiz>(hz, u0, v0, mip);
                const float h01 = hiz_sample<kCoherentHiz>(hz, u1, v0, mip);
                const float h10 = hiz_sample<kCoherentHiz>(hz, u0, v1, mip);
                const float h11 = hiz_sample<kCoherentHiz>(hz, u1, v1, mip);
                const float dist_sq = dot3(ctc, ctc);
                float near_z = 0.0f;
                if (dist_sq > fmul(wr, wr)) {
                    const F3 dir = divs3(ctc, fsqrt(dist_sq));
                    const F3 nws = sub3(c, muls3(dir, wr));
                    const float4 nc = mat4_point4(C.vp, nws);
                    if (nc.w > 0.0f) near_z = clampf(fdiv(nc.z, nc.w), 0.0f, 1.0f);
                }
                const float hzv = fmaxf(fmaxf(h00, h01), fmaxf(h10, h11));
                if (near_z > fadd(hzv, 1.0f / 65536.0f)) return false;
            }
        }
    }
    return true;
}

// cull_meshlet decision part (vg_cull.wgsl:143-240): true = emit a draw. kLazyCone: the
// cone inputs are loaded after the frustum test (fewer live registers), else with the sphere.
template <bool kCoherentHiz = false, bool kLazyCone = false>
__device__ __forceinline__ bool meshlet_visible(const VgSceneDev& S, const CullView& C, uint32_t mi,
                                                const Mat4& model, const HelioInstanceCullData& cd,
                                                const HelioGpuInstanceData* inst) {
    F3 c;
    float wr;
    const bool cand = kLazyCone ? meshlet_frustum_cone_lazy(C, S, mi, inst, model, cd, c, wr)
                                : meshlet_frustum_cone(C, load_meshlet(S, mi, inst), model, cd, c, wr);
    if (!cand) return false;
    return meshlet_hiz_visible<kCoherentHiz>(C, c, wr);
}

// Largest lane j whose exclusive offset is <= s (for s below the warp total this
// is the item that owns window slot s; empty items are skipped because they share
// their offset with the next item).
__device__ __forceinline__ int owner_lane(uint32_t off, uint32_t s) {
    int lo = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
        const uint32_t o = __shfl_sync(0xffffffffu, off, lo + step);
        if (o <= s) lo += step;
    }
    return lo;
}

// Bits [off, off + n) (n <= 64) of a little-endian bit array of 32-bit words; the
// two words after the field's first word must be readable.
__device__ __forceinline__ uint2 bit_field64(const uint32_t* words, uint32_t off, uint32_t n) {
    if (n == 0) return make_uint2(0u, 0u);
    const uint32_t w0 = off >> 5, sh = off & 31u;
    const unsigned long long a = (unsigned long long)words[w0] | ((unsigned long long)words[w0 + 1] << 32);
    const unsigned long long c = words[w0 + 2];
    unsigned long long field = sh ? ((a >> sh) | (c << (64 - sh))) : a;
    if (n < 64) field &= (1ull << n) - 1ull;
    return make_uint2((uint32_t)field, (uint32_t)(field >> 32));
}

}  // namespace helio
