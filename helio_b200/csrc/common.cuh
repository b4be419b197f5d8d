// common.cuh — device-side arithmetic in the reference WGSL operation order.
//
// Every float operation goes through a correctly-rounded intrinsic (__fadd_rn,
// __fmul_rn, __fdiv_rn, __fsqrt_rn), so no FMA contraction or approximate
// division can change a visibility / LOD / mip decision, whatever the compiler
// flags. The rules (identical on every path of this library):
//   dot(a, b)      = (a.x*b.x + a.y*b.y) + a.z*b.z
//   M * vec4(p,1)  = ((M[0]*p.x + M[1]*p.y) + M[2]*p.z) + M[3]      (column sums)
//   mat3 * v       = (N[0]*v.x + N[1]*v.y) + N[2]*v.z
//   length(v)      = sqrt(dot(v, v)),  normalize(v) = v / length(v)
//   max / min      = fmaxf / fminf,  clamp(x, lo, hi) = fminf(fmaxf(x, lo), hi)
//   u32(ceil(log2(d))) for d >= 1 is exact, from the binary32 exponent/mantissa
//   textureSampleLevel (nearest, clamp-to-edge):
//       level = min(mip, mip_count - 1); i = clamp(floor(u * W_level), 0, W_level - 1)
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/helio_cull.h"

namespace helio {

struct F3 {
    float x, y, z;
};

__device__ __forceinline__ F3 f3(float x, float y, float z) { return F3{x, y, z}; }
__device__ __forceinline__ float fadd(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fsqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ F3 sub3(F3 a, F3 b) { return f3(fsub(a.x, b.x), fsub(a.y, b.y), fsub(a.z, b.z)); }
__device__ __forceinline__ F3 muls3(F3 a, float s) { return f3(fmul(a.x, s), fmul(a.y, s), fmul(a.z, s)); }
__device__ __forceinline__ F3 divs3(F3 a, float s) { return f3(fdiv(a.x, s), fdiv(a.y, s), fdiv(a.z, s)); }
__device__ __forceinline__ float dot3(F3 a, F3 b) {
    return fadd(fadd(fmul(a.x, b.x), fmul(a.y, b.y)), fmul(a.z, b.z));
}
__device__ __forceinline__ float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// ── Exact `a / b <= thr` without the correctly rounded division in clear cases ──
// r = rcp.approx.f32(b) has at most 1 ulp of error (PTX ISA), so q = RN(a * r)
// lies within 2^-22 (relative) of a / b. With margins of |thr| * 2^-18 on either
// side of thr, q below the lower margin proves RN(a / b) <= thr and q above the
// upper margin proves RN(a / b) > thr; everything in between (and NaN) takes the
// correctly rounded division. The margins are -inf / +inf (always exact) unless
// 2^-60 <= |thr| <= 2^60, and r is NaN (always exact) unless 2^-64 <= b <= 2^64,
// which keeps q clear of underflow relative to thr.
struct QuotientBound {
    float thr, lo, hi;
};

__device__ __forceinline__ QuotientBound quotient_bound(float thr) {
    const float at = fabsf(thr);
    if (at >= 0x1p-60f && at <= 0x1p60f) {
        const float m = fmul(at, 0x1p-18f);
        return QuotientBound{thr, fsub(thr, m), fadd(thr, m)};
    }
    return QuotientBound{thr, -__int_as_float(0x7f800000), __int_as_float(0x7f800000)};
}

__device__ __forceinline__ float quotient_rcp(float b) {
    if (!(b >= 0x1p-64f && b <= 0x1p64f)) return __int_as_float(0x7fffffff);
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(b));
    return r;
}

// RN(a / b) <= q.thr, bit-for-bit; r = quotient_rcp(b).
__device__ __forceinline__ bool quotient_le(float a, float b, float r, const QuotientBound& q) {
    const float approx = fmul(a, r);
    if (approx < q.lo) return true;
    if (approx > q.hi) return false;
    return fdiv(a, b) <= q.thr;
}

// Column-major 4x4 matrix held as four columns.
struct Mat4 {
    float4 c0, c1, c2, c3;
};

__device__ __forceinline__ Mat4 load_mat4(const float* m) {
    const float4* p = reinterpret_cast<const float4*>(m);
    return Mat4{p[0], p[1], p[2], p[3]};
}
__device__ __forceinline__ Mat4 ldg_mat4(const float* m) {
    const float4* p = reinterpret_cast<const float4*>(m);
    return Mat4{__ldg(p), __ldg(p + 1), __ldg(p + 2), __ldg(p + 3)};
}

// (M * vec4(p, 1)).xyz
__device__ __forceinline__ F3 mat4_point3(const Mat4& m, F3 p) {
    return f3(fadd(fadd(fadd(fmul(m.c0.x, p.x), fmul(m.c1.x, p.y)), fmul(m.c2.x, p.z)), m.c3.x),
              fadd(fadd(fadd(fmul(m.c0.y, p.x), fmul(m.c1.y, p.y)), fmul(m.c2.y, p.z)), m.c3.y),
              fadd(fadd(fadd(fmul(m.c0.z, p.x), fmul(m.c1.z, p.y)), fmul(m.c2.z, p.z)), m.c3.z));
}
// M * vec4(p, 1), all four components.
__device__ __forceinline__ float4 mat4_point4(const Mat4& m, F3 p) {
    F3 xyz = mat4_point3(m, p);
    float w = fadd(fadd(fadd(fmul(m.c0.w, p.x), fmul(m.c1.w, p.y)), fmul(m.c2.w, p.z)), m.c3.w);
    return make_float4(xyz.x, xyz.y, xyz.z, w);
}
// mat3(n0.xyz, n1.xyz, n2.xyz) * v
__device__ __forceinline__ F3 mat3_vec(float4 n0, float4 n1, float4 n2, F3 v) {
    return f3(fadd(fadd(fmul(n0.x, v.x), fmul(n1.x, v.y)), fmul(n2.x, v.z)),
              fadd(fadd(fmul(n0.y, v.x), fmul(n1.y, v.y)), fmul(n2.y, v.z)),
              fadd(fadd(fmul(n0.z, v.x), fmul(n1.z, v.y)), fmul(n2.z, v.z)));
}

// Exact u32(ceil(log2(d))) for d >= 1; values >= 2^32 (and +inf) give 0xFFFFFFFF.
__device__ __forceinline__ uint32_t ceil_log2_exact(float d) {
    if (!(d >= 1.0f)) return 0u;
    if (d >= 4294967296.0f) return 0xFFFFFFFFu;
    uint32_t bits = __float_as_uint(d);
    uint32_t e = ((bits >> 23) & 0xFFu) - 127u;
    return (bits & 0x7FFFFFu) ? e + 1u : e;
}

// Hi-Z pyramid as passed to kernels (a copy of helio_hiz_pyramid in param space).
struct HizView {
    const float* levels[HELIO_HIZ_MAX_MIPS];
    uint32_t width[HELIO_HIZ_MAX_MIPS];
    uint32_t height[HELIO_HIZ_MAX_MIPS];
    uint32_t pitch[HELIO_HIZ_MAX_MIPS];
    uint32_t mip_count;
};

// Copy with static indices (kernel parameters must not be indexed dynamically).
__device__ __forceinline__ void copy_hiz(const HizView& src, HizView& dst) {
#pragma unroll
    for (int l = 0; l < HELIO_HIZ_MAX_MIPS; ++l) {
        dst.levels[l] = src.levels[l];
        dst.width[l] = src.width[l];
        dst.height[l] = src.height[l];
        dst.pitch[l] = src.pitch[l];
    }
    dst.mip_count = src.mip_count;
}

// kCoherent: the pyramid was written earlier in the same launch, so it is read
// through L2 (ld.global.cg) instead of the read-only path.
template <bool kCoherent = false>
__device__ __forceinline__ float hiz_sample(const HizView& hz, float u, float v, uint32_t mip) {
    uint32_t l = min(mip, hz.mip_count - 1u);
    uint32_t w = hz.width[l], h = hz.height[l];
    // u, v lie in [0, 1] at every call site, so the products lie in [0, w] / [0, h].
    int ix = (int)floorf(fmul(u, (float)w));
    int iy = (int)floorf(fmul(v, (float)h));
    ix = min(max(ix, 0), (int)w - 1);
    iy = min(max(iy, 0), (int)h - 1);
    const float* p = hz.levels[l] + (size_t)iy * hz.pitch[l] + ix;
    return kCoherent ? __ldcg(p) : __ldg(p);
}

// Frustum planes as published by vg_cull.wgsl:266-280 (GPU form, no length guard).
struct Planes {
    float4 p[6];
};

// p / length(p.xyz) for the six Gribb–Hartmann rows of view_proj (column-major).
__device__ __forceinline__ Planes publish_planes(const float* vp) {
    auto e = [&](int c, int r) { return vp[c * 4 + r]; };
    float p[6][4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        p[0][c] = fadd(e(c, 3), e(c, 0));
        p[1][c] = fsub(e(c, 3), e(c, 0));
        p[2][c] = fadd(e(c, 3), e(c, 1));
        p[3][c] = fsub(e(c, 3), e(c, 1));
        p[4][c] = e(c, 2);
        p[5][c] = fsub(e(c, 3), e(c, 2));
    }
    Planes out;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        float len = fsqrt(dot3(f3(p[i][0], p[i][1], p[i][2]), f3(p[i][0], p[i][1], p[i][2])));
        out.p[i] = make_float4(fdiv(p[i][0], len), fdiv(p[i][1], len), fdiv(p[i][2], len), fdiv(p[i][3], len));
    }
    return out;
}

// The same planes computed by lanes 0..5 of one warp in parallel (lane i builds
// plane i); every lane of the warp must call it. Writes `out` (shared memory).
__device__ __forceinline__ void publish_planes_warp(const float* vp, Planes& out) {
    const int lane = threadIdx.x & 31;
    if (lane < 6) {
        float p[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float r3 = __ldg(vp + c * 4 + 3);
            const float rr = __ldg(vp + c * 4 + (lane >> 1));  // rows 0,0,1,1,2,2
            if (lane == 4) p[c] = __ldg(vp + c * 4 + 2);
            else if (lane == 5) p[c] = fsub(r3, __ldg(vp + c * 4 + 2));
            else if (lane & 1) p[c] = fsub(r3, rr);
            else p[c] = fadd(r3, rr);
        }
        const float len = fsqrt(dot3(f3(p[0], p[1], p[2]), f3(p[0], p[1], p[2])));
        out.p[lane] = make_float4(fdiv(p[0], len), fdiv(p[1], len), fdiv(p[2], len), fdiv(p[3], len));
    }
    __syncwarp();
}

// sphere_visible, vg_cull.wgsl:126-133: every plane satisfies dot(n, c) + d >= -r.
__device__ __forceinline__ bool sphere_visible_vg(const Planes& pl, F3 c, float r) {
    float nr = -r;
    bool v = true;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        float d = fadd(dot3(f3(pl.p[i].x, pl.p[i].y, pl.p[i].z), c), pl.p[i].w);
        v = v && (d >= nr);
    }
    return v;
}

// Programmatic dependent launch. A kernel launched with programmatic stream serialization
// may start while the previous kernel of its stream still runs; pdl_wait returns once that
// kernel has completed and its writes are visible (at once in a kernel launched normally), so
// it goes before the first read of anything the previous kernel wrote. pdl_launch_dependents
// lets the stream's next kernel, when so launched, be scheduled once every CTA of this kernel
// has called it or ended.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Device error word values.
enum : uint32_t { kDevOk = 0u, kDevTimeout = 1u };

constexpr uint32_t kSpinLimit = 1u << 22;  // polls before a bounded wait gives up (~1 s with backoff)

}  // namespace helio

// Host-side launch accounting (helio_kernel_launch_count) and the optional
// event profiler (helio_profiler_*): every launch is bracketed by these two calls.
void helio_launch_begin(const char* kernel, cudaStream_t stream);
void helio_launch_end(cudaStream_t stream);
// Counts one more launch inside an open begin/end bracket (a step of several kernels).
void helio_launch_note(void);
// Records `message` as the calling thread's helio_last_error() and returns `code`.
int32_t helio_report_error(int32_t code, const char* message);
