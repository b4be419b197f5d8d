// oracle.cpp — CPU restatement of Helio's GPU visibility path.
//
// TEST INFRASTRUCTURE ONLY (the reference the CUDA path is compared with): loaded by tests/, __graft_entry__.smoke()
// and bench.py's CPU-baseline / reference arm. Never linked into or called by the
// product library.
//
// Arithmetic rules (identical to the documented rules of the CUDA path, written
// independently here):
//   * binary32 everywhere, no contraction (-ffp-contract=off), IEEE '/' and sqrtf;
//   * dot(a, b)          = (a.x*b.x + a.y*b.y) + a.z*b.z
//   * M * vec4(p, 1)     = ((M[0]*p.x + M[1]*p.y) + M[2]*p.z) + M[3]   (column sums)
//   * mat3 * v           = (N[0]*v.x + N[1]*v.y) + N[2]*v.z
//   * length(v)          = sqrtf(dot(v, v)); normalize(v) = v / length(v)
//   * max/min            = fmaxf/fminf; clamp(x, lo, hi) = fminf(fmaxf(x, lo), hi)
//   * u32(ceil(log2(d))) = exact from the binary32 exponent/mantissa (d >= 1)
//   * textureSampleLevel, nearest + clamp-to-edge:
//       level = min(mip, mip_count-1); i = clamp(floor(u * W_level), 0, W_level-1)
// Expressions follow the WGSL source text left to right.
//
// Parity: pinned against the reference's own known-answer tests
// (tests/golden/reference_kats.json); the WGSL shaders themselves cannot run on
// either machine, so end-to-end execution of the reference is unpinned.

#include "oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

constexpr float kMarginRel = 1e-6f;

struct V3 {
    float x, y, z;
};

inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline float dot3(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3 divs(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
inline V3 muls(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline float clampf(float x, float lo, float hi) { return fminf(fmaxf(x, lo), hi); }

// M * vec4(p, 1.0) for a column-major 4x4 matrix: all four components.
inline void mat4_point(const float* m, V3 p, float out[4]) {
    for (int r = 0; r < 4; ++r) {
        out[r] = ((m[0 * 4 + r] * p.x + m[1 * 4 + r] * p.y) + m[2 * 4 + r] * p.z) + m[3 * 4 + r];
    }
}

// Relative closeness of two operands of a decision.
inline bool marginal(float a, float b) {
    float scale = fmaxf(fabsf(a), fabsf(b));
    if (!(scale > 0.0f)) return a == b;
    return fabsf(a - b) <= kMarginRel * scale;
}

struct Marg {
    uint64_t n = 0;
    void cmp(float a, float b) {
        if (marginal(a, b)) ++n;
    }
};

// Exact u32(ceil(log2(d))) for d >= 1 (d is max(.., 1.0), so never below 1).
// Values that do not fit return 0xFFFFFFFF, which the caller's clamp reduces.
uint32_t ceil_log2_exact(float d) {
    if (!(d >= 1.0f)) return 0u;                 // NaN cannot occur: fmaxf(NaN, 1) = 1
    if (d >= 4294967296.0f) return 0xFFFFFFFFu;  // includes +inf
    uint32_t bits;
    std::memcpy(&bits, &d, 4);
    uint32_t e = ((bits >> 23) & 0xFFu) - 127u;
    uint32_t mant = bits & 0x7FFFFFu;
    return mant == 0u ? e : e + 1u;
}

// Marginal when the mip's argument sits within the relative band of a power of two.
// `raw` is the value before the max(.., 1) clamp: a clamped 1.0 decides mip 0 however
// far below 1 the raw value lies, so only a raw value near 1 (or near a higher power
// of two) makes the mip choice marginal.
void mip_margin(float raw, Marg& mg) {
    if (!(raw >= 0.0f) || raw >= 4294967296.0f) return;
    if (raw < 1.0f) {
        mg.cmp(raw, 1.0f);
        return;
    }
    uint32_t k = ceil_log2_exact(raw);
    float hi = ldexpf(1.0f, (int)k);
    float lo = ldexpf(1.0f, (int)k - 1);
    mg.cmp(raw, hi);
    if (k > 0) mg.cmp(raw, lo);
}

float sample_nearest(const helio_hiz_pyramid* hz, float u, float v, uint32_t mip) {
    uint32_t l = std::min(mip, hz->mip_count - 1u);
    uint32_t w = hz->width[l], h = hz->height[l];
    float fx = floorf(u * (float)w);
    float fy = floorf(v * (float)h);
    // u, v are within [0, 1] at every call site, so fx, fy lie in [0, w], [0, h].
    int64_t ix = (int64_t)fx, iy = (int64_t)fy;
    ix = std::min<int64_t>(std::max<int64_t>(ix, 0), (int64_t)w - 1);
    iy = std::min<int64_t>(std::max<int64_t>(iy, 0), (int64_t)h - 1);
    return hz->levels[l][(size_t)iy * hz->pitch[l] + (size_t)ix];
}

// GPU-side plane publication: vg_cull.wgsl:266-280 (no length guard).
void publish_frustum_planes(const float* vp, float planes[6][4]) {
    auto e = [&](int c, int r) { return vp[c * 4 + r]; };
    float p[6][4];
    for (int c = 0; c < 4; ++c) {
        p[0][c] = e(c, 3) + e(c, 0);
        p[1][c] = e(c, 3) - e(c, 0);
        p[2][c] = e(c, 3) + e(c, 1);
        p[3][c] = e(c, 3) - e(c, 1);
        p[4][c] = e(c, 2);
        p[5][c] = e(c, 3) - e(c, 2);
    }
    for (int i = 0; i < 6; ++i) {
        float len = sqrtf((p[i][0] * p[i][0] + p[i][1] * p[i][1]) + p[i][2] * p[i][2]);
        for (int c = 0; c < 4; ++c) planes[i][c] = p[i][c] / len;
    }
}

// sphere_visible, vg_cull.wgsl:126-133.
bool vg_sphere_visible(const float planes[6][4], V3 c, float r, Marg* mg) {
    bool vis = true;
    for (int i = 0; i < 6; ++i) {
        float d = dot3(v3(planes[i][0], planes[i][1], planes[i][2]), c) + planes[i][3];
        if (mg) mg->cmp(d, -r);
        if (!(d >= -r)) vis = false;
    }
    return vis;
}

template <typename F>
void parallel_chunks(uint64_t n, int threads, F&& fn) {
    if (threads <= 1 || n < 4096) {
        fn(0, 0, n);
        return;
    }
    std::vector<std::thread> pool;
    uint64_t chunk = (n + threads - 1) / threads;
    for (int t = 0; t < threads; ++t) {
        uint64_t b = std::min<uint64_t>(n, t * chunk), e = std::min<uint64_t>(n, b + chunk);
        pool.emplace_back([&, t, b, e] { fn(t, b, e); });
    }
    for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

// crates/helio-pass-hiz/src/lib.rs:376-379
uint32_t oracle_mip_levels(uint32_t w, uint32_t h) {
    uint32_t m = std::max(w, h);
    uint32_t bits = 0;
    while (m) {
        ++bits;
        m >>= 1;
    }
    return std::max(bits, 1u);
}

uint32_t oracle_ceil_log2(float d) { return ceil_log2_exact(d); }

int oracle_sphere_visible(const float planes[24], const float center[3], float radius) {
    float p[6][4];
    for (int i = 0; i < 24; ++i) p[i / 4][i % 4] = planes[i];
    return vg_sphere_visible(p, v3(center[0], center[1], center[2]), radius, nullptr) ? 1 : 0;
}

// Loop of vg_cull.wgsl:323-337 (the shader form; lib.rs:205-234 restates it on the CPU
// with an explicit max(closest, 1e-4), which the shader applies when forming `closest`).
uint32_t oracle_select_lod(const float errors[8], uint32_t lod_count, float max_scale, float focal_px,
                           float closest, float max_error_px) {
    uint32_t selected = 0;
    float denom = fmaxf(closest, 1.0e-4f);
    for (uint32_t level = 1; level < std::min(lod_count, 8u); ++level) {
        float err = ((errors[level] * max_scale) * focal_px) / denom;
        if (err <= max_error_px) selected = level;
        else break;
    }
    return selected;
}

int oracle_cone_reject(const float camera[3], const float apex[3], const float axis_ws[3], float cutoff) {
    V3 cta = sub(v3(apex[0], apex[1], apex[2]), v3(camera[0], camera[1], camera[2]));
    float ads = dot3(cta, cta);
    if (!(ads > 1.0e-12f)) return 0;
    return dot3(divs(cta, sqrtf(ads)), v3(axis_ws[0], axis_ws[1], axis_ws[2])) >= cutoff ? 1 : 0;
}

int oracle_hiz_occludes(float near_z, float hiz) { return near_z > hiz + 1.0f / 65536.0f ? 1 : 0; }

// crates/helio-pass-indirect-dispatch/src/lib.rs:271-300 (CPU, len > 1e-10 guard).
void oracle_extract_frustum_planes(const float vp[16], float planes[24]) {
    auto row = [&](int r, float out[4]) {
        out[0] = vp[r];
        out[1] = vp[4 + r];
        out[2] = vp[8 + r];
        out[3] = vp[12 + r];
    };
    float r0[4], r1[4], r2[4], r3[4];
    row(0, r0);
    row(1, r1);
    row(2, r2);
    row(3, r3);
    float p[6][4];
    for (int i = 0; i < 4; ++i) {
        p[0][i] = r3[i] + r0[i];
        p[1][i] = r3[i] - r0[i];
        p[2][i] = r3[i] + r1[i];
        p[3][i] = r3[i] - r1[i];
        p[4][i] = r2[i];
        p[5][i] = r3[i] - r2[i];
    }
    for (int k = 0; k < 6; ++k) {
        float len = sqrtf((p[k][0] * p[k][0] + p[k][1] * p[k][1]) + p[k][2] * p[k][2]);
        for (int i = 0; i < 4; ++i) planes[k * 4 + i] = (len > 1e-10f) ? p[k][i] / len : p[k][i];
    }
}

// InstanceCullData::from_instance, crates/helio-pass-virtual-geometry/src/lib.rs:132-167.
void oracle_instance_cull_data(const HelioGpuInstanceData* inst, uint32_t n,
                               HelioInstanceCullData* out) {
    for (uint32_t i = 0; i < n; ++i) {
        const float* m = inst[i].model;
        float sx = sqrtf((m[0] * m[0] + m[1] * m[1]) + m[2] * m[2]);
        float sy = sqrtf((m[4] * m[4] + m[5] * m[5]) + m[6] * m[6]);
        float sz = sqrtf((m[8] * m[8] + m[9] * m[9]) + m[10] * m[10]);
        float max_scale = fmaxf(fmaxf(sx, sy), sz);
        float min_scale = fminf(fminf(sx, sy), sz);
        float dot_xy = (m[0] * m[4] + m[1] * m[5]) + m[2] * m[6];
        float dot_xz = (m[0] * m[8] + m[1] * m[9]) + m[2] * m[10];
        float dot_yz = (m[4] * m[8] + m[5] * m[9]) + m[6] * m[10];
        float det = (m[0] * (m[5] * m[10] - m[6] * m[9]) - m[4] * (m[1] * m[10] - m[2] * m[9])) +
                    m[8] * (m[1] * m[6] - m[2] * m[5]);
        bool affine = fabsf(m[3]) <= 1.0e-6f && fabsf(m[7]) <= 1.0e-6f &&
                      fabsf(m[11]) <= 1.0e-6f && fabsf(m[15] - 1.0f) <= 1.0e-4f;
        bool finite = true;
        for (int k = 0; k < 16; ++k) finite = finite && std::isfinite(m[k]);
        bool valid = finite && std::isfinite(max_scale) && min_scale > 1.0e-8f && affine;
        float ut = max_scale * 1.0e-4f;
        float ot = (max_scale * max_scale) * 1.0e-4f;
        bool ap = (max_scale - min_scale) <= ut && fabsf(dot_xy) <= ot && fabsf(dot_xz) <= ot &&
                  fabsf(dot_yz) <= ot;
        bool cone = valid && ap && det > 0.0f;
        out[i].max_scale = valid ? max_scale : 0.0f;
        out[i].min_scale = valid ? min_scale : 0.0f;
        out[i].cone_cull_enabled = cone ? 1u : 0u;
        out[i].valid_transform = valid ? 1u : 0u;
    }
}

// hiz_depth_copy.wgsl:13-19, then hiz_build.wgsl:12-23 once per level
// (crates/helio-pass-hiz/src/lib.rs:201-225, 516-531).
uint32_t oracle_hiz_build(const float* depth, uint32_t w, uint32_t h, uint32_t pitch,
                          float* const* levels) {
    uint32_t mips = std::min(oracle_mip_levels(w, h), (uint32_t)HELIO_HIZ_MAX_MIPS);
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) levels[0][(size_t)y * w + x] = depth[(size_t)y * pitch + x];
    for (uint32_t mip = 0; mip + 1 < mips; ++mip) {
        uint32_t sw = std::max(w >> mip, 1u), sh = std::max(h >> mip, 1u);
        uint32_t dw = std::max(w >> (mip + 1), 1u), dh = std::max(h >> (mip + 1), 1u);
        const float* src = levels[mip];
        float* dst = levels[mip + 1];
        for (uint32_t y = 0; y < dh; ++y) {
            for (uint32_t x = 0; x < dw; ++x) {
                uint32_t sx0 = 2 * x, sy0 = 2 * y;
                uint32_t sx1 = std::min(sx0 + 1, sw - 1), sy1 = std::min(sy0 + 1, sh - 1);
                float s00 = src[(size_t)sy0 * sw + sx0];
                float s10 = src[(size_t)sy0 * sw + sx1];
                float s01 = src[(size_t)sy1 * sw + sx0];
                float s11 = src[(size_t)sy1 * sw + sx1];
                dst[(size_t)y * dw + x] = fmaxf(fmaxf(s00, s10), fmaxf(s01, s11));
            }
        }
    }
    return mips;
}

// indirect_dispatch.wgsl:79-176 (planes from the CPU extraction above).
void oracle_indirect_dispatch(const HelioGpuCameraUniforms* cam, const float planes[24],
                              const HelioGpuInstanceData* inst, const HelioGpuDrawCall* dc,
                              const HelioGpuInstanceAabb* aabb, uint32_t draw_count,
                              uint32_t instance_count, uint32_t* indirect, uint32_t* stats) {
    for (uint32_t idx = 0; idx < draw_count; ++idx) {
        const HelioGpuDrawCall& d = dc[idx];
        if (d.first_instance >= instance_count) {
            // No representative instance: written as frustum-culled.
            uint32_t* o = indirect + (size_t)idx * 5;
            o[0] = d.index_count;
            o[1] = 0u;
            o[2] = d.first_index;
            std::memcpy(&o[3], &d.vertex_offset, 4);
            o[4] = d.first_instance;
            stats[1] += 1;
            stats[0] += 1;
            continue;
        }
        const HelioGpuInstanceData& in = inst[d.first_instance];
        const HelioGpuInstanceAabb& bb = aabb[d.first_instance];
        // aabb_in_frustum (:88-98)
        bool aabb_visible = true;
        for (int i = 0; i < 6; ++i) {
            const float* pl = planes + i * 4;
            float px = pl[0] >= 0.0f ? bb.max[0] : bb.min[0];
            float py = pl[1] >= 0.0f ? bb.max[1] : bb.min[1];
            float pz = pl[2] >= 0.0f ? bb.max[2] : bb.min[2];
            float dist = dot3(v3(pl[0], pl[1], pl[2]), v3(px, py, pz)) + pl[3];
            if (dist < 0.0f) {
                aabb_visible = false;
                break;
            }
        }
        bool degenerate = bb.min[0] == bb.max[0] && bb.min[1] == bb.max[1] && bb.min[2] == bb.max[2];
        V3 c = v3(in.bounds[0], in.bounds[1], in.bounds[2]);
        float r = in.bounds[3];
        // sphere_in_frustum (:79-86)
        bool sphere_visible = true;
        for (int i = 0; i < 6; ++i) {
            const float* pl = planes + i * 4;
            float dist = dot3(v3(pl[0], pl[1], pl[2]), c) + pl[3];
            if (dist + r < 0.0f) {
                sphere_visible = false;
                break;
            }
        }
        bool visible = degenerate ? sphere_visible : aabb_visible;
        bool should_draw = visible;
        if (visible) {
            float clip[4];
            mat4_point(cam->view_proj, c, clip);
            if (clip[3] > 0.0f) {
                float r_ndc = fabsf((r * cam->proj[1 * 4 + 1]) / clip[3]);
                if (r_ndc < 0.001f) should_draw = false;
            }
        }
        bool shadow = (in.flags & 1u) != 0u;
        if (shadow) stats[5] += 1;
        uint32_t* o = indirect + (size_t)idx * 5;
        o[0] = d.index_count;
        o[2] = d.first_index;
        std::memcpy(&o[3], &d.vertex_offset, 4);
        o[4] = d.first_instance;
        if (should_draw) {
            o[1] = d.instance_count;
            stats[3] += 1;
            if (shadow) stats[6] += 1;
        } else if (!visible) {
            o[1] = 0;
            stats[1] += 1;
        } else {
            o[1] = 0;
            stats[2] += 1;
        }
        stats[0] += 1;
    }
}

// occlusion_cull.wgsl:101-220 (static Hi-Z branch off).
// Static Hi-Z fetch: level 0, clamp to edge, linear filter with weights rounded to 8
// fractional bits, x then y then z, each (1 - w) a + w b (the library's stated rule).
static float static_hiz_sample(const helio_static_hiz* s, float x, float y, float z) {
    const uint32_t n[3] = {s->grid_resolution[0], s->grid_resolution[1], s->grid_resolution[2] * 6u};
    const float c[3] = {x, y, z};
    uint32_t i0[3], i1[3];
    float w[3];
    for (int a = 0; a < 3; ++a) {
        const float t = c[a] * (float)n[a] - 0.5f;
        const float fl = floorf(t);
        w[a] = rintf((t - fl) * 256.0f) / 256.0f;
        const int i = (int)fl, hi = (int)n[a] - 1;
        i0[a] = (uint32_t)std::min(std::max(i, 0), hi);
        i1[a] = (uint32_t)std::min(std::max(i + 1, 0), hi);
    }
    auto at = [&](uint32_t i, uint32_t j, uint32_t k) {
        return s->texels[((size_t)k * n[1] + j) * n[0] + i];
    };
    auto lerp = [](float a, float b, float t) { return (1.0f - t) * a + t * b; };
    const float c00 = lerp(at(i0[0], i0[1], i0[2]), at(i1[0], i0[1], i0[2]), w[0]);
    const float c10 = lerp(at(i0[0], i1[1], i0[2]), at(i1[0], i1[1], i0[2]), w[0]);
    const float c01 = lerp(at(i0[0], i0[1], i1[2]), at(i1[0], i0[1], i1[2]), w[0]);
    const float c11 = lerp(at(i0[0], i1[1], i1[2]), at(i1[0], i1[1], i1[2]), w[0]);
    return lerp(lerp(c00, c10, w[1]), lerp(c01, c11, w[1]), w[2]);
}

// occlusion_cull.wgsl:224-258: true = occluded.
static bool static_hiz_occludes(const helio_static_hiz* s, V3 c, V3 cam_pos) {
    const V3 d = sub(c, cam_pos);
    const float dist = sqrtf(dot3(d, d));
    if (!(dist > 0.001f)) return false;
    const V3 v = divs(d, dist);
    const float ax = fabsf(v.x), ay = fabsf(v.y), az = fabsf(v.z);
    uint32_t layer;
    if (ax >= ay && ax >= az) layer = v.x < 0.0f ? 1u : 0u;
    else if (ay >= az) layer = v.y < 0.0f ? 3u : 2u;
    else layer = v.z < 0.0f ? 5u : 4u;
    const float u = clampf((c.x - s->world_bounds_min[0]) / (s->world_bounds_max[0] - s->world_bounds_min[0]), 0.0f, 1.0f);
    const float vv = clampf((c.y - s->world_bounds_min[1]) / (s->world_bounds_max[1] - s->world_bounds_min[1]), 0.0f, 1.0f);
    const float w0 = clampf((c.z - s->world_bounds_min[2]) / (s->world_bounds_max[2] - s->world_bounds_min[2]), 0.0f, 1.0f);
    const float w = (w0 + (float)layer) / 6.0f;
    return dist > static_hiz_sample(s, u, vv, w) + 0.1f;
}

void oracle_occlusion_cull(const HelioGpuCameraUniforms* cam, uint32_t screen_w,
                           uint32_t screen_h, const helio_hiz_pyramid* hiz,
                           const HelioGpuInstanceData* inst, const HelioGpuDrawCall* dc,
                           uint32_t draw_count, uint32_t instance_count, uint32_t* indirect,
                           uint32_t* stats, oracle_stats* st) {
    oracle_occlusion_cull_static(cam, screen_w, screen_h, hiz, inst, dc, draw_count, instance_count, indirect,
                                 stats, st, nullptr);
}

void oracle_occlusion_cull_static(const HelioGpuCameraUniforms* cam, uint32_t screen_w,
                                  uint32_t screen_h, const helio_hiz_pyramid* hiz,
                                  const HelioGpuInstanceData* inst, const HelioGpuDrawCall* dc,
                                  uint32_t draw_count, uint32_t instance_count, uint32_t* indirect,
                                  uint32_t* stats, oracle_stats* st, const helio_static_hiz* static_hiz) {
    (void)screen_w;
    uint32_t mip_count = oracle_mip_levels(screen_w, screen_h);
    const float P00 = cam->proj[0], P11 = cam->proj[5];
    V3 cam_pos = v3(cam->position_near[0], cam->position_near[1], cam->position_near[2]);
    Marg mg;
    for (uint32_t idx = 0; idx < draw_count; ++idx) {
        if (dc[idx].first_instance >= instance_count) continue;
        const HelioGpuInstanceData& in = inst[dc[idx].first_instance];
        V3 c = v3(in.bounds[0], in.bounds[1], in.bounds[2]);
        float radius = in.bounds[3];
        if (radius <= 0.0f) continue;
        float clip[4];
        mat4_point(cam->view_proj, c, clip);
        if (clip[3] <= 0.0f) continue;
        float ndc_x = clip[0] / clip[3], ndc_y = clip[1] / clip[3];
        float uv_x = ndc_x * 0.5f + 0.5f, uv_y = ndc_y * -0.5f + 0.5f;
        float ndc_r = fmaxf(fabsf((radius * P00) / clip[3]), fabsf((radius * P11) / clip[3]));
        if (ndc_x + ndc_r < -1.0f || ndc_x - ndc_r > 1.0f || ndc_y + ndc_r < -1.0f ||
            ndc_y - ndc_r > 1.0f)
            continue;
        // sphere_near_depth (:124-140)
        float near_z;
        {
            V3 tc = sub(c, cam_pos);
            float dist_sq = dot3(tc, tc);
            if (dist_sq <= radius * radius) {
                near_z = 0.0f;
            } else {
                V3 dir = muls(tc, 1.0f / sqrtf(dist_sq));
                V3 nws = sub(c, muls(dir, radius));
                float nc[4];
                mat4_point(cam->view_proj, nws, nc);
                near_z = nc[3] <= 0.0f ? 0.0f : clampf(nc[2] / nc[3], 0.0f, 1.0f);
            }
        }
        // screen_radius_px (:110-113), pick_mip (:116-120)
        float half_h = (float)screen_h * 0.5f;
        float r_px = fabsf(((radius / clip[3]) * P11) * half_h);
        float diameter = fmaxf(r_px * 2.0f, 1.0f);
        uint32_t mip = std::min(ceil_log2_exact(diameter), mip_count - 1u);
        mip_margin(r_px * 2.0f, mg);
        float uv_half = ndc_r * 0.5f;
        float u0 = clampf(uv_x - uv_half, 0.0f, 1.0f), v0 = clampf(uv_y - uv_half, 0.0f, 1.0f);
        float u1 = clampf(uv_x + uv_half, 0.0f, 1.0f), v1 = clampf(uv_y + uv_half, 0.0f, 1.0f);
        float h00 = sample_nearest(hiz, u0, v0, mip);
        float h01 = sample_nearest(hiz, u1, v0, mip);
        float h10 = sample_nearest(hiz, u0, v1, mip);
        float h11 = sample_nearest(hiz, u1, v1, mip);
        float hz = fmaxf(fmaxf(h00, h01), fmaxf(h10, h11));
        float biased = hz + 1.0f / 65536.0f;
        mg.cmp(near_z, biased);
        bool occluded = near_z > biased;
        if (!occluded && static_hiz) occluded = static_hiz_occludes(static_hiz, c, cam_pos);
        if (occluded) {
            uint32_t* o = indirect + (size_t)idx * 5;
            bool was_visible = o[1] != 0u;
            o[1] = 0u;
            if (was_visible) {
                stats[4] += 1;
                if ((in.flags & 1u) != 0u) stats[7] += 1;
            }
        }
    }
    if (st) st->marginal_decisions += mg.n;
}

// cs_select_objects, vg_cull.wgsl:282-352.
void oracle_vg_select(const HelioGpuCameraUniforms* cam, const oracle_vg_uniforms* u,
                      const HelioGpuVgObject* objects, const HelioGpuInstanceData* inst,
                      const HelioInstanceCullData* cull, uint32_t* selected, uint32_t* counters,
                      oracle_stats* st, int threads) {
    float planes[6][4];
    publish_frustum_planes(cam->view_proj, planes);
    V3 cam_pos = v3(cam->position_near[0], cam->position_near[1], cam->position_near[2]);
    const float near = cam->position_near[3];
    const float focal = (fabsf(cam->proj[5]) * (float)u->screen_height) * 0.5f;
    int nt = std::max(threads, 1);
    struct Local {
        uint64_t hist[8] = {0};
        uint32_t max_lod = 0;
        bool any = false;
        uint64_t tested = 0, visible = 0, marg = 0, marg_obj = 0;
    };
    std::vector<Local> loc(nt);
    parallel_chunks(u->object_count, nt, [&](int t, uint64_t b, uint64_t e) {
        Local& L = loc[t];
        for (uint64_t i = b; i < e; ++i) {
            uint32_t sel = 0;
            const HelioGpuVgObject& o = objects[i];
            uint32_t lod_count = std::min(o.lod_count, 8u);
            Marg mg;
            if (lod_count > 0u && o.instance_index < u->instance_count) {
                const HelioGpuInstanceData& in = inst[o.instance_index];
                const HelioInstanceCullData& cd = cull[o.instance_index];
                if (cd.valid_transform != 0u) {
                    ++L.tested;
                    float cw[4];
                    mat4_point(in.model, v3(o.local_bounds[0], o.local_bounds[1], o.local_bounds[2]), cw);
                    V3 c = v3(cw[0], cw[1], cw[2]);
                    float wr = fmaxf(o.local_bounds[3] * cd.max_scale, 0.0f);
                    if (vg_sphere_visible(planes, c, wr, &mg)) {
                        ++L.visible;
                        V3 d = sub(c, cam_pos);
                        float dist = sqrtf(dot3(d, d));
                        float closest = fmaxf(dist - wr, fmaxf(near, 1.0e-4f));
                        uint32_t lod = 0;
                        for (uint32_t level = 1; level < lod_count; ++level) {
                            float err = ((o.lod_errors[level] * cd.max_scale) * focal) / closest;
                            mg.cmp(err, u->lod_error_threshold_px);
                            if (err <= u->lod_error_threshold_px) lod = level;
                            else break;
                        }
                        sel = lod + 1;
                        L.hist[lod] += 1;
                        L.max_lod = std::max(L.max_lod, lod_count - 1u);
                        L.any = true;
                    }
                }
            }
            L.marg += mg.n;
            if (mg.n) ++L.marg_obj;
            selected[i] = sel;
        }
    });
    for (auto& L : loc) {
        if (u->counter_count >= 11u) {
            for (int k = 0; k < 8; ++k) counters[2 + k] += (uint32_t)L.hist[k];
            if (L.any) counters[10] = std::max(counters[10], L.max_lod);
        }
        if (st) {
            st->objects_tested += L.tested;
            st->objects_visible += L.visible;
            st->marginal_decisions += L.marg;
            st->marginal_objects += L.marg_obj;
        }
    }
}

namespace {

struct CullCtx {
    const HelioGpuCameraUniforms* cam;
    const oracle_vg_uniforms* u;
    float planes[6][4];
    V3 cam_pos;
    const helio_hiz_pyramid* hiz;
};

struct MeshletVerdict {
    bool visible;
    bool cone_loaded;
    uint64_t marg;
};

// cull_meshlet, vg_cull.wgsl:135-241 (decision part; emission done by the caller).
MeshletVerdict cull_one(const CullCtx& C, const HelioGpuMeshletEntry& m,
                        const HelioGpuInstanceData& in, const HelioInstanceCullData& cd) {
    MeshletVerdict v{false, false, 0};
    Marg mg;
    if (cd.valid_transform == 0u) return v;
    const float* model = in.model;
    float cw[4];
    mat4_point(model, v3(m.center[0], m.center[1], m.center[2]), cw);
    V3 c = v3(cw[0], cw[1], cw[2]);
    float wr = fmaxf(m.radius * cd.max_scale, 0.0f);
    V3 ctc = sub(c, C.cam_pos);
    if (!vg_sphere_visible(C.planes, c, wr, &mg)) {
        v.marg = mg.n;
        return v;
    }
    v.cone_loaded = true;
    // Cone (:159-182)
    float cam_dist_sq = dot3(ctc, ctc);
    float guard = wr * 1.5f;
    if (m.cone_cutoff <= 1.0f && cd.cone_cull_enabled != 0u) mg.cmp(cam_dist_sq, guard * guard);
    if (cam_dist_sq > guard * guard && m.cone_cutoff <= 1.0f && cd.cone_cull_enabled != 0u) {
        const float* n = in.normal_mat;
        V3 ax = v3((n[0] * m.cone_axis[0] + n[4] * m.cone_axis[1]) + n[8] * m.cone_axis[2],
                   (n[1] * m.cone_axis[0] + n[5] * m.cone_axis[1]) + n[9] * m.cone_axis[2],
                   (n[2] * m.cone_axis[0] + n[6] * m.cone_axis[1]) + n[10] * m.cone_axis[2]);
        V3 axis_ws = divs(ax, sqrtf(dot3(ax, ax)));
        float aw[4];
        mat4_point(model, v3(m.cone_apex[0], m.cone_apex[1], m.cone_apex[2]), aw);
        V3 cta = sub(v3(aw[0], aw[1], aw[2]), C.cam_pos);
        float ads = dot3(cta, cta);
        if (ads > 1.0e-12f) {
            float dd = dot3(divs(cta, sqrtf(ads)), axis_ws);
            mg.cmp(dd, m.cone_cutoff);
            if (dd >= m.cone_cutoff) {
                v.marg = mg.n;
                return v;
            }
        }
    }
    // Hi-Z (:184-240)
    const HelioGpuCameraUniforms* cam = C.cam;
    float clip[4];
    mat4_point(cam->view_proj, c, clip);
    if (clip[3] > 0.0f) {
        float ndc_x = clip[0] / clip[3], ndc_y = clip[1] / clip[3];
        float uv_x = ndc_x * 0.5f + 0.5f, uv_y = ndc_y * -0.5f + 0.5f;
        float nvd = clip[3] - wr;
        mg.cmp(nvd, cam->position_near[3]);
        if (nvd > cam->position_near[3]) {
            float ndc_r = fmaxf(fabsf((wr * cam->proj[0]) / nvd), fabsf((wr * cam->proj[5]) / nvd));
            float uvr = ndc_r * 0.5f;
            float u0 = uv_x - uvr, v0 = uv_y - uvr, u1 = uv_x + uvr, v1 = uv_y + uvr;
            mg.cmp(u0, 0.0f);
            mg.cmp(v0, 0.0f);
            mg.cmp(u1, 1.0f);
            mg.cmp(v1, 1.0f);
            if (u0 >= 0.0f && v0 >= 0.0f && u1 <= 1.0f && v1 <= 1.0f) {
                float dist_sq = dot3(ctc, ctc);
                float near_z = 0.0f;
                if (dist_sq > wr * wr) {
                    V3 dir = divs(ctc, sqrtf(dist_sq));
                    V3 nws = sub(c, muls(dir, wr));
                    float nc[4];
                    mat4_point(cam->view_proj, nws, nc);
                    if (nc[3] > 0.0f) near_z = clampf(nc[2] / nc[3], 0.0f, 1.0f);
                }
                float half_h = (float)C.u->screen_height * 0.5f;
                float dpx = fmaxf((ndc_r * half_h) * 2.0f, 1.0f);
                mip_margin((ndc_r * half_h) * 2.0f, mg);
                uint32_t mip = std::min(ceil_log2_exact(dpx), C.u->hiz_mip_count - 1u);
                float h00 = sample_nearest(C.hiz, u0, v0, mip);
                float h01 = sample_nearest(C.hiz, u1, v0, mip);
                float h10 = sample_nearest(C.hiz, u0, v1, mip);
                float h11 = sample_nearest(C.hiz, u1, v1, mip);
                float hz = fmaxf(fmaxf(h00, h01), fmaxf(h10, h11));
                float biased = hz + 1.0f / 65536.0f;
                mg.cmp(near_z, biased);
                if (near_z > biased) {
                    v.marg = mg.n;
                    return v;
                }
            }
        }
    }
    v.visible = true;
    v.marg = mg.n;
    return v;
}

}  // namespace

// cs_cull_meshlets, vg_cull.wgsl:354-405, with emission (:242-263) in canonical
// (work item, lane) order: slot = number of visible meshlets before this one.
void oracle_vg_cull(const HelioGpuCameraUniforms* cam, const oracle_vg_uniforms* u,
                    const HelioGpuMeshletEntry* meshlets, const HelioGpuVgObject* objects,
                    const uint32_t* selected, const HelioGpuInstanceData* inst,
                    const HelioInstanceCullData* cull, const HelioGpuVgWorkItem* items,
                    const helio_hiz_pyramid* hiz, HelioDrawIndexedIndirectArgs* indirect,
                    HelioGpuVgDraw* draws, uint32_t* counters, uint32_t* visibility,
                    oracle_stats* st, int threads) {
    CullCtx C;
    C.cam = cam;
    C.u = u;
    C.hiz = hiz;
    publish_frustum_planes(cam->view_proj, C.planes);
    C.cam_pos = v3(cam->position_near[0], cam->position_near[1], cam->position_near[2]);
    int nt = std::max(threads, 1);
    uint64_t W = u->work_item_count;
    struct Local {
        std::vector<uint32_t> vis;  // (meshlet_index, instance, lod, lane-in-item) packed as 3 words
        uint64_t tested = 0, cone = 0, marg = 0, marg_m = 0;
    };
    std::vector<Local> loc(nt);
    std::vector<uint64_t> chunk_begin(nt + 1, W);
    parallel_chunks(W, nt, [&](int t, uint64_t b, uint64_t e) {
        Local& L = loc[t];
        chunk_begin[t] = b;
        for (uint64_t w = b; w < e; ++w) {
            uint32_t mask[2] = {0u, 0u};
            const HelioGpuVgWorkItem& it = items[w];
            if (it.object_index < u->object_count) {
                const HelioGpuVgObject& o = objects[it.object_index];
                uint32_t sp1 = selected[it.object_index];
                if (sp1 != 0u) {
                    uint32_t lod = sp1 - 1u;
                    uint32_t count = o.lod_meshlet_counts[lod];
                    if (it.local_meshlet_base < count) {
                        uint32_t first = o.lod_first_meshlets[lod];
                        for (uint32_t lane = 0; lane < 64; ++lane) {
                            uint32_t local = it.local_meshlet_base + lane;
                            if (local >= count) break;
                            uint32_t mi = first + local;
                            uint32_t ii = o.instance_index;
                            if (mi >= u->meshlet_count || ii >= u->instance_count) continue;
                            ++L.tested;
                            MeshletVerdict v = cull_one(C, meshlets[mi], inst[ii], cull[ii]);
                            if (v.cone_loaded) ++L.cone;
                            L.marg += v.marg;
                            if (v.marg) ++L.marg_m;
                            if (v.visible) {
                                mask[lane >> 5] |= 1u << (lane & 31);
                                L.vis.push_back(mi);
                                L.vis.push_back(ii);
                                L.vis.push_back(lod);
                            }
                        }
                    }
                }
            }
            if (visibility) {
                visibility[2 * w] = mask[0];
                visibility[2 * w + 1] = mask[1];
            }
        }
    });
    // Deterministic merge in chunk (= work item) order.
    uint32_t capacity = u->draw_capacity;
    uint64_t slot = 0;
    for (int t = 0; t < nt; ++t) {
        Local& L = loc[t];
        for (size_t k = 0; k < L.vis.size(); k += 3, ++slot) {
            if (slot < capacity) {
                const HelioGpuMeshletEntry& m = meshlets[L.vis[k]];
                HelioDrawIndexedIndirectArgs& a = indirect[slot];
                a.index_count = m.index_count;
                a.instance_count = 1u;
                a.first_index = m.first_index;
                a.base_vertex = m.vertex_offset;
                a.first_instance = (uint32_t)slot;
                HelioGpuVgDraw& d = draws[slot];
                d.instance_index = L.vis[k + 1];
                d.meshlet_index = L.vis[k];
                d.lod_level = L.vis[k + 2];
                d.reserved = 0u;
            } else {
                counters[1] += 1u;
            }
        }
        if (st) {
            st->meshlets_tested += L.tested;
            st->meshlets_cone_loaded += L.cone;
            st->marginal_decisions += L.marg;
            st->marginal_meshlets += L.marg_m;
        }
    }
    counters[0] += (uint32_t)slot;
    if (st) st->meshlets_visible += slot;
}


// rebuild_vg_buffers, crates/helio/src/scene/virtual_geometry/rebuild.rs:98-172, with
// append_unique_meshlets (:18-43) and append_work_items (:45-58). A slot whose mesh
// index is not below mesh_count stands for a free dense slot or a missing mesh record
// (both skipped by the reference, :110-129).
int oracle_vg_rebuild(const HelioGpuMeshletEntry* pool, uint32_t pool_count, const HelioVgMeshRecord* meshes,
                      uint32_t mesh_count, const uint32_t* slot_mesh, const HelioGpuInstanceData* slot_instances,
                      uint32_t slot_count, HelioGpuMeshletEntry* out_meshlets, HelioGpuVgObject* out_objects,
                      HelioGpuInstanceData* out_instances, HelioGpuVgWorkItem* out_items, uint64_t counts[4]) {
    const uint64_t kU32 = 0xFFFFFFFFull;
    std::vector<int64_t> base(mesh_count, -1);
    uint64_t descriptors = 0;
    // append_unique_meshlets over the referenced meshes in dense order (:25-40).
    for (uint32_t o = 0; o < slot_count; ++o) {
        const uint32_t m = slot_mesh[o];
        if (m >= mesh_count || base[m] >= 0) continue;
        const HelioVgMeshRecord& r = meshes[m];
        if (r.meshlet_count == 0 || r.lod_count == 0) continue;
        if ((uint64_t)r.first_meshlet + r.meshlet_count > pool_count) return 1;
        if (descriptors > kU32) return 1;  // u32::try_from(output.len()) (:36-37)
        base[m] = (int64_t)descriptors;
        if (out_meshlets)
            std::memcpy(out_meshlets + descriptors, pool + r.first_meshlet, sizeof(HelioGpuMeshletEntry) * r.meshlet_count);
        descriptors += r.meshlet_count;
    }
    if (descriptors > kU32) return 1;  // meshlet_count = u32::try_from(len) (vg_frame_data, :72-73)
    uint64_t objects = 0, items = 0, draws = 0;
    for (uint32_t o = 0; o < slot_count; ++o) {
        const uint32_t m = slot_mesh[o];
        if (m >= mesh_count || base[m] < 0) continue;  // :124-129
        const HelioVgMeshRecord& r = meshes[m];
        HelioGpuVgObject ob;
        ob.instance_index = (uint32_t)objects;  // instance and object indices advance together (:131-134)
        ob.lod_count = r.lod_count;
        ob.max_meshlet_count = r.max_meshlet_count;
        ob.reserved = 0;
        for (int k = 0; k < 4; ++k) ob.local_bounds[k] = r.local_bounds[k];
        for (int l = 0; l < HELIO_VG_LOD_LEVELS; ++l) {
            const uint64_t first = (uint64_t)base[m] + r.lod_first_meshlets[l];  // checked_add (:137-139)
            if (first > kU32) return 1;
            ob.lod_errors[l] = r.lod_errors[l];
            ob.lod_first_meshlets[l] = (uint32_t)first;
            ob.lod_meshlet_counts[l] = r.lod_meshlet_counts[l];
        }
        if (out_objects) out_objects[objects] = ob;
        if (out_instances) out_instances[objects] = slot_instances[o];
        // append_work_items: (object, 0), (object, 64), ... below max_meshlet_count (:45-58).
        for (uint64_t b = 0; b < r.max_meshlet_count; b += HELIO_VG_MESHLETS_PER_WORK_ITEM) {
            if (out_items) out_items[items] = HelioGpuVgWorkItem{(uint32_t)objects, (uint32_t)b};
            ++items;
        }
        draws += r.max_meshlet_count;  // checked_add (:158-161)
        if (draws > kU32) return 1;
        ++objects;
    }
    if (items > kU32) return 1;  // work_item_count = u32::try_from(len) (:76-77)
    counts[0] = descriptors;
    counts[1] = objects;
    counts[2] = items;
    counts[3] = draws;
    return 0;
}


// normalize_plane (shadow_cull.wgsl:49-55): p / length(p.xyz) when that length exceeds 1e-10.
static void shadow_normalize(float p[4]) {
    const float len = sqrtf((p[0] * p[0] + p[1] * p[1]) + p[2] * p[2]);
    if (len > 1e-10f) {
        p[0] = p[0] / len;
        p[1] = p[1] / len;
        p[2] = p[2] / len;
        p[3] = p[3] / len;
    }
}

// sphere_in_frustum (shadow_cull.wgsl:57-71): planes from the columns of vp (vp[i] is
// column i): c3 + c0, c3 - c0, c3 + c1, c3 - c1, c2, c3 - c2.
static void shadow_planes(const float* vp, float pl[6][4]) {
    const float* c0 = vp;
    const float* c1 = vp + 4;
    const float* c2 = vp + 8;
    const float* c3 = vp + 12;
    for (int k = 0; k < 4; ++k) {
        pl[0][k] = c3[k] + c0[k];
        pl[1][k] = c3[k] - c0[k];
        pl[2][k] = c3[k] + c1[k];
        pl[3][k] = c3[k] - c1[k];
        pl[4][k] = c2[k];
        pl[5][k] = c3[k] - c2[k];
    }
    for (int i = 0; i < 6; ++i) shadow_normalize(pl[i]);
}

int oracle_shadow_cull(const float* matrices, const HelioGpuInstanceData* instances, uint32_t instance_count,
                       const HelioDrawIndexedIndirectArgs* src, uint32_t draw_count, const uint32_t* face_dirty,
                       uint32_t face_count, uint32_t max_per_face, HelioDrawIndexedIndirectArgs* dst,
                       uint32_t* face_counts) {
    constexpr uint32_t kFaces = 256;
    if (face_count == 0 || draw_count == 0) return 0;  // lib.rs:261-263
    for (uint32_t f = 0; f < kFaces; ++f) face_counts[f] = 0;  // lib.rs:266-270
    std::vector<std::array<std::array<float, 4>, 6>> planes(kFaces);
    for (uint32_t f = 0; f < kFaces; ++f) {
        if (face_dirty[f] == 0) continue;
        float pl[6][4];
        shadow_planes(matrices + 16 * f, pl);
        for (int i = 0; i < 6; ++i)
            for (int k = 0; k < 4; ++k) planes[f][i][k] = pl[i][k];
    }
    for (uint32_t d = 0; d < draw_count; ++d) {
        const HelioDrawIndexedIndirectArgs draw = src[d];
        if (draw.first_instance >= instance_count) continue;
        const float* b = instances[draw.first_instance].bounds;
        const V3 c = v3(b[0], b[1], b[2]);
        const float radius = b[3];
        if (radius <= 0.0f) continue;  // shadow_cull.wgsl:82 (a NaN radius goes on)
        for (uint32_t f = 0; f < kFaces; ++f) {
            if (face_dirty[f] == 0) continue;
            bool inside = true;
            for (int i = 0; i < 6 && inside; ++i) {
                const auto& p = planes[f][i];
                if ((dot3(v3(p[0], p[1], p[2]), c) + p[3]) + radius < 0.0f) inside = false;
            }
            if (!inside) continue;
            const uint32_t slot = face_counts[f]++;
            if (slot < max_per_face) dst[(size_t)f * max_per_face + slot] = draw;
        }
    }
    return 1;
}

}  // extern "C"
