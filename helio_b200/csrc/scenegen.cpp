// scenegen.cpp — seeded synthetic inputs for the visibility path: virtual-geometry
// scenes in libhelio byte layouts, cameras (GpuCameraUniforms) and occluder depth.
//
// Deterministic: xoshiro256** streams seeded through splitmix64; each instance,
// mesh and depth band has its own stream, so the output bytes do not depend on
// the thread count. Values are drawn in double and rounded to binary32 once.
//
// Shapes follow the reference's scene build (crates/helio/src/scene/virtual_geometry/
// rebuild.rs:98-172): per-LOD descriptor ranges, 64-meshlet work spans
// (:45-58) and max_draw_count = sum of max_meshlet_count (:158-161). Instance
// bounds / AABBs follow crates/helio/src/scene/helpers.rs:54-66 (sphere_to_aabb).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/helio_cull.h"

namespace {

inline uint64_t splitmix64(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (auto& v : s) v = splitmix64(x);
    }
    static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        uint64_t r = rotl(s[1] * 5, 7) * 9;
        uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uni() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    double uni(double a, double b) { return a + (b - a) * uni(); }
    double normal() {
        double u1 = uni(), u2 = uni();
        if (u1 < 1e-300) u1 = 1e-300;
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

inline uint64_t stream_seed(uint64_t seed, uint64_t tag, uint64_t index) {
    uint64_t x = seed ^ (tag * 0xD1B54A32D192ED03ull);
    splitmix64(x);
    x ^= index * 0x9E3779B97F4A7C15ull;
    return splitmix64(x);
}

template <typename F>
void parallel_for(uint64_t n, uint32_t threads, F&& fn) {
    uint32_t nt = std::max(1u, threads);
    if (nt == 1 || n < 256) {
        for (uint64_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::vector<std::thread> pool;
    uint64_t chunk = (n + nt - 1) / nt;
    for (uint32_t t = 0; t < nt; ++t) {
        uint64_t b = std::min<uint64_t>(n, (uint64_t)t * chunk), e = std::min<uint64_t>(n, b + chunk);
        pool.emplace_back([&fn, b, e] {
            for (uint64_t i = b; i < e; ++i) fn(i);
        });
    }
    for (auto& th : pool) th.join();
}

struct D3 {
    double x, y, z;
};
inline D3 dsub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline double ddot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline D3 dcross(D3 a, D3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline D3 dnorm(D3 a) {
    double l = std::sqrt(ddot(a, a));
    return {a.x / l, a.y / l, a.z / l};
}

D3 unit_sphere(Rng& r) {
    double z = r.uni(-1.0, 1.0), phi = r.uni(0.0, 6.283185307179586);
    double s = std::sqrt(std::max(0.0, 1.0 - z * z));
    return {s * std::cos(phi), s * std::sin(phi), z};
}

// Column-major 4x4 in double.
struct M4 {
    double m[16];
};
M4 mmul(const M4& a, const M4& b) {
    M4 r;
    for (int c = 0; c < 4; ++c)
        for (int rr = 0; rr < 4; ++rr) {
            double s = 0;
            for (int k = 0; k < 4; ++k) s += a.m[k * 4 + rr] * b.m[c * 4 + k];
            r.m[c * 4 + rr] = s;
        }
    return r;
}
bool minv(const M4& a, M4& out) {
    // Gauss-Jordan on a row-major copy.
    double t[4][8];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) {
            t[r][c] = a.m[c * 4 + r];
            t[r][c + 4] = (r == c) ? 1.0 : 0.0;
        }
    for (int c = 0; c < 4; ++c) {
        int p = c;
        for (int r = c + 1; r < 4; ++r)
            if (std::fabs(t[r][c]) > std::fabs(t[p][c])) p = r;
        if (std::fabs(t[p][c]) < 1e-300) return false;
        if (p != c)
            for (int k = 0; k < 8; ++k) std::swap(t[p][k], t[c][k]);
        double inv = 1.0 / t[c][c];
        for (int k = 0; k < 8; ++k) t[c][k] *= inv;
        for (int r = 0; r < 4; ++r)
            if (r != c) {
                double f = t[r][c];
                for (int k = 0; k < 8; ++k) t[r][k] -= f * t[c][k];
            }
    }
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) out.m[c * 4 + r] = t[r][c + 4];
    return true;
}

M4 look_at_rh(D3 eye, D3 target, D3 up) {
    D3 f = dnorm(dsub(target, eye));
    D3 s = dnorm(dcross(f, up));
    D3 u = dcross(s, f);
    M4 v = {{s.x, u.x, -f.x, 0, s.y, u.y, -f.y, 0, s.z, u.z, -f.z, 0, -ddot(s, eye), -ddot(u, eye),
             ddot(f, eye), 1}};
    return v;
}

void fill_camera(const M4& view, const M4& proj, D3 eye, double near, double far,
                 HelioGpuCameraUniforms* out) {
    M4 vp = mmul(proj, view);
    M4 inv;
    if (!minv(vp, inv)) std::memset(&inv, 0, sizeof(inv));
    D3 fwd = dnorm({-view.m[2], -view.m[6], -view.m[10]});
    for (int i = 0; i < 16; ++i) {
        out->view[i] = (float)view.m[i];
        out->proj[i] = (float)proj.m[i];
        out->view_proj[i] = (float)vp.m[i];
        out->inv_view_proj[i] = (float)inv.m[i];
        out->prev_view_proj[i] = (float)vp.m[i];
    }
    out->position_near[0] = (float)eye.x;
    out->position_near[1] = (float)eye.y;
    out->position_near[2] = (float)eye.z;
    out->position_near[3] = (float)near;
    out->forward_far[0] = (float)fwd.x;
    out->forward_far[1] = (float)fwd.y;
    out->forward_far[2] = (float)fwd.z;
    out->forward_far[3] = (float)far;
    out->jitter_frame[0] = out->jitter_frame[1] = out->jitter_frame[2] = out->jitter_frame[3] = 0.0f;
}

}  // namespace

extern "C" {

typedef struct sg_scene_params {
    uint64_t seed;
    uint32_t instance_count;
    uint32_t lod0_meshlets;  // meshlets of LOD 0; LOD k has ceil(lod0 / 2^k)
    uint32_t lod_count;      // 1..8
    uint32_t placement;      // 0 = uniform in a cube, 1 = Gaussian blobs in a cube
    float cube_half;         // half side of the placement cube (m)
    uint32_t blob_count;
    float blob_sigma;
    uint32_t lod_error_mode;   // 0 = coverage thresholds 0.25/0.06/0.015, 1 = log-uniform [1e-4, 1e-1]
    float coverage_height_px;  // viewport height used by lod_error_mode 0
    float coverage_tau_px;     // pixel threshold used by lod_error_mode 0 (2.0)
    uint32_t mesh_library;     // 0 = one unique mesh per instance, else shared library size
    uint32_t threads;
    float scale_min, scale_max;
} sg_scene_params;

typedef struct sg_scene_counts {
    uint64_t meshlets;
    uint64_t objects;
    uint64_t work_items;
    uint64_t max_draw_count;
    uint64_t mesh_count;
    uint64_t meshlets_per_mesh;
} sg_scene_counts;

static uint32_t lod_size(uint32_t lod0, uint32_t k) { return (lod0 + (1u << k) - 1u) >> k; }

int32_t sg_scene_counts_fn(const sg_scene_params* p, sg_scene_counts* c) {
    if (!p || !c || p->lod_count == 0 || p->lod_count > 8) return HELIO_ERR_INVALID_ARG;
    uint64_t per_mesh = 0;
    for (uint32_t k = 0; k < p->lod_count; ++k) per_mesh += lod_size(p->lod0_meshlets, k);
    uint64_t meshes = p->mesh_library ? p->mesh_library : p->instance_count;
    c->mesh_count = meshes;
    c->meshlets_per_mesh = per_mesh;
    c->meshlets = per_mesh * meshes;
    c->objects = p->instance_count;
    uint64_t spans = (p->lod0_meshlets + 63u) / 64u;
    c->work_items = spans * p->instance_count;
    c->max_draw_count = (uint64_t)p->lod0_meshlets * p->instance_count;
    return HELIO_OK;
}

// Generates the complete scene. Array lengths follow sg_scene_counts_fn; aabbs and
// draw_calls (one per instance, instance-level passes) may be NULL.
int32_t sg_scene_generate(const sg_scene_params* p, HelioGpuMeshletEntry* meshlets,
                          HelioGpuVgObject* objects, HelioGpuInstanceData* instances,
                          HelioGpuVgWorkItem* work_items, HelioGpuInstanceAabb* aabbs,
                          HelioGpuDrawCall* draw_calls) {
    sg_scene_counts c;
    int32_t st = sg_scene_counts_fn(p, &c);
    if (st != HELIO_OK) return st;
    const uint32_t L = p->lod_count;
    uint32_t lod_first[8] = {0}, lod_cnt[8] = {0};
    {
        uint32_t off = 0;
        for (uint32_t k = 0; k < L; ++k) {
            lod_first[k] = off;
            lod_cnt[k] = lod_size(p->lod0_meshlets, k);
            off += lod_cnt[k];
        }
    }
    const uint64_t per_mesh = c.meshlets_per_mesh;
    // Per-mesh data: meshlets, LOD errors, local radius, LOD0 index count.
    std::vector<float> mesh_err((size_t)c.mesh_count * 8, 0.0f);
    std::vector<float> mesh_radius((size_t)c.mesh_count, 1.0f);
    std::vector<uint32_t> mesh_lod0_indices((size_t)c.mesh_count, 0u);
    static const double cov[4] = {0.0, 0.25, 0.06, 0.015};
    parallel_for(c.mesh_count, p->threads, [&](uint64_t mi) {
        Rng r(stream_seed(p->seed, 1, mi));
        double maxr = 0.0;
        HelioGpuMeshletEntry* base = meshlets + mi * per_mesh;
        // LOD errors (levels 1..L-1).
        double err[8] = {0};
        if (p->lod_error_mode == 1) {
            std::vector<double> e;
            for (uint32_t k = 1; k < L; ++k) e.push_back(std::exp(r.uni(std::log(1e-4), std::log(1e-1))));
            std::sort(e.begin(), e.end());
            for (uint32_t k = 1; k < L; ++k) err[k] = e[k - 1];
        }
        uint32_t lod0_idx = 0;
        for (uint64_t j = 0; j < per_mesh; ++j) {
            HelioGpuMeshletEntry& m = base[j];
            uint32_t level = 0;
            while (level + 1 < L && j >= lod_first[level + 1]) ++level;
            D3 dir = unit_sphere(r);
            double rad = std::cbrt(r.uni());
            double mr = r.uni(0.05, 0.3);
            maxr = std::max(maxr, mr);
            D3 ax = unit_sphere(r);
            double cutoff = r.uni(-1.0, 1.0);
            uint32_t tris = 1u + (uint32_t)(r.uni() * 124.0);
            if (tris > 124u) tris = 124u;
            m.center[0] = (float)(dir.x * rad);
            m.center[1] = (float)(dir.y * rad);
            m.center[2] = (float)(dir.z * rad);
            m.radius = (float)mr;
            m.cone_apex[0] = m.center[0];
            m.cone_apex[1] = m.center[1];
            m.cone_apex[2] = m.center[2];
            m.cone_cutoff = (float)cutoff;
            m.cone_axis[0] = (float)ax.x;
            m.cone_axis[1] = (float)ax.y;
            m.cone_axis[2] = (float)ax.z;
            m.lod_error = 0.0f;
            m.first_index = (uint32_t)(((mi * per_mesh + j) * 372ull) & 0xFFFFFFFFull);
            m.index_count = tris * 3u;
            m.vertex_offset = (int32_t)((mi * 4096ull) & 0x7FFFFFFFull);
            m.instance_index = 0u;
            if (level == 0) lod0_idx += m.index_count;
        }
        double R = 1.0 + maxr;
        if (p->lod_error_mode == 0) {
            for (uint32_t k = 1; k < L && k < 4; ++k)
                err[k] = p->coverage_tau_px * R / (cov[k] * p->coverage_height_px * 0.5);
            for (uint32_t k = 4; k < L; ++k) err[k] = err[k - 1] * 4.0;
        }
        for (uint64_t j = 0; j < per_mesh; ++j) {
            uint32_t level = 0;
            while (level + 1 < L && j >= lod_first[level + 1]) ++level;
            base[j].lod_error = (float)err[level];
        }
        for (uint32_t k = 0; k < 8; ++k) mesh_err[mi * 8 + k] = (float)err[k];
        mesh_radius[mi] = (float)R;
        mesh_lod0_indices[mi] = lod0_idx;
    });
    // Blob centres.
    std::vector<D3> blobs;
    if (p->placement == 1) {
        Rng r(stream_seed(p->seed, 2, 0));
        for (uint32_t b = 0; b < std::max(1u, p->blob_count); ++b)
            blobs.push_back({r.uni(-p->cube_half, p->cube_half), r.uni(-p->cube_half, p->cube_half),
                             r.uni(-p->cube_half, p->cube_half)});
    }
    const uint64_t spans = (p->lod0_meshlets + 63u) / 64u;
    parallel_for(p->instance_count, p->threads, [&](uint64_t i) {
        Rng r(stream_seed(p->seed, 3, i));
        uint64_t mesh = p->mesh_library ? (uint64_t)(r.next() % p->mesh_library) : i;
        D3 pos;
        if (p->placement == 1) {
            const D3& b = blobs[(size_t)(r.next() % blobs.size())];
            pos = {b.x + r.normal() * p->blob_sigma, b.y + r.normal() * p->blob_sigma,
                   b.z + r.normal() * p->blob_sigma};
        } else {
            pos = {r.uni(-p->cube_half, p->cube_half), r.uni(-p->cube_half, p->cube_half),
                   r.uni(-p->cube_half, p->cube_half)};
        }
        double s = r.uni(p->scale_min, p->scale_max);
        // Uniform random rotation (Shoemake).
        double u1 = r.uni(), u2 = r.uni(), u3 = r.uni();
        double qx = std::sqrt(1 - u1) * std::sin(6.283185307179586 * u2);
        double qy = std::sqrt(1 - u1) * std::cos(6.283185307179586 * u2);
        double qz = std::sqrt(u1) * std::sin(6.283185307179586 * u3);
        double qw = std::sqrt(u1) * std::cos(6.283185307179586 * u3);
        double R[9] = {1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy + qz * qw), 2 * (qx * qz - qy * qw),
                       2 * (qx * qy - qz * qw), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz + qx * qw),
                       2 * (qx * qz + qy * qw), 2 * (qy * qz - qx * qw), 1 - 2 * (qx * qx + qy * qy)};
        HelioGpuInstanceData& in = instances[i];
        std::memset(&in, 0, sizeof(in));
        for (int col = 0; col < 3; ++col)
            for (int row = 0; row < 3; ++row) in.model[col * 4 + row] = (float)(R[col * 3 + row] * s);
        in.model[12] = (float)pos.x;
        in.model[13] = (float)pos.y;
        in.model[14] = (float)pos.z;
        in.model[15] = 1.0f;
        for (int col = 0; col < 3; ++col)
            for (int row = 0; row < 3; ++row) in.normal_mat[col * 4 + row] = (float)(R[col * 3 + row] / s);
        float rad = mesh_radius[mesh] * (float)s;
        in.bounds[0] = (float)pos.x;
        in.bounds[1] = (float)pos.y;
        in.bounds[2] = (float)pos.z;
        in.bounds[3] = rad;
        in.mesh_id = (uint32_t)mesh;
        in.material_id = 0u;
        in.flags = (r.next() & 1ull) ? 1u : 0u;
        in.lightmap_index = 0xFFFFFFFFu;
        HelioGpuVgObject& o = objects[i];
        std::memset(&o, 0, sizeof(o));
        o.instance_index = (uint32_t)i;
        o.lod_count = L;
        o.max_meshlet_count = p->lod0_meshlets;
        o.reserved = 0u;
        o.local_bounds[3] = mesh_radius[mesh];
        for (uint32_t k = 0; k < 8; ++k) {
            o.lod_errors[k] = mesh_err[mesh * 8 + k];
            o.lod_first_meshlets[k] = (uint32_t)(mesh * per_mesh) + (k < L ? lod_first[k] : 0u);
            o.lod_meshlet_counts[k] = k < L ? lod_cnt[k] : 0u;
        }
        for (uint64_t sIdx = 0; sIdx < spans; ++sIdx) {
            work_items[i * spans + sIdx].object_index = (uint32_t)i;
            work_items[i * spans + sIdx].local_meshlet_base = (uint32_t)(sIdx * 64u);
        }
        if (aabbs) {
            HelioGpuInstanceAabb& a = aabbs[i];
            a.min[0] = in.bounds[0] - rad;
            a.min[1] = in.bounds[1] - rad;
            a.min[2] = in.bounds[2] - rad;
            a.max[0] = in.bounds[0] + rad;
            a.max[1] = in.bounds[1] + rad;
            a.max[2] = in.bounds[2] + rad;
            a.pad0 = a.pad1 = 0.0f;
        }
        if (draw_calls) {
            HelioGpuDrawCall& d = draw_calls[i];
            d.index_count = mesh_lod0_indices[mesh];
            d.first_index = meshlets[mesh * per_mesh].first_index;
            d.vertex_offset = meshlets[mesh * per_mesh].vertex_offset;
            d.first_instance = (uint32_t)i;
            d.instance_count = 1u;
        }
    });
    return HELIO_OK;
}

// glam Mat4::perspective_rh + look_at_rh, GpuCameraUniforms::new (camera.rs:34-57).
void sg_camera_perspective(const double eye[3], const double target[3], const double up[3],
                           double fov_y, double aspect, double near, double far,
                           HelioGpuCameraUniforms* out) {
    double h = std::cos(0.5 * fov_y) / std::sin(0.5 * fov_y);
    double w = h / aspect;
    double r = far / (near - far);
    M4 proj = {{w, 0, 0, 0, 0, h, 0, 0, 0, 0, r, -1, 0, 0, r * near, 0}};
    M4 view = look_at_rh({eye[0], eye[1], eye[2]}, {target[0], target[1], target[2]},
                         {up[0], up[1], up[2]});
    fill_camera(view, proj, {eye[0], eye[1], eye[2]}, near, far, out);
}

// glam Mat4::orthographic_rh + look_at_rh.
void sg_camera_ortho(const double eye[3], const double target[3], const double up[3], double left,
                     double right, double bottom, double top, double near, double far,
                     HelioGpuCameraUniforms* out) {
    double rw = 1.0 / (right - left), rh = 1.0 / (top - bottom), r = 1.0 / (near - far);
    M4 proj = {{rw + rw, 0, 0, 0, 0, rh + rh, 0, 0, 0, 0, r, 0, -(left + right) * rw,
                -(top + bottom) * rh, r * near, 1}};
    M4 view = look_at_rh({eye[0], eye[1], eye[2]}, {target[0], target[1], target[2]},
                         {up[0], up[1], up[2]});
    fill_camera(view, proj, {eye[0], eye[1], eye[2]}, near, far, out);
}

// Occluder depth: background 1.0 (standard Z, far plane; crates/helio-pass-depth-prepass/
// src/lib.rs:105,149), n_rects axis-aligned rectangles composited with Less (min).
// Rectangle sides ~ U[W/64, W/4] * side_scale; top-left corner uniform over the
// image; linear view depth t ~ U[0,1] mapped to d = near + t (far - near) and
// stored as the camera's NDC depth (perspective: far/(far-near) * (1 - near/d);
// orthographic: t).
int32_t sg_depth(uint64_t seed, uint32_t w, uint32_t h, uint32_t pitch, uint32_t n_rects,
                 float side_scale, float near, float far, uint32_t orthographic, float* out,
                 uint32_t threads) {
    if (!out || w == 0 || h == 0 || pitch < w) return HELIO_ERR_INVALID_ARG;
    struct Rect {
        uint32_t x0, y0, x1, y1;
        float z;
    };
    std::vector<Rect> rects(n_rects);
    Rng r(stream_seed(seed, 4, 0));
    double smin = (double)w / 64.0 * side_scale, smax = (double)w / 4.0 * side_scale;
    for (uint32_t k = 0; k < n_rects; ++k) {
        double sx = r.uni(smin, smax), sy = r.uni(smin, smax);
        double x0 = r.uni(0.0, (double)w), y0 = r.uni(0.0, (double)h);
        double t = r.uni();
        double d = (double)near + t * ((double)far - (double)near);
        double z = orthographic ? t : ((double)far / ((double)far - (double)near)) * (1.0 - (double)near / d);
        Rect& q = rects[k];
        q.x0 = (uint32_t)x0;
        q.y0 = (uint32_t)y0;
        q.x1 = (uint32_t)std::min<double>((double)w, std::ceil(x0 + sx));
        q.y1 = (uint32_t)std::min<double>((double)h, std::ceil(y0 + sy));
        q.z = (float)std::min(1.0, std::max(0.0, z));
    }
    uint32_t nt = std::max(1u, threads);
    uint32_t bands = std::min<uint32_t>(h, nt * 8);
    parallel_for(bands, nt, [&](uint64_t b) {
        uint32_t y_begin = (uint32_t)((uint64_t)h * b / bands), y_end = (uint32_t)((uint64_t)h * (b + 1) / bands);
        for (uint32_t y = y_begin; y < y_end; ++y) {
            float* row = out + (size_t)y * pitch;
            for (uint32_t x = 0; x < w; ++x) row[x] = 1.0f;
            for (uint32_t x = w; x < pitch; ++x) row[x] = 1.0f;
        }
        for (const Rect& q : rects) {
            uint32_t ya = std::max(q.y0, y_begin), yb = std::min(q.y1, y_end);
            for (uint32_t y = ya; y < yb; ++y) {
                float* row = out + (size_t)y * pitch;
                for (uint32_t x = q.x0; x < q.x1; ++x) row[x] = q.z < row[x] ? q.z : row[x];
            }
        }
    });
    return HELIO_OK;
}

}  // extern "C"
