// batch.cu — one persistent, cooperative launch that culls every view of a batch
// against one device-resident virtual-geometry scene.
//
// Per view the results are those of the single-view passes (HiZBuildPass, then
// VirtualGeometryPass's object select and meshlet cull: crates/helio-pass-hiz/,
// crates/helio-pass-virtual-geometry/shaders/vg_cull.wgsl:126-405), with the
// draws of each view compacted in the canonical (object, span, lane) order. The
// work of all views is shared as follows (phases separated by grid barriers):
//
//   0  view constants (planes, camera fields, pyramid descriptor, reject box), one
//      warp per view
//   1  Hi-Z tiles of every view  +  object select: each object is loaded once and
//      tested against a group of views; per (view, object) the selected LOD + 1 is
//      stored and per (view, 256-object chunk) the number of active 64-meshlet spans
//      and of visible objects. An object whose world centre lies outside a view's
//      reject box fails that view's sphere test for certain (see reject_box_warp)
//      and skips it; the remaining (object, view) pairs are compacted per warp into
//      full 32-lane batches for the exact test and the LOD choice
//   2  exclusive scan of the (view, chunk) span counts
//   3  expansion into one list of active spans, view-major, each view padded to a
//      multiple of 32 spans so every group of 32 spans belongs to one view
//   4  meshlet tests: a warp takes a group of 32 spans and packs their meshlets
//      densely into 32-lane windows (window ballots and per-group counts stored)
//   5  exclusive scan of the group counts
//   6  emission of each view's draws at slot = position in the view's order
//
// Grid barriers and the wait for the published views are bounded: a wait that is not
// released after spin_limit polls sets kBatchErrTimeout and ends its CTA (the others
// end at their next barrier, and the second launch returns at once), so the launch
// always ends and reads nothing a timed-out phase left incomplete; the host then
// reports HELIO_ERR_TIMEOUT.

#include "batch.h"
#include "hiz_tile.cuh"
#include "vg_device.cuh"

namespace helio {

namespace {

// Select constants of a view in shared memory. 144 bytes (36 words): the 128-bit
// plane loads of 8 lanes that read 8 consecutive views hit 8 different bank groups.
struct SelView {
    Planes planes;
    float4 pos_near;
    float focal, thr, thr_lo, thr_hi;  // thr_lo / thr_hi: QuotientBound margins of thr
    float4 pad;
};
static_assert(sizeof(SelView) == 144, "SelView layout");

struct SelBox {
    float lo[3], hi[3];
    uint32_t pad[2];
};

// Dynamic shared memory layout (bytes).
constexpr uint32_t kSelectMaxViews = 32;  // views per select unit, at most
constexpr uint32_t kHizTailUnits = 3;      // Hi-Z units per CTA held back for the end of the work queue
constexpr uint32_t kExpandBatch = 8;       // (view, chunk) units per claim of the expansion queue
static_assert(kSelectMaxViews * 8 <= kBatchThreads, "one thread per (view, mask word) in the write-out");
constexpr size_t kSmSelViews = 0;                                               // SelView[kBatchMaxViews]
constexpr size_t kSmSelBox = kSmSelViews + sizeof(SelView) * kBatchMaxViews;    // SelBox[kBatchMaxViews]
constexpr size_t kSmSelLod = kSmSelBox + sizeof(SelBox) * kBatchMaxViews;       // u8[kSelectMaxViews][256]
constexpr size_t kSmSelSpans = kSmSelLod + kSelectMaxViews * kBatchChunk;       // u32[kSelectMaxViews]
constexpr size_t kSmSelMask = kSmSelSpans + 4 * kSelectMaxViews;                // u32[kSelectMaxViews][8]
constexpr size_t kSmSelStats = kSmSelMask + 4 * 8 * kSelectMaxViews;             // u32[kSelectMaxViews][9]
constexpr size_t kSmHizJob = kSmSelStats + 4 * 9 * kSelectMaxViews;             // HizJob
constexpr size_t kSmHizL5 = kSmHizJob + ((sizeof(HizJob) + 15) / 16) * 16;    // float[2][4]
constexpr size_t kSmMisc = kSmHizL5 + 2 * 4 * 4;                              // u32[64]
constexpr size_t kSmTileBegin = kSmMisc + 64 * 4;                             // u32[kBatchMaxViews]
constexpr size_t kSmTotal = kSmTileBegin + 4 * kBatchMaxViews;
// An attached shadow cull's stages use the select units' LOD tile region, which no
// other part of phases 1..3 touches while they run.
constexpr size_t kSmShadow = kSmSelLod;
static_assert(kSmShadow % 16 == 0 && sizeof(ShadowSmem) <= kSelectMaxViews * kBatchChunk,
              "the shadow stages' shared memory fits the LOD tile region");
// Phases 2..6 reuse the region from offset 0.
constexpr size_t kSmTestViews = 0;                                       // CullView per warp
constexpr size_t kSmTestBits = kSmTestViews + sizeof(CullView) * 8;      // u32[8][66]
constexpr int kBits = kWindowsPerWarp + 2;
constexpr size_t kSmTestQueue = kSmTestBits + 8 * kBits * 4;            // u16[8][64]
constexpr size_t kSmVStart = 0;                                          // u32[kBatchMaxViews + 1]
constexpr size_t kSmTestSpheres = ((kSmTestQueue + 8 * 64 * 2) + 15) / 16 * 16;  // float4[8][64]
// The cull kernel (phases 4..6) has its own, small layout: the test phase's region
// from offset 0, then the scan scratch.
constexpr size_t kSm2Misc = kSmTestSpheres + 8 * 64 * 16;  // u32[64]
constexpr size_t kSm2Total = kSm2Misc + 64 * 4;

__device__ __forceinline__ uint32_t ld_cg(const uint32_t* p) { return __ldcg(p); }

// Grid barrier with a bounded wait (all CTAs are co-resident: cooperative launch).
// It releases once gridDim.x + P.barrier_extra CTAs have arrived (barrier_extra is 0
// except in tests of the bounded wait). Returns false, uniformly over the CTA, when
// the wait gave up after P.spin_limit polls: kBatchErrTimeout is set and the caller
// must end the CTA, since the data of the phase before the barrier may be incomplete
// (the other CTAs then time out at their next barrier and end too).
// GPU-scope acquire / release operations of the barrier and the setup counter.
__device__ __forceinline__ uint32_t atom_add_acq_rel(uint32_t* p, uint32_t v) {
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ void red_add_release(uint32_t* p, uint32_t v) {
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Thread 0 of each CTA arrives with an acquire-release add (releasing what the CTA wrote
// before the block barrier); the last arrival resets the count and releases the next
// generation, which the others poll with acquire loads (spinning first, then backing off).
__device__ bool grid_sync(const BatchParams& P) {
    __syncthreads();
    int timed_out = 0;
    if (threadIdx.x == 0) {
        uint32_t* gen = P.barrier + 1;
        const uint32_t g = ld_acquire(gen);
        if (atom_add_acq_rel(P.barrier, 1u) == gridDim.x - 1 + P.barrier_extra) {
            P.barrier[0] = 0u;
            red_add_release(gen, 1u);
        } else {
            uint32_t polls = 0;
            while (ld_acquire(gen) == g) {
                if (++polls > P.spin_limit) {
                    atomicOr(P.error, kBatchErrTimeout);
                    timed_out = 1;
                    break;
                }
                if (polls > 64) __nanosleep(polls < 512 ? 64 : 256);
            }
        }
    }
    return __syncthreads_or(timed_out) == 0;
}

__device__ __forceinline__ uint32_t warp_inclusive(uint32_t x) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t t = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += t;
    }
    return x;
}

// Sum over the CTA; every thread gets the result. s: 9 words of shared memory.
__device__ uint32_t block_sum(uint32_t x, uint32_t* s) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    __syncthreads();
    if (lane == 0) s[warp] = x;
    __syncthreads();
    uint32_t t = 0;
#pragma unroll
    for (int w = 0; w < (int)(kBatchThreads / 32); ++w) t += s[w];
    return t;
}

// Exclusive scan over the CTA; `total` receives the CTA sum. s: 9 words.
__device__ uint32_t block_exclusive(uint32_t x, uint32_t* s, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t inc = warp_inclusive(x);
    __syncthreads();
    if (lane == 31) s[warp] = inc;
    __syncthreads();
    uint32_t before = 0;
    total = 0;
#pragma unroll
    for (int w = 0; w < (int)(kBatchThreads / 32); ++w) {
        const uint32_t t = s[w];
        if (w < warp) before += t;
        total += t;
    }
    return before + inc - x;
}

// out[i] = sum of in[0..i) for i <= n, over the whole grid (two grid barriers).
// Returns false when a barrier timed out (the CTA must end).
__device__ bool grid_exclusive_scan(const BatchParams& P, const uint32_t* in, uint32_t* out, uint32_t n,
                                    uint32_t* s_tmp) {
    const uint32_t G = gridDim.x, b = blockIdx.x, tid = threadIdx.x;
    const uint32_t seg = (n + G - 1) / G;
    const uint32_t b0 = min(n, b * seg), b1 = min(n, b0 + seg);
    uint32_t sum = 0;
    for (uint32_t i = b0 + tid; i < b1; i += kBatchThreads) sum += ld_cg(in + i);
    sum = block_sum(sum, s_tmp);
    if (tid == 0) P.seg_totals[b] = sum;
    if (!grid_sync(P)) return false;
    uint32_t base = 0;
    for (uint32_t k = tid; k < b; k += kBatchThreads) base += ld_cg(P.seg_totals + k);
    base = block_sum(base, s_tmp);
    for (uint32_t t0 = b0; t0 < b1; t0 += kBatchThreads) {
        const uint32_t i = t0 + tid;
        const uint32_t x = i < b1 ? ld_cg(in + i) : 0u;
        uint32_t total;
        const uint32_t ex = block_exclusive(x, s_tmp, total);
        if (i < b1) out[i] = base + ex;
        base += total;
    }
    if (b == G - 1 && tid == 0) out[n] = base;
    return grid_sync(P);
}

// ── Reject box of a view ──────────────────────────────────────────────────────
// sphere_visible_vg rejects (c, r) when some plane gives fl(d_i) < -r, where d_i =
// dot(n_i, c) + w_i is evaluated with 4 roundings, so |fl(d_i) - d_i| <= 5u S_i
// (u = 2^-24, S_i = |n_i.x c.x| + |n_i.y c.y| + |n_i.z c.z| + |w_i|). For every
// valid object of the scene r <= rmax and |c|_1 <= cl1, and the normalised plane
// components are at most 1 + 2^-23 in magnitude, so with
//     s_i = rmax + 2^-20 (cl1 + |w_i| + rmax)
// a centre outside Q = { p : n_i . p + w_i + s_i >= 0 for all i } (exact
// arithmetic on the float planes) has some d_i < -s_i, hence fl(d_i) < -rmax <= -r:
// the sphere test fails for certain. The box is the axis-aligned bound of Q,
// widened and rounded outward to float; a centre outside it is outside Q.
//
// Q is bounded and its vertices are intersections of three planes. Lane t < 20
// solves triple t in double (Cramer's rule) and keeps the point if it satisfies
// every constraint within a relative 1e-7. The box is disabled (infinite, so
// nothing is rejected) when an input is not finite, when one of the eight corner
// triples (one plane of each pair x, y, z) is ill-conditioned (relative
// determinant below 1e-4) or infeasible, when an ill-conditioned triple (relative
// determinant in (1e-12, 1e-4]) lands within a loose 1e-3 of Q (a vertex that
// double precision may have misplaced), or when Q is unbounded: a recession
// direction of Q is a cross product of two normals (lanes 0..14, both signs) that
// no plane rejects.
struct PlaneD {
    double x, y, z, w;  // normal and offset pushed out by s_i
    __device__ double norm() const { return sqrt(x * x + y * y + z * z); }
    __device__ double at(double px, double py, double pz) const { return x * px + y * py + z * pz + w; }
};

// Plane i of `pl` (shared memory, so a lane-dependent i costs no local memory) with
// its offset pushed out by rmax + 2^-20 (cl1 + |w| + rmax).
__device__ __forceinline__ PlaneD pushed_plane(const Planes& pl, int i, double rmax, double cl1) {
    const float4 p = pl.p[i];
    return PlaneD{p.x, p.y, p.z, (double)p.w + rmax + 0x1p-20 * (cl1 + fabs((double)p.w) + rmax)};
}

__device__ void reject_box_warp(const Planes& pl, float rmax_f, float cl1_f, float box[6]) {
    const int lane = threadIdx.x & 31;
    bool finite = isfinite(rmax_f) && isfinite(cl1_f);
    const double rmax = rmax_f, cl1 = cl1_f;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const float4 p = pl.p[i];
        finite = finite && isfinite(p.x) && isfinite(p.y) && isfinite(p.z) && isfinite(p.w);
    }
    auto scale = [&](const PlaneD& q, double x, double y, double z) {
        return (fabs(x) + fabs(y) + fabs(z)) * q.norm() + fabs(q.w) + 1e-30;
    };
    bool bad = !finite;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (finite && lane < 20) {
        // lane -> (a < b < c)
        int a = 0, b = 1, c = 2;
        for (int k = 0; k < lane; ++k) {
            if (++c == 6) {
                if (++b == 5) {
                    ++a;
                    b = a + 1;
                }
                c = b + 1;
            }
        }
        const PlaneD A = pushed_plane(pl, a, rmax, cl1), B = pushed_plane(pl, b, rmax, cl1),
                     Cc = pushed_plane(pl, c, rmax, cl1);
        const double bc[3] = {B.y * Cc.z - B.z * Cc.y, B.z * Cc.x - B.x * Cc.z, B.x * Cc.y - B.y * Cc.x};
        const double ca[3] = {Cc.y * A.z - Cc.z * A.y, Cc.z * A.x - Cc.x * A.z, Cc.x * A.y - Cc.y * A.x};
        const double ab[3] = {A.y * B.z - A.z * B.y, A.z * B.x - A.x * B.z, A.x * B.y - A.y * B.x};
        const double det = A.x * bc[0] + A.y * bc[1] + A.z * bc[2];
        const double rel = fabs(det) / (A.norm() * B.norm() * Cc.norm() + 1e-300);
        const bool corner = a < 2 && b >= 2 && b < 4 && c >= 4;
        double p[3] = {0.0, 0.0, 0.0};
        bool feasible = false, loose = false;
        if (rel > 1e-12) {
#pragma unroll
            for (int k = 0; k < 3; ++k) p[k] = -(A.w * bc[k] + B.w * ca[k] + Cc.w * ab[k]) / det;
            feasible = isfinite(p[0]) && isfinite(p[1]) && isfinite(p[2]);
            loose = feasible;
#pragma unroll
            for (int j = 0; j < 6; ++j) {
                const PlaneD q = pushed_plane(pl, j, rmax, cl1);
                const double sl = q.at(p[0], p[1], p[2]), sc = scale(q, p[0], p[1], p[2]);
                feasible = feasible && sl >= -1e-7 * sc;
                loose = loose && sl >= -1e-3 * sc;
            }
        }
        if (corner && !(rel > 1e-4 && feasible)) bad = true;
        if (!corner && rel > 1e-12 && rel <= 1e-4 && loose) bad = true;
        if (rel > 1e-4 && feasible)
            for (int k = 0; k < 3; ++k) lo[k] = hi[k] = p[k];
    }
    if (finite && lane < 15) {
        int a = 0, b = 1;
        for (int k = 0; k < lane; ++k)
            if (++b == 6) {
                ++a;
                b = a + 1;
            }
        const PlaneD A = pushed_plane(pl, a, rmax, cl1), B = pushed_plane(pl, b, rmax, cl1);
        const double d[3] = {A.y * B.z - A.z * B.y, A.z * B.x - A.x * B.z, A.x * B.y - A.y * B.x};
        const double len = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        if (len > 1e-12 * A.norm() * B.norm()) {
            for (int sgn = -1; sgn <= 1; sgn += 2) {
                bool ray = true;
#pragma unroll
                for (int j = 0; j < 6; ++j) {
                    const PlaneD q = pushed_plane(pl, j, rmax, cl1);
                    ray = ray && sgn * (q.x * d[0] + q.y * d[1] + q.z * d[2]) >= -1e-9 * q.norm() * len;
                }
                if (ray) bad = true;
            }
        }
    }
    bad = __any_sync(0xffffffffu, bad);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            lo[k] = fmin(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
            hi[k] = fmax(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
        }
        if (bad || !(lo[k] <= hi[k])) {
            box[k] = -INFINITY;
            box[3 + k] = INFINITY;
        } else {
            const double pad = 1e-6 * (fabs(lo[k]) + fabs(hi[k]) + rmax + 1.0);
            box[k] = __double2float_rd(lo[k] - pad);
            box[3 + k] = __double2float_ru(hi[k] + pad);
        }
    }
}

// ── Phase 0: view constants ──────────────────────────────────────────────────
__device__ void phase_setup(const BatchParams& P) {
    for (uint32_t v = blockIdx.x; v < P.view_count; v += gridDim.x) {
        if (threadIdx.x >= 32) continue;
        const BatchViewDev& V = P.views[v];
        __shared__ Planes s_pl;
        publish_planes_warp(V.camera.view_proj, s_pl);
        float box[6];
        reject_box_warp(s_pl, __uint_as_float(__ldg(P.scene_bounds)), __uint_as_float(__ldg(P.scene_bounds + 1)),
                        box);
        if (threadIdx.x == 0) {
            for (int k = 0; k < 6; ++k) P.views[v].reject_box[k] = box[k];
            CullView c;
            c.planes = s_pl;
            c.vp = ldg_mat4(V.camera.view_proj);
            c.pos_near = __ldg(reinterpret_cast<const float4*>(V.camera.position_near));
            c.p00 = __ldg(&V.camera.proj[0]);
            c.p11 = __ldg(&V.camera.proj[5]);
            c.focal = fmul(fmul(fabsf(c.p11), (float)V.height), 0.5f);
            c.lod_threshold_px = V.lod_threshold_px;
            for (int l = 0; l < HELIO_HIZ_MAX_MIPS; ++l) {
                c.hiz.levels[l] = V.hiz.levels[l];
                c.hiz.width[l] = V.hiz.lw[l];
                c.hiz.height[l] = V.hiz.lh[l];
                c.hiz.pitch[l] = V.hiz.lpitch[l];
            }
            c.hiz.mip_count = V.hiz.mip_count;
            c.screen_height = V.height;
            c.hiz_mip_count = V.hiz_mip_count;
            c.pad[0] = c.pad[1] = 0u;
            P.cviews[v] = c;
            red_add_release(P.setup_done, 1u);  // the select units wait for every view
        }
        __syncwarp();
    }
}

// ── Phase 1a: one Hi-Z unit: two consecutive tiles of a view (levels 0..6; the
// tails follow the phase barrier) ──
// The view's HizJob stays in shared memory while consecutive tiles of a CTA
// belong to the same view (s_job holds its index, ~0u before the first tile).
__device__ void load_hiz_job(const BatchParams& P, uint32_t v, char* sm) {
    // Warp 0 copies the job word by word.
    uint32_t* dst = reinterpret_cast<uint32_t*>(sm + kSmHizJob);
    const uint32_t* src = reinterpret_cast<const uint32_t*>(&P.views[v].hiz);
    for (uint32_t w = threadIdx.x & 31u; w < sizeof(HizJob) / 4; w += 32u) dst[w] = __ldg(src + w);
}

__device__ void phase_hiz_tile(const BatchParams& P, uint32_t tile, char* sm) {
    const HizJob& J = *reinterpret_cast<const HizJob*>(sm + kSmHizJob);
    volatile uint32_t* s_job = reinterpret_cast<volatile uint32_t*>(sm + kSmMisc);
    const uint32_t* s_tb = reinterpret_cast<const uint32_t*>(sm + kSmTileBegin);
    __syncthreads();  // the previous unit's threads 0 and 32 may still read its level-5 texels / J
    if (threadIdx.x < 32) {
        uint32_t lo = 0, hi = P.view_count - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (s_tb[mid] <= tile) lo = mid;
            else hi = mid - 1;
        }
        if (*s_job != lo) {
            load_hiz_job(P, lo, sm);
            __syncwarp();
            if (threadIdx.x == 0) *s_job = lo;
        }
    }
    __syncthreads();
    // Warps 0..3 take the quadrants of the unit's first tile, warps 4..7 those of its
    // second; each warp reduces its quadrant to level 5 alone, and one barrier brings the
    // quadrants' level-5 texels together for level 6.
    const uint32_t lp = tile - s_tb[*s_job], t0 = 2u * lp, t1 = t0 + 1u;
    const bool has1 = t1 < J.tiles_x * J.tiles_y;  // uniform over the CTA
    const uint32_t warp = threadIdx.x >> 5, half = warp >> 2;
    const int q = (int)(warp & 3u);
    float* s_l5 = reinterpret_cast<float*>(sm + kSmHizL5);  // [2][4]
    if (half == 0u || has1) {
        const uint32_t t = half ? t1 : t0;
        const uint32_t ty = t / J.tiles_x, tx = t - ty * J.tiles_x;
        float v[8][4];
        hiz_quad_load(J, t, q, v);
        hiz_quad_copy0(J, tx * kHizTile, ty * kHizTile, q, v);
        if (J.mip_count > 1) {
            const float m5 = hiz_quad_levels(J, tx * kHizTile, ty * kHizTile, q, v);
            if ((threadIdx.x & 31u) == 0u) s_l5[half * 4u + q] = m5;
        }
    }
    if (J.mip_count <= 6) return;
    __syncthreads();
    if (threadIdx.x == 0) hiz_quad_level6(J, t0, s_l5);
    else if (threadIdx.x == 32 && has1) hiz_quad_level6(J, t1, s_l5 + 4);
}

// ── Phase 1b: object select against a group of views (vg_cull.wgsl:282-352) ──
// Unit = (256-object chunk, group of at most kSelectMaxViews views); lane j of warp
// w holds object chunk * 256 + 32 w + j. Each lane tests its object's world centre
// against the reject boxes of all views of the group (broadcast from shared memory)
// into a bit mask; the warp's (object, view) pairs that pass are then flattened in
// lane-major order and tested exactly, 32 pairs at a time, one pair per lane
// (select_batch). The selected LOD + 1 of the
// unit's pairs collects in a shared tile (zero = culled) that is written out row by
// row; spans and visible objects per view are counted with shared atomics.

// Exact sphere test and LOD walk of the pair (view v_begin + k, object of lane j) on
// each active lane (vg_cull.wgsl:315-336). Every lane of the warp calls it.
__device__ void select_batch(const BatchParams& P, uint32_t chunk, uint32_t v_begin, bool active, uint32_t k,
                             uint32_t j, F3 c, float wr, float max_scale, char* sm) {
    const SelView* s_sv = reinterpret_cast<const SelView*>(sm + kSmSelViews);
    uint8_t* s_lod = reinterpret_cast<uint8_t*>(sm + kSmSelLod);
    uint32_t* s_spans = reinterpret_cast<uint32_t*>(sm + kSmSelSpans);
    uint32_t* s_vmask = reinterpret_cast<uint32_t*>(sm + kSmSelMask);
    uint32_t* s_stats = reinterpret_cast<uint32_t*>(sm + kSmSelStats);
    const uint32_t warp = threadIdx.x >> 5;
    const F3 cj = f3(__shfl_sync(0xffffffffu, c.x, j), __shfl_sync(0xffffffffu, c.y, j),
                     __shfl_sync(0xffffffffu, c.z, j));
    const float wrj = __shfl_sync(0xffffffffu, wr, j), msj = __shfl_sync(0xffffffffu, max_scale, j);
    if (!active) return;
    const SelView& sv = s_sv[v_begin + k];
    if (!sphere_visible_vg(sv.planes, cj, wrj)) return;
    const uint32_t slot = warp * 32u + j;
    const HelioGpuVgObject* obj = P.scene.objects + (chunk * kBatchChunk + slot);
    const uint32_t lod_count = min(__ldg(&obj->lod_count), 8u);
    const float4 e0 = __ldg(reinterpret_cast<const float4*>(obj->lod_errors));
    const float4 e1 = __ldg(reinterpret_cast<const float4*>(obj->lod_errors + 4));
    const float err[8] = {e0.x, e0.y, e0.z, e0.w, e1.x, e1.y, e1.z, e1.w};
    const F3 d = sub3(cj, f3(sv.pos_near.x, sv.pos_near.y, sv.pos_near.z));
    const float dist = fsqrt(dot3(d, d));
    const float closest = fmaxf(fsub(dist, wrj), fmaxf(sv.pos_near.w, 1.0e-4f));
    const QuotientBound qb{sv.thr, sv.thr_lo, sv.thr_hi};
    const float r = quotient_rcp(closest);
    uint32_t lod = 0;
#pragma unroll
    for (uint32_t level = 1; level < 8; ++level) {
        if (level >= lod_count) break;
        // px = err * max_scale * focal / closest; px <= threshold keeps the level.
        if (quotient_le(fmul(fmul(err[level], msj), sv.focal), closest, r, qb)) lod = level;
        else break;
    }
    const uint32_t cnt = __ldg(&obj->lod_meshlet_counts[lod]);
    s_lod[k * kBatchChunk + slot] = (uint8_t)(lod + 1u);
    atomicOr(s_vmask + k * 8u + (slot >> 5), 1u << (slot & 31u));
    if (cnt) atomicAdd(s_spans + k, (cnt + 63u) >> 6);
    // LOD histogram and largest lod_count of the view's visible objects, per unit.
    atomicAdd(s_stats + k * 9u + lod, 1u);
    atomicMax(s_stats + k * 9u + 8u, lod_count);
}

// Position of the r-th (0-based) set bit of x; x has more than r set bits.
__device__ __forceinline__ uint32_t select_bit(uint32_t x, uint32_t r) {
    uint32_t p = 0;
#pragma unroll
    for (uint32_t w = 16; w; w >>= 1) {
        const uint32_t c = __popc(x & ((1u << w) - 1u));
        if (r >= c) {
            r -= c;
            x >>= w;
            p += w;
        }
    }
    return p;
}

// The visible objects of the unit's views, in object order: thread t takes mask word
// w = t % 8 of view k = t / 8 (nv <= 32 views, so nv * 8 <= 256 threads) and writes
// entry slot | LOD << 8 for each set bit of the word, after the entries of the view's
// words 0..w-1 (a scan over the view's 8 lanes). The last word's thread writes the
// (view, chunk) counts; the view's lanes add the unit's share of counters 2..9 (LOD
// histogram) and 10 (largest lod_count - 1).
__device__ void select_write_lists(const BatchParams& P, uint32_t chunk, uint32_t v_begin, uint32_t nv,
                                   const uint8_t* s_lod, const uint32_t* s_vmask, const uint32_t* s_stats,
                                   const uint32_t* s_spans) {
    const uint32_t tid = threadIdx.x, k = tid >> 3, w = tid & 7u;
    const bool has = k < nv;
    const uint32_t m = has ? s_vmask[k * 8u + w] : 0u;
    const uint32_t c = __popc(m);
    uint32_t inc = c;
#pragma unroll
    for (uint32_t d = 1; d < 8u; d <<= 1) {
        const uint32_t x = __shfl_up_sync(0xffffffffu, inc, d, 8);
        if (w >= d) inc += x;
    }
    if (!has) return;
    const uint32_t v = v_begin + k;
    const size_t u = (size_t)v * P.object_chunks + chunk;
    uint16_t* list = P.vis_list + u * kBatchChunk + (inc - c);
    const uint8_t* row = s_lod + k * kBatchChunk;
    for (uint32_t left = m, i = 0; left; left &= left - 1u, ++i) {
        const uint32_t slot = w * 32u + (uint32_t)(__ffs(left) - 1);
        list[i] = (uint16_t)(slot | ((uint32_t)(row[slot] - 1u) << 8));
    }
    if (w == 7u) {
        P.chunk_counts[u] = s_spans[k];
        P.chunk_vis[u] = inc;
    }
    const uint32_t* st = s_stats + k * 9u;
    uint32_t* counters = P.views[v].counters;
    if (st[w]) atomicAdd(counters + 2 + w, st[w]);
    if (w == 0u && st[8]) atomicMax(counters + 10, st[8] - 1u);
}

__device__ void phase_select_chunk(const BatchParams& P, uint32_t chunk, uint32_t v_begin, uint32_t v_end, char* sm) {
    const SelBox* s_box = reinterpret_cast<const SelBox*>(sm + kSmSelBox);
    uint4* s_lod4 = reinterpret_cast<uint4*>(sm + kSmSelLod);
    uint32_t* s_spans = reinterpret_cast<uint32_t*>(sm + kSmSelSpans);
    uint32_t* s_vmask = reinterpret_cast<uint32_t*>(sm + kSmSelMask);
    const uint32_t tid = threadIdx.x, lane = tid & 31u, nv = v_end - v_begin;
    const VgSceneDev& S = P.scene;
    const uint32_t o = chunk * kBatchChunk + tid;
    bool valid = false;
    F3 c = f3(0.f, 0.f, 0.f);
    float wr = 0.0f, max_scale = 0.0f;
    if (o < S.object_count) {
        const HelioGpuVgObject* obj = S.objects + o;
        const uint4 head = __ldg(reinterpret_cast<const uint4*>(obj));
        const float4 lb = __ldg(reinterpret_cast<const float4*>(obj->local_bounds));
        const uint32_t lod_count = min(head.y, 8u), ii = head.x;
        if (lod_count > 0u && ii < S.instance_count) {
            const HelioInstanceCullData cd = load_cull(S.cull + ii);
            const Mat4 model = ldg_mat4(S.instances[ii].model);
            if (cd.valid_transform != 0u) {
                valid = true;
                max_scale = cd.max_scale;
                c = mat4_point3(model, f3(lb.x, lb.y, lb.z));
                wr = fmaxf(fmul(lb.w, cd.max_scale), 0.0f);
            }
        }
    }
    __syncthreads();  // the previous unit is done with the tile and the counters
    constexpr uint32_t kRow4 = kBatchChunk / 16;  // 16-byte words per tile row
    for (uint32_t i = tid; i < nv * kRow4; i += kBatchThreads) s_lod4[i] = make_uint4(0u, 0u, 0u, 0u);
    if (tid < nv) s_spans[tid] = 0u;
    if (tid < nv * 8u) s_vmask[tid] = 0u;
    uint32_t* s_stats = reinterpret_cast<uint32_t*>(sm + kSmSelStats);
    for (uint32_t i = tid; i < nv * 9u; i += kBatchThreads) s_stats[i] = 0u;
    __syncthreads();
    // Bit k of hits: the box of view v_begin + k does not reject this object. The
    // views' tests are independent of one another, so they pipeline. NaN centres are
    // never rejected here; the exact test decides them.
    uint32_t hits = 0;
    if (valid) {
        const float4* bx = reinterpret_cast<const float4*>(s_box + v_begin);  // lo.xyz hi.x | hi.yz pad
#pragma unroll 4
        for (uint32_t k = 0; k < nv; ++k) {
            const float4 a = bx[2 * k], b = bx[2 * k + 1];
            const bool out = (c.x < a.x) | (c.x > a.w) | (c.y < a.y) | (c.y > b.x) | (c.z < a.z) | (c.z > b.y);
            hits |= (out ? 0u : 1u) << k;
        }
    }
    const uint32_t hit_count = __popc(hits);
    const uint32_t hit_inc = warp_inclusive(hit_count);
    const uint32_t total = __shfl_sync(0xffffffffu, hit_inc, 31);
    for (uint32_t base = 0; base < total; base += 32u) {
        const uint32_t i = base + lane;
        // Owner lane j of pair i: the number of lanes whose inclusive count is <= i
        // (binary search over the non-decreasing counts; at most 31 when i < total).
        uint32_t j = 0;
#pragma unroll
        for (uint32_t step = 16; step; step >>= 1)
            if (__shfl_sync(0xffffffffu, hit_inc, j + step - 1u) <= i) j += step;
        const uint32_t hj = __shfl_sync(0xffffffffu, hits, j);
        const uint32_t before = __shfl_sync(0xffffffffu, hit_inc - hit_count, j);
        const bool active = i < total;
        const uint32_t k = active ? select_bit(hj, i - before) : 0u;
        select_batch(P, chunk, v_begin, active, k, j, c, wr, max_scale, sm);
    }
    __syncthreads();
    for (uint32_t i = tid; i < nv * kRow4; i += kBatchThreads) {
        const uint32_t k = i / kRow4, w4 = i - k * kRow4;
        *reinterpret_cast<uint4*>(P.lod + (size_t)(v_begin + k) * P.lod_pitch + chunk * kBatchChunk + w4 * 16u) =
            s_lod4[i];
    }
    select_write_lists(P, chunk, v_begin, nv, reinterpret_cast<const uint8_t*>(sm + kSmSelLod), s_vmask,
                       reinterpret_cast<const uint32_t*>(sm + kSmSelStats), s_spans);
}

// ── Phase 3: expansion into the view-major list of active spans ──────────────
__device__ void phase_expand(const BatchParams& P, char* sm) {
    uint32_t* s_vstart = reinterpret_cast<uint32_t*>(sm + kSmVStart);
    uint32_t* s_tmp = reinterpret_cast<uint32_t*>(sm + kSmMisc);
    const uint32_t V = P.view_count, C = P.object_chunks, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    // Padded first span of every view (a multiple of 32).
    {
        uint32_t padded = 0;
        if (tid < V) {
            const uint32_t a = ld_cg(P.chunk_offs + (size_t)tid * C), e = ld_cg(P.chunk_offs + (size_t)(tid + 1) * C);
            padded = (e - a + 31u) & ~31u;
        }
        uint32_t total;
        const uint32_t ex = block_exclusive(padded, s_tmp, total);
        if (tid < V) s_vstart[tid] = ex;
        if (tid == 0) s_vstart[V] = total;
        __syncthreads();
        if (blockIdx.x == 0)
            for (uint32_t v = tid; v <= V; v += kBatchThreads) P.view_span_start[v] = s_vstart[v];
        if (tid == 0 && total > P.span_capacity) atomicOr(P.error, kBatchErrSpanCapacity);
    }
    // Hi-Z levels 7.. of each view, by warp 0 of CTA v (mod grid), from the level 6
    // that phase 1 wrote (after the view starts, whose block barriers would otherwise
    // hold the CTA's other warps for the tail); the test phase reads them after the
    // next barrier.
    if (warp == 0) {
        const HizJob& J = *reinterpret_cast<const HizJob*>(sm + kSmHizJob);
        for (uint32_t v = blockIdx.x; v < V; v += gridDim.x) {
            if (P.views[v].hiz.mip_count <= 7u) continue;
            load_hiz_job(P, v, sm);
            __syncwarp();
            hiz_tail_warp(J);
            __syncwarp();
        }
    }
    const VgSceneDev& S = P.scene;
    const uint32_t n_units = V * C;
    // Warps claim batches of kExpandBatch units from a queue; batch b holds the units
    // b + k * NB (lane k < kExpandBatch), strided so that the heavy consecutive chunks of
    // a large view spread over many batches, and small enough that warps which drew light
    // batches draw more of them. A warp flattens its batch's visible lists into one
    // sequence: round r gives lane i the entry 32 r + i, so the list and object loads of
    // every unit are in flight together (two round trips per round instead of two per
    // unit). The spans of an entry go to its unit's first span + the spans of the unit's
    // earlier entries: a scan of the span counts within the round, less the scan before
    // the unit's first entry in the round, plus what the unit wrote in earlier rounds
    // (carried by the unit's lane).
    const uint32_t NB = (n_units + kExpandBatch - 1) / kExpandBatch;
    for (;;) {
        uint32_t bq = 0;
        if (lane == 0) bq = atomicAdd(P.expand_work, 1u);
        bq = __shfl_sync(0xffffffffu, bq, 0);
        if (bq >= NB) break;
        const size_t u = bq + (size_t)lane * NB;
        const bool live = (uint32_t)lane < kExpandBatch && u < n_units;
        const uint32_t vis = live ? ld_cg(P.chunk_vis + u) : 0u;
        if (!__any_sync(0xffffffffu, vis != 0u)) continue;
        const uint32_t v = live ? (uint32_t)(u / C) : 0u, ch = live ? (uint32_t)(u - (size_t)v * C) : 0u;
        uint32_t pos = 0;  // the unit's first span in the view-major list
        if (vis) pos = s_vstart[v] + (ld_cg(P.chunk_offs + u) - ld_cg(P.chunk_offs + (size_t)v * C));
        const uint32_t inc_vis = warp_inclusive(vis);
        const uint32_t first_e = inc_vis - vis, total = __shfl_sync(0xffffffffu, inc_vis, 31);
        uint32_t written = 0;  // spans this lane's unit has written in earlier rounds
        for (uint32_t base = 0; base < total; base += 32u) {
            const uint32_t e = base + lane;
            const int j = owner_lane(first_e, e);  // the unit (lane) owning entry e
            const uint32_t jfirst = __shfl_sync(0xffffffffu, first_e, j);
            const uint32_t jv = __shfl_sync(0xffffffffu, v, j), jch = __shfl_sync(0xffffffffu, ch, j);
            const uint32_t jpos = __shfl_sync(0xffffffffu, pos, j), jdone = __shfl_sync(0xffffffffu, written, j);
            const size_t ju = bq + (size_t)j * NB;
            uint32_t count = 0, first = 0, inst = 0, lod = 0, o = 0;
            if (e < total) {
                const uint32_t en = __ldcg(P.vis_list + ju * kBatchChunk + (e - jfirst));
                lod = en >> 8;
                o = jch * kBatchChunk + (en & 0xFFu);
                const HelioGpuVgObject* obj = S.objects + o;
                count = __ldg(&obj->lod_meshlet_counts[lod]);
                first = __ldg(&obj->lod_first_meshlets[lod]);
                inst = __ldg(&obj->instance_index);
            }
            const uint32_t ns = (count + 63u) >> 6;
            const uint32_t inc = warp_inclusive(ns);
            // Lane of the unit's first entry in this round, and the scan before it.
            const uint32_t lead = jfirst > base ? jfirst - base : 0u;
            // Every lane takes part in the shuffle (its source differs per lane).
            const uint32_t inc_before_lead = __shfl_sync(0xffffffffu, inc, lead ? lead - 1u : 0u);
            const uint32_t before = lead ? inc_before_lead : 0u;
            uint32_t p = jpos + jdone + (inc - ns - before);
            for (uint32_t q = 0; q < ns; ++q, ++p) {
                if (p < P.span_capacity)
                    P.spans[p] = make_uint4(first + 64u * q, min(64u, count - 64u * q) | (lod << 8) | (jv << 16), inst, o);
            }
            // Each unit's lane adds the spans its entries wrote in this round.
            const uint32_t lo = first_e > base ? first_e - base : 0u;
            const uint32_t end = inc_vis > base ? min(inc_vis - base, 32u) : 0u;  // one past the unit's last lane here
            const uint32_t at_end = __shfl_sync(0xffffffffu, inc, end ? end - 1u : 0u);
            const uint32_t at_lo = __shfl_sync(0xffffffffu, inc, lo ? lo - 1u : 0u);
            if (vis && end > lo && lo < 32u) written += at_end - (lo ? at_lo : 0u);
        }
    }
    // Padding spans (n = 0) complete every view to a multiple of 32.
    for (uint32_t v = blockIdx.x; v < V; v += gridDim.x) {
        const uint32_t end = ld_cg(P.chunk_offs + (size_t)(v + 1) * C) - ld_cg(P.chunk_offs + (size_t)v * C);
        for (uint32_t p = s_vstart[v] + end + tid; p < s_vstart[v + 1]; p += kBatchThreads)
            if (p < P.span_capacity) P.spans[p] = make_uint4(0u, v << 16, 0u, 0u);
    }
    // The attached shadow cull's placement: after their expansion, CTAs claim blocks of
    // 256 draws from a queue, so that CTAs whose warps finished early take more.
    if (P.shadow_blocks) {
        volatile uint32_t* s_claim = s_tmp + 20;
        for (;;) {
            __syncthreads();  // every thread has read the previous claim
            if (tid == 0) *s_claim = atomicAdd(P.shadow_work, 1u);
            __syncthreads();
            const uint32_t b = *s_claim;
            if (b >= P.shadow_blocks) break;
            shadow_place_block(P.shadow, b, 0u, kShadowFaces, *reinterpret_cast<ShadowSmem*>(sm + kSmShadow));
        }
    }
}

// The 32 spans of a group (lane = span): meshlet range and packing offsets.
struct GroupSpans {
    uint32_t n, first, inst, lod, off, total, view;
};

__device__ __forceinline__ GroupSpans load_group(const BatchParams& P, uint32_t g) {
    const int lane = threadIdx.x & 31;
    const ActiveSpan s = __ldcg(P.spans + (size_t)g * 32u + lane);
    GroupSpans r;
    r.n = span_n(s);
    r.first = s.x;
    r.inst = s.z;
    r.lod = span_lod(s);
    r.view = __shfl_sync(0xffffffffu, span_view(s), 0);
    const uint32_t inc = warp_inclusive(r.n);
    r.off = inc - r.n;
    r.total = __shfl_sync(0xffffffffu, inc, 31);
    return r;
}

// ── Phase 4: meshlet tests of every group of 32 spans ────────────────────────
// Hi-Z tests of n <= 32 queued candidates of a group: lane i takes entry i, a
// meshlet position s of the group with the world sphere the frustum test computed;
// visible ones set bit s of the group's bits.
__device__ void test_hiz_batch(const CullView& cv, const uint16_t* q, const float4* spheres, uint32_t n,
                               uint32_t* bits) {
    const uint32_t lane = threadIdx.x & 31u;
    if (lane >= n) return;
    const uint32_t s = q[lane];
    const float4 sp = spheres[lane];
    if (meshlet_hiz_visible<true>(cv, f3(sp.x, sp.y, sp.z), sp.w)) atomicOr(bits + (s >> 5), 1u << (s & 31u));
}

// Per group of 32 spans, the warp runs the frustum and cone tests window by window
// (32 meshlets packed densely across the spans) and queues the meshlets that pass;
// every 32 queued meshlets take the Hi-Z test together, so that the costly Hi-Z
// test runs on full warps although about half the meshlets leave earlier.
__device__ void phase_test(const BatchParams& P, uint32_t groups, char* sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    CullView& cv = *reinterpret_cast<CullView*>(sm + kSmTestViews + sizeof(CullView) * warp);
    uint32_t* bits = reinterpret_cast<uint32_t*>(sm + kSmTestBits) + warp * kBits;
    uint16_t* q = reinterpret_cast<uint16_t*>(sm + kSmTestQueue) + warp * 64;
    float4* qs = reinterpret_cast<float4*>(sm + kSmTestSpheres) + warp * 64;
    const uint32_t lt = (1u << lane) - 1u;
    const VgSceneDev& S = P.scene;
    uint32_t cached_view = 0xFFFFFFFFu;
    // Warps claim groups from a queue (a group's work ranges from one window to 64) when
    // they are done with the previous one. (Claiming the next group ahead ties it to a
    // warp that is still busy: the queue's last groups then wait.) The queue hands out
    // the groups from the last view's end backwards: the main view, whose groups are the
    // lightest, then fills the queue's tail (89.8 against 93.0 us in view order).
    for (;;) {
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(P.test_work, 1u);
        g = __shfl_sync(0xffffffffu, g, 0);
        if (g >= groups) break;
        g = groups - 1u - g;
        const GroupSpans gs = load_group(P, g);
        if (gs.view >= P.view_count) continue;  // never true: every span below the group count is written
        if (gs.view != cached_view) {
            const uint4* src = reinterpret_cast<const uint4*>(P.cviews + gs.view);
            uint4* dst = reinterpret_cast<uint4*>(&cv);
            for (int k = lane; k < (int)(sizeof(CullView) / 16); k += 32) dst[k] = __ldcg(src + k);
            cached_view = gs.view;
        }
        for (int k = lane; k < kBits; k += 32) bits[k] = 0u;
        __syncwarp();
        const uint32_t windows = (gs.total + 31u) >> 5;
        uint32_t qn = 0;  // warp-uniform
        for (uint32_t win = 0; win < windows; ++win) {
            const uint32_t s = win * 32u + lane;
            const int j = owner_lane(gs.off, s);
            const uint32_t j_off = __shfl_sync(0xffffffffu, gs.off, j);
            const uint32_t j_first = __shfl_sync(0xffffffffu, gs.first, j);
            const uint32_t j_inst = __shfl_sync(0xffffffffu, gs.inst, j);
            bool cand = false;
            F3 c = f3(0.f, 0.f, 0.f);
            float wr = 0.0f;
            if (s < gs.total) {
                const uint32_t mi = j_first + (s - j_off);
                if (mi < S.meshlet_count) {
                    const HelioGpuInstanceData* in = S.instances + j_inst;
                    const HelioInstanceCullData cd = load_cull(S.cull + j_inst);
                    const Mat4 model = ldg_mat4(in->model);
                    cand = meshlet_frustum_cone_lazy(cv, S, mi, in, model, cd, c, wr);
                }
            }
            const uint32_t b = __ballot_sync(0xffffffffu, cand);
            if (cand) {
                const uint32_t at = qn + __popc(b & lt);
                q[at] = (uint16_t)s;
                qs[at] = make_float4(c.x, c.y, c.z, wr);
            }
            qn += __popc(b);
            if (qn >= 32u) {
                __syncwarp();
                test_hiz_batch(cv, q, qs, 32u, bits);
                __syncwarp();
                const uint32_t rest = qn - 32u;
                const bool mv = (uint32_t)lane < rest;
                const uint16_t x = mv ? q[32 + lane] : (uint16_t)0;
                const float4 xs = mv ? qs[32 + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
                __syncwarp();
                if (mv) {
                    q[lane] = x;
                    qs[lane] = xs;
                }
                __syncwarp();
                qn = rest;
            }
        }
        if (qn) {
            __syncwarp();
            test_hiz_batch(cv, q, qs, qn, bits);
        }
        __syncwarp();
        uint32_t count = __popc(bits[lane]) + __popc(bits[lane + 32]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) count += __shfl_xor_sync(0xffffffffu, count, o);
        if (lane == 0) P.group_counts[g] = count;
        if (count)
            for (uint32_t k = lane; k < windows; k += 32) P.group_bits[(size_t)g * kWindowsPerWarp + k] = bits[k];
        if (P.span_vis) {
            const uint2 w = bit_field64(bits, gs.off, gs.n);
            reinterpret_cast<uint2*>(P.span_vis)[(size_t)g * 32u + lane] = w;
        }
        __syncwarp();
    }
}

// Visible meshlets of a group: the set bits of all its window ballots (lane k holds
// windows k and k + 32).
__device__ __forceinline__ uint32_t cnt_of(uint32_t lo, uint32_t hi) {
    uint32_t c = __popc(lo) + __popc(hi);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    return c;
}

// ── Phase 6: emission, per view, in the canonical order ───────────────────────
// The loads of one group that do not depend on another group's data: its scan offset,
// lane k's span and lane k's two window ballots (windows k and k + 32; the ballot row has
// kWindowsPerWarp entries, read whole and masked to the group's windows later).
struct EmitLoads {
    uint32_t goff, bits_lo, bits_hi;
    ActiveSpan span;
};

__device__ __forceinline__ EmitLoads emit_loads(const BatchParams& P, uint32_t g) {
    const int lane = threadIdx.x & 31;
    EmitLoads e;
    e.goff = ld_cg(P.group_offs + g);
    e.span = __ldcg(P.spans + (size_t)g * 32u + lane);
    const uint32_t* gbits = P.group_bits + (size_t)g * kWindowsPerWarp;
    e.bits_lo = ld_cg(gbits + lane);
    e.bits_hi = ld_cg(gbits + lane + 32);
    return e;
}

__device__ void phase_emit(const BatchParams& P, uint32_t groups) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const VgSceneDev& S = P.scene;
    const uint32_t gw = blockIdx.x * (kBatchThreads / 32) + warp, GW = gridDim.x * (kBatchThreads / 32);
    // Groups are dealt out strided (lane k of warp w looks at group w + k * W): the heavy
    // consecutive groups of a large view spread over many warps. A warp's groups are
    // software-pipelined: the next group's offset, spans and ballots are loaded before the
    // current group's draws are written, so that those round trips overlap the writes.
    for (uint32_t k0 = 0; gw + (size_t)k0 * GW < groups; k0 += 32u) {
        const size_t gl = gw + (size_t)(k0 + lane) * GW;
        const uint32_t cnt = gl < groups ? ld_cg(P.group_counts + gl) : 0u;
        uint32_t mask = __ballot_sync(0xffffffffu, cnt != 0u);
        if (!mask) continue;
        uint32_t g = gw + (k0 + (__ffs(mask) - 1)) * GW;
        mask &= mask - 1u;
        EmitLoads cur = emit_loads(P, g);
        for (;;) {
            const bool more = mask != 0u;
            const uint32_t g_next = more ? gw + (k0 + (__ffs(mask) - 1)) * GW : 0u;
            mask &= mask - 1u;
            EmitLoads nxt{};
            if (more) nxt = emit_loads(P, g_next);
            // The current group: its spans' packing offsets, then its view's table entry.
            GroupSpans gs;
            gs.n = span_n(cur.span);
            gs.first = cur.span.x;
            gs.inst = cur.span.z;
            gs.lod = span_lod(cur.span);
            gs.view = __shfl_sync(0xffffffffu, span_view(cur.span), 0);
            const uint32_t inc = warp_inclusive(gs.n);
            gs.off = inc - gs.n;
            gs.total = __shfl_sync(0xffffffffu, inc, 31);
            if (gs.view < P.view_count) {
                const BatchViewDev& V = P.views[gs.view];
                const uint32_t first_group = ld_cg(P.view_span_start + gs.view) >> 5;
                const uint32_t cap = V.capacity;
                HelioDrawIndexedIndirectArgs* indirect = V.indirect;
                HelioGpuVgDraw* draws = V.draws;
                uint32_t* counters = V.counters;
                const uint32_t windows = (gs.total + 31u) >> 5;
                const uint32_t bits_lo = (uint32_t)lane < windows ? cur.bits_lo : 0u;
                const uint32_t bits_hi = (uint32_t)lane + 32u < windows ? cur.bits_hi : 0u;
                const uint32_t count = cnt_of(bits_lo, bits_hi);
                uint32_t slot0 = cur.goff - ld_cg(P.group_offs + first_group);
                if (lane == 0) {
                    atomicAdd(counters + 0, count);
                    const unsigned long long end = (unsigned long long)slot0 + count;
                    const unsigned long long lo = slot0 > cap ? slot0 : cap;
                    if (end > lo) atomicAdd(counters + 1, (uint32_t)(end - lo));
                }
                // Windows in groups of 4: the draw records of 4 windows are loaded before
                // any of them is written.
                for (uint32_t w0 = 0; w0 < windows; w0 += 4) {
                    uint4 d[4];
                    uint32_t b[4], mi[4], ji[4], jl[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const uint32_t win = w0 + k;
                        const uint32_t src = win < 32u ? bits_lo : bits_hi;
                        b[k] = win < windows ? __shfl_sync(0xffffffffu, src, win & 31u) : 0u;
                        const uint32_t s = win * 32u + lane;
                        const int j = owner_lane(gs.off, s);
                        const uint32_t j_off = __shfl_sync(0xffffffffu, gs.off, j);
                        const uint32_t j_first = __shfl_sync(0xffffffffu, gs.first, j);
                        ji[k] = __shfl_sync(0xffffffffu, gs.inst, j);
                        jl[k] = __shfl_sync(0xffffffffu, gs.lod, j);
                        mi[k] = j_first + (s - j_off);
                        if ((b[k] >> lane) & 1u) d[k] = __ldg(S.m_draw + mi[k]);
                    }
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        if ((b[k] >> lane) & 1u) {
                            const uint32_t slot = slot0 + __popc(b[k] & ((1u << lane) - 1u));
                            if (slot < cap) {
                                uint32_t* out = reinterpret_cast<uint32_t*>(indirect + slot);
                                out[0] = d[k].y;
                                out[1] = 1u;
                                out[2] = d[k].x;
                                out[3] = d[k].z;
                                out[4] = slot;
                                reinterpret_cast<uint4*>(draws)[slot] = make_uint4(ji[k], mi[k], jl[k], 0u);
                            }
                        }
                        slot0 += __popc(b[k]);
                    }
                }
            }
            if (!more) break;
            cur = nxt;
        }
    }
}

// Block 0 records the global timer after each phase (tracing; a few stores per launch).
__device__ __forceinline__ void stamp(const BatchParams& P, int k) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        P.phase_ns[k] = t;
    }
}

// The views' select constants and reject boxes into shared memory, once the view setup
// has published all of them (thread 0 waits, bounded, for the counter). Returns false,
// uniformly over the CTA, when the wait gave up (kBatchErrTimeout set; the CTA must end).
__device__ bool load_sel_views(const BatchParams& P, char* sm) {
    int timed_out = 0;
    if (threadIdx.x == 0) {
        uint32_t polls = 0;
        while (ld_acquire(P.setup_done) < P.view_count) {
            if (++polls > P.spin_limit) {
                atomicOr(P.error, kBatchErrTimeout);
                timed_out = 1;
                break;
            }
            if (polls > 64) __nanosleep(polls < 512 ? 64 : 256);
        }
    }
    if (__syncthreads_or(timed_out)) return false;
    SelView* s_sv = reinterpret_cast<SelView*>(sm + kSmSelViews);
    for (uint32_t k = threadIdx.x; k < P.view_count; k += kBatchThreads) {
        const CullView* cvp = P.cviews + k;
        SelView sv;
        const uint4* src = reinterpret_cast<const uint4*>(&cvp->planes);
        uint4* dst = reinterpret_cast<uint4*>(&sv.planes);
        for (int w = 0; w < 6; ++w) dst[w] = __ldcg(src + w);
        sv.pos_near = __ldcg(&cvp->pos_near);
        sv.focal = __ldcg(&cvp->focal);
        sv.thr = __ldcg(&cvp->lod_threshold_px);
        const QuotientBound qb = quotient_bound(sv.thr);
        sv.thr_lo = qb.lo;
        sv.thr_hi = qb.hi;
        sv.pad = make_float4(0.f, 0.f, 0.f, 0.f);
        s_sv[k] = sv;
        SelBox bx;
        for (int i = 0; i < 3; ++i) {
            bx.lo[i] = __ldcg(&P.views[k].reject_box[i]);
            bx.hi[i] = __ldcg(&P.views[k].reject_box[3 + i]);
        }
        bx.pad[0] = bx.pad[1] = 0u;
        reinterpret_cast<SelBox*>(sm + kSmSelBox)[k] = bx;
    }
    __syncthreads();
    return true;
}

__global__ void __launch_bounds__(kBatchThreads, 3) batch_kernel(const __grid_constant__ BatchParams P) {
    extern __shared__ __align__(16) char sm[];
    uint32_t* s_tmp = reinterpret_cast<uint32_t*>(sm + kSmMisc);

    stamp(P, 0);
    phase_setup(P);
    // No barrier: the Hi-Z units need nothing from the view setup, and a CTA waits for
    // the published views only before its first select unit (load_sel_views).
    stamp(P, 1);

    // Phase 1: Hi-Z tiles and object chunks share one work list.
    {
        for (uint32_t k = threadIdx.x; k < P.view_count; k += kBatchThreads)
            reinterpret_cast<uint32_t*>(sm + kSmTileBegin)[k] = P.views[k].hiz_pair_begin;
        // Hi-Z tiles (memory bound) and select units (arithmetic bound) are spread
        // evenly through one work queue, so that the CTAs sharing an SM overlap the two
        // kinds of work and CTAs that draw cheap units draw more of them. Thread 0
        // claims the next unit while the block works on the current one. The first h0
        // units are Hi-Z tiles (two per CTA: time for the view setup to finish); the
        // last h1 units are Hi-Z tiles too (the cheaper kind, so that the queue ends on
        // short units); between them, unit h0 + u is a select unit iff
        // floor((u + 1) S / U) > floor(u S / U) over the U units in between.
        const uint32_t group_cap = min(max(P.select_views, 1u), kSelectMaxViews);
        const uint32_t vgroups = (P.view_count + group_cap - 1) / group_cap;
        const uint32_t gsize = (P.view_count + vgroups - 1) / vgroups;  // balanced view groups
        const uint32_t sel_units = P.object_chunks * vgroups;
        const uint32_t units = P.hiz_tiles + sel_units;
        const uint32_t h0 = min(P.hiz_tiles, 2u * gridDim.x);
        const uint32_t h1 = min(P.hiz_tiles - h0, kHizTailUnits * gridDim.x);
        const uint32_t rest = units - h0 - h1;
        bool have_views = false;  // uniform over the CTA
        volatile uint32_t* s_unit = s_tmp + 8;
        if (threadIdx.x == 0) {
            *s_unit = atomicAdd(P.work, 1u);
            s_tmp[0] = ~0u;  // no HizJob in shared memory yet
        }
        __syncthreads();
        unsigned long long t_hiz = 0, t_sel = 0, t0, t1;
        // An attached shadow cull's S test blocks are spread evenly through the queue
        // (they need neither the view setup nor the pyramid): with K = (units + S) / S,
        // queue position q is shadow block (q + 1) / K - 1 when K divides q + 1 and that
        // block exists, else unit q - min(q / K, S) below.
        const uint32_t S = P.shadow_blocks;
        const uint32_t queue = units + S;
        const uint32_t K = S ? queue / S : 1u;
        for (;;) {
            const uint32_t q = *s_unit;
            if (q >= queue) break;
            uint32_t next = 0;
            if (threadIdx.x == 0) next = atomicAdd(P.work, 1u);
            if (S && (q + 1u) % K == 0u && (q + 1u) / K <= S) {
                shadow_test_block(P.shadow, (q + 1u) / K - 1u, 0u, kShadowFaces,
                                  *reinterpret_cast<ShadowSmem*>(sm + kSmShadow));
                __syncthreads();  // every thread has read *s_unit
                if (threadIdx.x == 0) *s_unit = next;
                __syncthreads();
                continue;
            }
            const uint32_t u = S ? q - min(q / K, S) : q;
            const bool mid = u >= h0 && u - h0 < rest;
            const uint32_t ur = mid ? u - h0 : 0u;
            const uint32_t sel_before = mid ? (uint32_t)((uint64_t)ur * sel_units / rest) : 0u;
            const bool is_hiz = !mid || (uint32_t)((uint64_t)(ur + 1) * sel_units / rest) == sel_before;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
            if (is_hiz) {
                // Prefix tiles 0..h0-1, then the middle's tiles, then the last h1 tiles.
                phase_hiz_tile(P, u < h0 ? u : (mid ? h0 + ur - sel_before : u - sel_units), sm);
            } else {
                if (!have_views) {
                    if (!load_sel_views(P, sm)) return;
                    have_views = true;
                }
                const uint32_t chunk = sel_before / vgroups, vg = sel_before - chunk * vgroups;
                phase_select_chunk(P, chunk, vg * gsize, min(P.view_count, (vg + 1) * gsize), sm);
            }
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
            (is_hiz ? t_hiz : t_sel) += t1 - t0;
            __syncthreads();  // every thread has read *s_unit
            if (threadIdx.x == 0) *s_unit = next;
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            atomicMax(P.phase_ns + 8, t_hiz);
            atomicMax(P.phase_ns + 9, t_sel);
        }
    }
    if (!grid_sync(P)) return;
    stamp(P, 2);
    // The attached shadow cull's scan: CTA j takes the j-th dirty face (and clears face
    // j's count when face j is clean); done before the phase's last barrier.
    if (P.shadow_blocks)
        for (uint32_t j = blockIdx.x; j < kShadowFaces; j += gridDim.x)
            shadow_scan_face(P.shadow, j, *reinterpret_cast<ShadowSmem*>(sm + kSmShadow));

    if (!grid_exclusive_scan(P, P.chunk_counts, P.chunk_offs, P.view_count * P.object_chunks, s_tmp)) return;
    stamp(P, 3);
    phase_expand(P, sm);
}

// Phases 4..6 as a second cooperative launch: the meshlet tests need fewer registers
// than the select, so this kernel runs more warps per SM. The kernel boundary is the
// barrier after the expansion.
__global__ void __launch_bounds__(kBatchThreads, 5) batch_cull_kernel(BatchParams P) {
    extern __shared__ __align__(16) char sm[];
    uint32_t* s_tmp = reinterpret_cast<uint32_t*>(sm + kSm2Misc);
    // A barrier of the first launch gave up: its span list may be incomplete.
    if (ld_cg(P.error) & kBatchErrTimeout) return;
    stamp(P, 4);
    const uint32_t total_spans = min(ld_cg(P.view_span_start + P.view_count), P.span_capacity);
    const uint32_t groups = total_spans >> 5;
    phase_test(P, groups, sm);
    if (!grid_sync(P)) return;
    stamp(P, 5);

    if (!grid_exclusive_scan(P, P.group_counts, P.group_offs, groups, s_tmp)) return;
    stamp(P, 6);
    phase_emit(P, groups);
    // End of the launch: the latest block end (no barrier needed).
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
        atomicMax(P.phase_ns + 7, t);
    }
}

__global__ void scene_bounds_kernel(VgSceneDev S, uint32_t* bounds) {
    const uint32_t o = blockIdx.x * blockDim.x + threadIdx.x;
    float wr = 0.0f, cl1 = 0.0f;
    if (o < S.object_count) {
        const HelioGpuVgObject* obj = S.objects + o;
        const uint4 head = __ldg(reinterpret_cast<const uint4*>(obj));
        const uint32_t lod_count = min(head.y, 8u), ii = head.x;
        if (lod_count > 0u && ii < S.instance_count) {
            const HelioInstanceCullData cd = load_cull(S.cull + ii);
            if (cd.valid_transform != 0u) {
                const float4 lb = __ldg(reinterpret_cast<const float4*>(obj->local_bounds));
                const F3 c = mat4_point3(ldg_mat4(S.instances[ii].model), f3(lb.x, lb.y, lb.z));
                wr = fmaxf(fmul(lb.w, cd.max_scale), 0.0f);
                cl1 = fabsf(c.x) + fabsf(c.y) + fabsf(c.z);  // rounding up is not needed: 2^-20 slack
            }
        }
    }
    // Non-negative floats (and NaN above +inf) order like their bit patterns.
    uint32_t a = __float_as_uint(wr), b = __float_as_uint(cl1);
#pragma unroll
    for (int k = 16; k > 0; k >>= 1) {
        a = max(a, __shfl_xor_sync(0xffffffffu, a, k));
        b = max(b, __shfl_xor_sync(0xffffffffu, b, k));
    }
    if ((threadIdx.x & 31) == 0) {
        if (a) atomicMax(bounds, a);
        if (b) atomicMax(bounds + 1, b);
    }
}

}  // namespace

// One CTA per view: the view's first packed draw is the sum of the earlier views'
// published counts; its draws are copied with the CTA's threads.
__global__ void pack_draws_kernel(const BatchViewDev* views, uint32_t V, HelioDrawIndexedIndirectArgs* indirect,
                                  HelioGpuVgDraw* draws, uint32_t* offsets, uint64_t capacity) {
    __shared__ uint32_t s_part[kBatchThreads / 32];
    const uint32_t v = blockIdx.x, tid = threadIdx.x;
    uint32_t before = 0;
    for (uint32_t u = tid; u < v; u += blockDim.x) before += min(__ldg(views[u].counters), views[u].capacity);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) before += __shfl_xor_sync(0xffffffffu, before, o);
    if ((tid & 31u) == 0) s_part[tid >> 5] = before;
    __syncthreads();
    uint64_t base = 0;
    for (uint32_t w = 0; w < blockDim.x / 32; ++w) base += s_part[w];
    const uint32_t n = min(__ldg(views[v].counters), views[v].capacity);
    if (tid == 0) {
        offsets[v] = (uint32_t)(base < capacity ? base : capacity);
        if (v == V - 1) offsets[V] = (uint32_t)(base + n < capacity ? base + n : capacity);
    }
    const uint32_t* src_i = reinterpret_cast<const uint32_t*>(views[v].indirect);
    uint32_t* dst_i = reinterpret_cast<uint32_t*>(indirect);
    const uint64_t room = base >= capacity ? 0u : capacity - base;
    const uint64_t m = (uint64_t)n < room ? (uint64_t)n : room;
    for (uint64_t k = tid; k < m * 5u; k += blockDim.x) dst_i[base * 5u + k] = __ldg(src_i + k);
    const uint4* src_d = reinterpret_cast<const uint4*>(views[v].draws);
    uint4* dst_d = reinterpret_cast<uint4*>(draws);
    for (uint64_t k = tid; k < m; k += blockDim.x) dst_d[base + k] = __ldg(src_d + k);
}

cudaError_t launch_scene_bounds(const VgSceneDev& scene, uint32_t* bounds, cudaStream_t stream) {
    const uint32_t n = scene.object_count;
    if (n) scene_bounds_kernel<<<(n + 255) / 256, 256, 0, stream>>>(scene, bounds);
    return cudaGetLastError();
}

cudaError_t launch_pack_draws(const BatchViewDev* views, uint32_t view_count, HelioDrawIndexedIndirectArgs* indirect,
                              HelioGpuVgDraw* draws, uint32_t* offsets, uint64_t capacity, cudaStream_t stream) {
    if (view_count) pack_draws_kernel<<<view_count, kBatchThreads, 0, stream>>>(views, view_count, indirect, draws,
                                                                                offsets, capacity);
    return cudaGetLastError();
}

size_t batch_dynamic_smem() { return kSmTotal; }

uint32_t batch_max_grid() {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmTotal);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_kernel, kBatchThreads, kSmTotal);
    return (uint32_t)(sms * per_sm);
}

uint32_t batch_cull_max_grid() {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_cull_kernel, kBatchThreads, kSm2Total);
    return (uint32_t)(sms * per_sm);
}

namespace {

cudaError_t launch_coop(const void* fn, uint32_t grid, size_t smem, const BatchParams& p, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(kBatchThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void* args[] = {const_cast<BatchParams*>(&p)};
    return cudaLaunchKernelExC(&cfg, fn, args);
}

}  // namespace

cudaError_t launch_batch(const BatchParams& p, uint32_t grid, uint32_t cull_grid, cudaStream_t stream) {
    cudaError_t e = cudaFuncSetAttribute(batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmTotal);
    if (e != cudaSuccess) return e;
    helio_launch_begin("batch_kernel", stream);
    e = launch_coop(reinterpret_cast<const void*>(batch_kernel), grid, kSmTotal, p, stream);
    helio_launch_end(stream);
    if (e != cudaSuccess) return e;
    helio_launch_begin("batch_cull_kernel", stream);
    e = launch_coop(reinterpret_cast<const void*>(batch_cull_kernel), cull_grid, kSm2Total, p, stream);
    helio_launch_end(stream);
    return e;
}

}  // namespace helio
