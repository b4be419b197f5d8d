// shadow_device.cuh — the three stages of the per-face shadow frustum cull
// (ShadowCullPass, crates/helio-pass-shadow-cull/src/lib.rs:246-328,
// shaders/shadow_cull.wgsl:49-96) as block-level device functions, shared by the
// standalone launches (shadow_cull.cu) and the batched kernel (batch.cu), which runs
// them as units of its own phases.
//
// Per movable draw and per dirty shadow face (at most 256): the draw's instance sphere
// against the face's six planes, built from the columns of its matrix (c3 + c0,
// c3 - c0, c3 + c1, c3 - c1, c2, c3 - c2), each divided by the length of its normal
// when that exceeds 1e-10; the draw is culled when some plane gives
// (dot(n, c) + w) + r < 0, and skipped when r <= 0. The reference appends the visible
// draws of a face with an atomic counter, so their order within the face is not
// defined; here it is the draw order, and face_counts[f] counts all of them as the
// reference's counter does (only the first 4096 are stored).
//
// Stages (no atomics on the data path; every block first lists the dirty faces in
// ascending order from the 256 dirty words):
//   test   block of 256 draws x chunks of 32 dirty faces: the chunk's planes (one per
//          thread), then one ballot word per (face, 32 draws) and one count per
//          (face, block);
//   scan   dirty face j: exclusive scan of its block counts and its total; the counts
//          of clean faces are cleared (lib.rs:266-270);
//   place  block of 256 draws x chunks of 32 dirty faces: the chunk's ballot words,
//          per-warp prefixes and block offsets staged in shared memory with one round
//          trip, then each visible draw stored at block offset + rank in the block.
#pragma once

#include "common.cuh"

namespace helio {

constexpr uint32_t kShadowFaces = HELIO_SHADOW_MAX_FACES;
constexpr uint32_t kShadowMaxPerFace = HELIO_SHADOW_MAX_DRAWS_PER_FACE;
constexpr uint32_t kShadowThreads = 256;  // draws per block; threads of every stage's block
constexpr uint32_t kShadowWarps = kShadowThreads / 32;
constexpr uint32_t kShadowChunk = 32;     // dirty faces a block stages at once
static_assert(kShadowThreads == kShadowFaces, "one thread per face when a block lists the dirty faces");
static_assert(kShadowChunk * kShadowWarps == kShadowThreads, "one thread per (face, warp) of a chunk");
static_assert(kShadowChunk * 6 <= kShadowThreads, "one thread per plane of a chunk");

struct ShadowDev {
    const float* matrices;  // [256][16], column-major
    const HelioGpuInstanceData* instances;
    const HelioDrawIndexedIndirectArgs* src;
    const uint32_t* face_dirty;  // [256]
    uint32_t instance_count, draw_count, blocks, words;
    uint32_t* bits;         // [256][words]
    uint32_t* block_counts; // [256][blocks]
    uint32_t* block_offs;   // [256][blocks]
    HelioDrawIndexedIndirectArgs* dst;  // [256][4096]
    uint32_t* face_counts;              // [256]
};

// Shared memory of one block running a stage.
struct ShadowSmem {
    float4 pl[kShadowChunk][6];                 // test: the chunk's planes
    uint32_t word[kShadowChunk][kShadowWarps];  // test: visible per (face, warp); place: ballot words
    uint32_t pre[kShadowChunk][kShadowWarps];   // place: visible draws of the block before each warp
    uint32_t off[kShadowChunk];                 // place: the block's first slot in each face
    uint32_t active[kShadowFaces];
    uint32_t warp[kShadowWarps];
};

// normalize_plane (shadow_cull.wgsl:49-55).
__device__ __forceinline__ float4 shadow_normalize(float4 p) {
    const float len = fsqrt(fadd(fadd(fmul(p.x, p.x), fmul(p.y, p.y)), fmul(p.z, p.z)));
    if (len > 1e-10f) return make_float4(fdiv(p.x, len), fdiv(p.y, len), fdiv(p.z, len), fdiv(p.w, len));
    return p;
}

// The dirty faces in ascending order into s.active; returns their number. Every thread
// of the (256-thread) block calls it.
__device__ __forceinline__ uint32_t shadow_list_dirty(const uint32_t* face_dirty, ShadowSmem& s) {
    const uint32_t f = threadIdx.x, lane = f & 31u, warp = f >> 5;
    const bool dirty = face_dirty[f] != 0u;
    const uint32_t bal = __ballot_sync(0xffffffffu, dirty);
    __syncthreads();  // the block's previous use of s is over
    if (lane == 0) s.warp[warp] = __popc(bal);
    __syncthreads();
    uint32_t before = 0, n = 0;
    for (uint32_t w = 0; w < kShadowWarps; ++w) {
        if (w < warp) before += s.warp[w];
        n += s.warp[w];
    }
    if (dirty) s.active[before + __popc(bal & ((1u << lane) - 1u))] = f;
    __syncthreads();
    return n;
}

// Plane i of sphere_in_frustum (shadow_cull.wgsl:58-68) for the column-major matrix m:
// c3 + c0, c3 - c0, c3 + c1, c3 - c1, c2, c3 - c2, normalised.
__device__ __forceinline__ float4 shadow_face_plane(const float* m, uint32_t i) {
    const float4* c = reinterpret_cast<const float4*>(m);
    const float4 c3 = c[3];
    float4 p;
    if (i == 4) {
        p = c[2];
    } else {
        const float4 a = c[i == 5 ? 2 : i >> 1];
        p = (i & 1u) || i == 5 ? make_float4(fsub(c3.x, a.x), fsub(c3.y, a.y), fsub(c3.z, a.z), fsub(c3.w, a.w))
                               : make_float4(fadd(c3.x, a.x), fadd(c3.y, a.y), fadd(c3.z, a.z), fadd(c3.w, a.w));
    }
    return shadow_normalize(p);
}

// The draw's sphere, or r = 0 when the draw is skipped (outside the draw list, an
// instance index past the instance array, or r <= 0; a NaN radius goes on, as in the
// reference's `radius <= 0.0` test).
__device__ __forceinline__ float4 shadow_draw_sphere(const ShadowDev& D, uint32_t d, bool& live) {
    live = false;
    if (d >= D.draw_count) return make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t fi = D.src[d].first_instance;
    if (fi >= D.instance_count) return make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 b = __ldg(reinterpret_cast<const float4*>(D.instances[fi].bounds));
    live = !(b.w <= 0.0f);
    return b;
}

__device__ __forceinline__ bool shadow_sphere_in_face(const float4* pl, float4 s) {
    bool in = true;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const float4 p = pl[i];
        const float d = fadd(fadd(fadd(fadd(fmul(p.x, s.x), fmul(p.y, s.y)), fmul(p.z, s.z)), p.w), s.w);
        in = in && !(d < 0.0f);
    }
    return in;
}

// Test stage of draw block `block` against the dirty faces [g_begin, g_end) of the
// ascending dirty list (clamped to the list), 32 faces at a time. Every thread of the
// block calls it.
static __device__ __noinline__ void shadow_test_block(const ShadowDev& D, uint32_t block, uint32_t g_begin,
                                                      uint32_t g_end, ShadowSmem& s) {
    const uint32_t n_active = shadow_list_dirty(D.face_dirty, s);
    const uint32_t g_stop = min(g_end, n_active);
    if (g_begin >= g_stop) return;  // uniform over the block
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t d = block * kShadowThreads + threadIdx.x;
    bool live;
    const float4 sp = shadow_draw_sphere(D, d, live);
    for (uint32_t g0 = g_begin; g0 < g_stop; g0 += kShadowChunk) {
        const uint32_t nf = min(kShadowChunk, g_stop - g0);
        __syncthreads();  // the previous chunk's planes and counts are read
        if (threadIdx.x < nf * 6) {
            const uint32_t j = threadIdx.x / 6, i = threadIdx.x - j * 6;
            s.pl[j][i] = shadow_face_plane(D.matrices + 16 * s.active[g0 + j], i);
        }
        __syncthreads();
        for (uint32_t j = 0; j < nf; ++j) {
            const bool vis = live && shadow_sphere_in_face(s.pl[j], sp);
            const uint32_t bal = __ballot_sync(0xffffffffu, vis);
            if (lane == 0) {
                D.bits[(size_t)s.active[g0 + j] * D.words + (d >> 5)] = bal;
                s.word[j][warp] = __popc(bal);
            }
        }
        __syncthreads();
        if (threadIdx.x < nf) {
            uint32_t c = 0;
            for (uint32_t w = 0; w < kShadowWarps; ++w) c += s.word[threadIdx.x][w];
            D.block_counts[(size_t)s.active[g0 + threadIdx.x] * D.blocks + block] = c;
        }
    }
}

// Scan stage of the j-th dirty face (nothing when there are at most j), and the clear of
// face j's count when face j is clean (j < 256). Every thread of the block calls it.
static __device__ __noinline__ void shadow_scan_face(const ShadowDev& D, uint32_t j, ShadowSmem& s) {
    const uint32_t n_active = shadow_list_dirty(D.face_dirty, s);
    if (threadIdx.x == 0 && j < kShadowFaces && D.face_dirty[j] == 0u) D.face_counts[j] = 0u;
    if (j >= n_active) return;  // uniform over the block
    const uint32_t f = s.active[j], lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t* in = D.block_counts + (size_t)f * D.blocks;
    uint32_t* out = D.block_offs + (size_t)f * D.blocks;
    uint32_t carry = 0;
    for (uint32_t b0 = 0; b0 < D.blocks; b0 += kShadowThreads) {
        const uint32_t b = b0 + threadIdx.x;
        const uint32_t x = b < D.blocks ? __ldcg(in + b) : 0u;
        uint32_t inc = x;
#pragma unroll
        for (uint32_t k = 1; k < 32u; k <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, inc, k);
            if (lane >= k) inc += t;
        }
        if (lane == 31u) s.warp[warp] = inc;
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (uint32_t w = 0; w < kShadowWarps; ++w) {
            if (w < warp) before += s.warp[w];
            total += s.warp[w];
        }
        if (b < D.blocks) out[b] = carry + before + inc - x;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) D.face_counts[f] = carry;
}

// Place stage of draw block `block` for the dirty faces [g_begin, g_end) of the
// ascending dirty list, 32 faces at a time. Every thread of the block calls it.
static __device__ __noinline__ void shadow_place_block(const ShadowDev& D, uint32_t block, uint32_t g_begin,
                                                       uint32_t g_end, ShadowSmem& s) {
    const uint32_t n_active = shadow_list_dirty(D.face_dirty, s);
    const uint32_t g_stop = min(g_end, n_active);
    if (g_begin >= g_stop) return;  // uniform over the block
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t d = block * kShadowThreads + threadIdx.x;
    const bool live = d < D.draw_count;
    HelioDrawIndexedIndirectArgs draw{};
    if (live) draw = D.src[d];
    const uint32_t w0 = block * kShadowWarps;  // the block's first ballot word
    const uint32_t tj = threadIdx.x / kShadowWarps, tw = threadIdx.x % kShadowWarps;  // (face, warp) of this thread
    const uint32_t lt = (1u << lane) - 1u;
    for (uint32_t g0 = g_begin; g0 < g_stop; g0 += kShadowChunk) {
        const uint32_t nf = min(kShadowChunk, g_stop - g0);
        __syncthreads();  // the previous chunk's tables are read
        if (tj < nf) s.word[tj][tw] = __ldcg(D.bits + (size_t)s.active[g0 + tj] * D.words + w0 + tw);
        if (threadIdx.x < nf) s.off[threadIdx.x] = __ldcg(D.block_offs + (size_t)s.active[g0 + threadIdx.x] * D.blocks + block);
        __syncthreads();
        if (tj < nf) {
            uint32_t before = 0;
            for (uint32_t k = 0; k < tw; ++k) before += __popc(s.word[tj][k]);
            s.pre[tj][tw] = before;
        }
        __syncthreads();
        if (!live) continue;
        for (uint32_t j = 0; j < nf; ++j) {
            const uint32_t word = s.word[j][warp];
            if (!((word >> lane) & 1u)) continue;
            const uint32_t pos = s.off[j] + s.pre[j][warp] + __popc(word & lt);
            if (pos < kShadowMaxPerFace) D.dst[(size_t)s.active[g0 + j] * kShadowMaxPerFace + pos] = draw;
        }
    }
}

}  // namespace helio
