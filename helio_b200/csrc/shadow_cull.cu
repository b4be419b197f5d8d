// shadow_cull.cu — the per-face shadow frustum cull (ShadowCullPass,
// crates/helio-pass-shadow-cull/src/lib.rs:246-328, shaders/shadow_cull.wgsl:49-96).
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
// Three launches, no atomics on the data path. Every block first lists the dirty faces
// in ascending order from the 256 dirty words (a ballot and a prefix over 8 warps).
//   test   (block of 256 draws) x (group of 8 dirty faces): the group's planes, then one
//          ballot word per (face, 32 draws) and one count per (face, block);
//   scan   block j: exclusive scan of the block counts of the j-th dirty face and its
//          total; face j's count cleared when face j is clean (lib.rs:266-270);
//   place  the visible draws of each face at block offset + rank in the block.

#include <new>

#include "common.cuh"
#include "host_util.h"

namespace helio {
namespace {

constexpr uint32_t kFaces = HELIO_SHADOW_MAX_FACES;
constexpr uint32_t kMaxPerFace = HELIO_SHADOW_MAX_DRAWS_PER_FACE;
constexpr uint32_t kThreads = 256;       // draws per block of the test and place launches
constexpr uint32_t kWarps = kThreads / 32;
constexpr uint32_t kFaceGroup = 8;       // dirty faces per block of the test and place launches

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

// normalize_plane (shadow_cull.wgsl:49-55).
__device__ __forceinline__ float4 shadow_normalize(float4 p) {
    const float len = fsqrt(fadd(fadd(fmul(p.x, p.x), fmul(p.y, p.y)), fmul(p.z, p.z)));
    if (len > 1e-10f) return make_float4(fdiv(p.x, len), fdiv(p.y, len), fdiv(p.z, len), fdiv(p.w, len));
    return p;
}

static_assert(kThreads == kFaces, "one thread per face when a block lists the dirty faces");

// The dirty faces in ascending order into s_active; returns their number. Every thread
// of the (256-thread) block calls it.
__device__ uint32_t list_dirty_faces(const uint32_t* face_dirty, uint32_t* s_active, uint32_t* s_warp) {
    const uint32_t f = threadIdx.x, lane = f & 31u, warp = f >> 5;
    const bool dirty = face_dirty[f] != 0u;
    const uint32_t bal = __ballot_sync(0xffffffffu, dirty);
    if (lane == 0) s_warp[warp] = __popc(bal);
    __syncthreads();
    uint32_t before = 0, n = 0;
    for (uint32_t w = 0; w < kWarps; ++w) {
        if (w < warp) before += s_warp[w];
        n += s_warp[w];
    }
    if (dirty) s_active[before + __popc(bal & ((1u << lane) - 1u))] = f;
    __syncthreads();
    return n;
}

// Plane i of sphere_in_frustum (shadow_cull.wgsl:58-68) for the column-major matrix m:
// c3 + c0, c3 - c0, c3 + c1, c3 - c1, c2, c3 - c2, normalised.
__device__ float4 face_plane(const float* m, uint32_t i) {
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
__device__ __forceinline__ float4 draw_sphere(const ShadowDev& D, uint32_t d, bool& live) {
    live = false;
    if (d >= D.draw_count) return make_float4(0.f, 0.f, 0.f, 0.f);
    const uint32_t fi = D.src[d].first_instance;
    if (fi >= D.instance_count) return make_float4(0.f, 0.f, 0.f, 0.f);
    const float4 b = __ldg(reinterpret_cast<const float4*>(D.instances[fi].bounds));
    live = !(b.w <= 0.0f);
    return b;
}

__device__ __forceinline__ bool sphere_in_face(const float4* pl, float4 s) {
    bool in = true;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const float4 p = pl[i];
        const float d = fadd(fadd(fadd(fadd(fmul(p.x, s.x), fmul(p.y, s.y)), fmul(p.z, s.z)), p.w), s.w);
        in = in && !(d < 0.0f);
    }
    return in;
}

__global__ void __launch_bounds__(kThreads) shadow_test_kernel(ShadowDev D) {
    __shared__ float4 s_pl[kFaceGroup][6];
    __shared__ uint32_t s_cnt[kFaceGroup][kWarps];
    __shared__ uint32_t s_active[kFaces], s_warp[kWarps];
    const uint32_t n_active = list_dirty_faces(D.face_dirty, s_active, s_warp);
    const uint32_t g0 = blockIdx.y * kFaceGroup;
    if (g0 >= n_active) return;  // uniform over the block
    const uint32_t nf = min(kFaceGroup, n_active - g0);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (threadIdx.x < nf * 6) {
        const uint32_t j = threadIdx.x / 6, i = threadIdx.x - j * 6;
        s_pl[j][i] = face_plane(D.matrices + 16 * s_active[g0 + j], i);
    }
    __syncthreads();
    const uint32_t d = blockIdx.x * kThreads + threadIdx.x;
    bool live;
    const float4 s = draw_sphere(D, d, live);
    for (uint32_t j = 0; j < nf; ++j) {
        const bool vis = live && sphere_in_face(s_pl[j], s);
        const uint32_t bal = __ballot_sync(0xffffffffu, vis);
        const uint32_t f = s_active[g0 + j];
        if (lane == 0) {
            D.bits[(size_t)f * D.words + (d >> 5)] = bal;
            s_cnt[j][warp] = __popc(bal);
        }
    }
    __syncthreads();
    if (threadIdx.x < nf) {
        uint32_t c = 0;
        for (uint32_t w = 0; w < kWarps; ++w) c += s_cnt[threadIdx.x][w];
        D.block_counts[(size_t)s_active[g0 + threadIdx.x] * D.blocks + blockIdx.x] = c;
    }
}

__global__ void __launch_bounds__(kThreads) shadow_scan_kernel(ShadowDev D) {
    __shared__ uint32_t s_warp[kWarps];
    __shared__ uint32_t s_active[kFaces];
    const uint32_t n_active = list_dirty_faces(D.face_dirty, s_active, s_warp);
    if (threadIdx.x == 0 && D.face_dirty[blockIdx.x] == 0u) D.face_counts[blockIdx.x] = 0u;
    if (blockIdx.x >= n_active) return;  // uniform over the block
    const uint32_t f = s_active[blockIdx.x], lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t* in = D.block_counts + (size_t)f * D.blocks;
    uint32_t* out = D.block_offs + (size_t)f * D.blocks;
    uint32_t carry = 0;
    for (uint32_t b0 = 0; b0 < D.blocks; b0 += kThreads) {
        const uint32_t b = b0 + threadIdx.x;
        const uint32_t x = b < D.blocks ? in[b] : 0u;
        uint32_t inc = x;
#pragma unroll
        for (uint32_t k = 1; k < 32u; k <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, inc, k);
            if (lane >= k) inc += t;
        }
        if (lane == 31u) s_warp[warp] = inc;
        __syncthreads();
        uint32_t before = 0, total = 0;
        for (uint32_t w = 0; w < kWarps; ++w) {
            if (w < warp) before += s_warp[w];
            total += s_warp[w];
        }
        if (b < D.blocks) out[b] = carry + before + inc - x;
        carry += total;
        __syncthreads();
    }
    if (threadIdx.x == 0) D.face_counts[f] = carry;
}

__global__ void __launch_bounds__(kThreads) shadow_place_kernel(ShadowDev D) {
    __shared__ uint32_t s_active[kFaces], s_warp[kWarps];
    const uint32_t n_active = list_dirty_faces(D.face_dirty, s_active, s_warp);
    const uint32_t g0 = blockIdx.y * kFaceGroup;
    if (g0 >= n_active) return;
    const uint32_t nf = min(kFaceGroup, n_active - g0);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t d = blockIdx.x * kThreads + threadIdx.x;
    const bool live = d < D.draw_count;
    HelioDrawIndexedIndirectArgs draw{};
    if (live) draw = D.src[d];
    const uint32_t w0 = blockIdx.x * kWarps;  // the block's first ballot word
    for (uint32_t j = 0; j < nf; ++j) {
        const uint32_t f = s_active[g0 + j];
        const uint32_t* fb = D.bits + (size_t)f * D.words;
        // Lanes 0..7 load the block's eight ballot words; an exclusive scan of their bit
        // counts gives every warp the number of visible draws before it in the block.
        const uint32_t mine = lane < kWarps ? fb[w0 + lane] : 0u;
        uint32_t inc = __popc(mine);
#pragma unroll
        for (uint32_t k = 1; k < kWarps; k <<= 1) {
            const uint32_t t = __shfl_up_sync(0xffffffffu, inc, k);
            if (lane >= k) inc += t;
        }
        const uint32_t word = __shfl_sync(0xffffffffu, mine, warp);
        const uint32_t before = __shfl_sync(0xffffffffu, inc, warp) - __popc(word);
        if (!live || !((word >> lane) & 1u)) continue;
        const uint32_t pos =
            D.block_offs[(size_t)f * D.blocks + blockIdx.x] + before + __popc(word & ((1u << lane) - 1u));
        if (pos < kMaxPerFace) D.dst[(size_t)f * kMaxPerFace + pos] = draw;
    }
}

}  // namespace
}  // namespace helio

using helio::DevBuf;

struct helio_shadow_cull_pass {
    DevBuf dst, counts, bits, block_counts, block_offs;
    helio_shadow_cull_inputs in{};
    uint32_t blocks = 0, words = 0;
    bool prepared = false;
};

extern "C" {

int32_t helio_shadow_cull_create(helio_shadow_cull_pass** out) {
    HELIO_ARG(out, "null pointer");
    *out = nullptr;
    helio_shadow_cull_pass* p = new (std::nothrow) helio_shadow_cull_pass();
    if (!p) return helio_fail(HELIO_ERR_RESOURCE, "out of host memory");
    // lib.rs:104-117: 256 faces x 4096 draws of 20 bytes, and 256 counts.
    constexpr size_t F = HELIO_SHADOW_MAX_FACES;
    cudaError_t e = p->dst.ensure(F * HELIO_SHADOW_MAX_DRAWS_PER_FACE * sizeof(HelioDrawIndexedIndirectArgs));
    if (e == cudaSuccess) e = p->counts.ensure(F * 4);
    if (e == cudaSuccess) e = cudaMemset(p->counts.ptr, 0, F * 4);
    if (e != cudaSuccess) {
        delete p;
        return helio_fail(HELIO_ERR_CUDA, "shadow cull buffers: %s", cudaGetErrorString(e));
    }
    *out = p;
    return HELIO_OK;
}

int32_t helio_shadow_cull_prepare(helio_shadow_cull_pass* p, const helio_shadow_cull_inputs* in) {
    HELIO_ARG(p && in, "null pointer");
    HELIO_ARG(in->face_count == 0 || in->draw_count == 0 || (in->shadow_matrices && in->face_dirty),
              "shadow matrices and face dirty words missing");
    HELIO_ARG(in->draw_count == 0 || (in->src_indirect && (in->instances || in->instance_count == 0)),
              "draws or instances missing");
    HELIO_ARG((reinterpret_cast<uintptr_t>(in->shadow_matrices) & 15u) == 0 &&
                  (reinterpret_cast<uintptr_t>(in->instances) & 15u) == 0,
              "shadow_matrices and instances must be 16-byte aligned");
    const uint32_t blocks = (uint32_t)(((uint64_t)in->draw_count + helio::kThreads - 1) / helio::kThreads);
    const uint32_t words = blocks * helio::kWarps;
    constexpr size_t F = HELIO_SHADOW_MAX_FACES;
    HELIO_CK(p->bits.ensure(F * words * 4));
    HELIO_CK(p->block_counts.ensure(F * blocks * 4));
    HELIO_CK(p->block_offs.ensure(F * blocks * 4));
    p->in = *in;
    p->blocks = blocks;
    p->words = words;
    p->prepared = true;
    return HELIO_OK;
}

int32_t helio_shadow_cull_execute(helio_shadow_cull_pass* p, void* stream) {
    HELIO_ARG(p, "null pointer");
    HELIO_ARG(p->prepared, "pass not prepared");
    if (p->in.face_count == 0 || p->in.draw_count == 0) return HELIO_OK;  // lib.rs:261-263
    cudaStream_t s = helio::as_stream(stream);
    helio::ShadowDev D{};
    D.matrices = p->in.shadow_matrices;
    D.instances = p->in.instances;
    D.src = p->in.src_indirect;
    D.face_dirty = p->in.face_dirty;
    D.instance_count = p->in.instance_count;
    D.draw_count = p->in.draw_count;
    D.blocks = p->blocks;
    D.words = p->words;
    D.bits = p->bits.as<uint32_t>();
    D.block_counts = p->block_counts.as<uint32_t>();
    D.block_offs = p->block_offs.as<uint32_t>();
    D.dst = p->dst.as<HelioDrawIndexedIndirectArgs>();
    D.face_counts = p->counts.as<uint32_t>();
    const dim3 grid(p->blocks, helio::kFaces / helio::kFaceGroup);
    helio_launch_begin("shadow_cull", s);
    helio::shadow_test_kernel<<<grid, helio::kThreads, 0, s>>>(D);
    helio::shadow_scan_kernel<<<helio::kFaces, helio::kThreads, 0, s>>>(D);
    helio_launch_note();
    helio::shadow_place_kernel<<<grid, helio::kThreads, 0, s>>>(D);
    helio_launch_note();
    helio_launch_end(s);
    HELIO_CK(cudaGetLastError());
    return HELIO_OK;
}

int32_t helio_shadow_cull_publish(const helio_shadow_cull_pass* p, helio_shadow_cull_outputs* out) {
    HELIO_ARG(p && out, "null pointer");
    out->face_indirect = p->dst.as<HelioDrawIndexedIndirectArgs>();
    out->face_counts = p->counts.as<uint32_t>();
    out->max_faces = HELIO_SHADOW_MAX_FACES;
    out->max_draws_per_face = HELIO_SHADOW_MAX_DRAWS_PER_FACE;
    return HELIO_OK;
}

void helio_shadow_cull_destroy(helio_shadow_cull_pass* p) { delete p; }

}  // extern "C"
