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
//   test   (block of 256 draws) x (chunk of 32 dirty faces): the chunk's planes, then
//          one ballot word per (face, 32 draws) and one count per (face, block);
//   scan   block j: exclusive scan of the block counts of the j-th dirty face and its
//          total; face j's count cleared when face j is clean (lib.rs:266-270);
//   place  (block of 256 draws) x (chunk of 32 dirty faces): the visible draws of each
//          face at block offset + rank in the block.

#include <new>

#include "common.cuh"
#include "host_util.h"
#include "shadow_device.cuh"
#include "shadow_host.h"

namespace helio {
namespace {

constexpr uint32_t kThreads = kShadowThreads;
constexpr uint32_t kWarps = kShadowWarps;
constexpr uint32_t kFaces = kShadowFaces;
constexpr uint32_t kChunk = kShadowChunk;

// Standalone launches: test and place over (block of 256 draws) x (chunk of 32 dirty
// faces), the scan over the 256 faces.
__global__ void __launch_bounds__(kThreads) shadow_test_kernel(const __grid_constant__ ShadowDev D) {
    __shared__ ShadowSmem s;
    const uint32_t g0 = blockIdx.y * kChunk;
    shadow_test_block(D, blockIdx.x, g0, g0 + kChunk, s);
}

__global__ void __launch_bounds__(kThreads) shadow_scan_kernel(const __grid_constant__ ShadowDev D) {
    __shared__ ShadowSmem s;
    shadow_scan_face(D, blockIdx.x, s);
}

__global__ void __launch_bounds__(kThreads) shadow_place_kernel(const __grid_constant__ ShadowDev D) {
    __shared__ ShadowSmem s;
    const uint32_t g0 = blockIdx.y * kChunk;
    shadow_place_block(D, blockIdx.x, g0, g0 + kChunk, s);
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

bool helio::shadow_dev(const helio_shadow_cull_pass* p, ShadowDev* out) {
    if (!p || !p->prepared || p->in.face_count == 0 || p->in.draw_count == 0) return false;
    ShadowDev D{};
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
    *out = D;
    return true;
}

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
    helio::shadow_dev(p, &D);
    const dim3 grid(p->blocks, helio::kFaces / helio::kChunk);
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
