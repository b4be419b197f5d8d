// vg_build.cu — the VG input producer: the reference's rebuild_vg_buffers
// (crates/helio/src/scene/virtual_geometry/rebuild.rs:18-58, 98-172) on the device.
//
// The reference walks the dense object slots on the host. A slot is used when its
// mesh exists and has descriptors and LODs (rebuild.rs:29-33, 121-129). Each used
// mesh's descriptors are appended once, at its first reference (rebuild.rs:25-40);
// each used slot appends one object, whose LOD ranges are offset by the mesh's base
// (rebuild.rs:135-152), one instance, ceil(max_meshlet_count / 64) work items
// (rebuild.rs:45-58) and max_meshlet_count draws of capacity (rebuild.rs:158-161).
//
// Here every append position is an exclusive prefix sum over the slots, so all
// slots are placed in parallel with the reference's order:
//   1. first_ref[m] = the smallest used slot of mesh m (atomicMin);
//   2. per slot five counts (used, descriptors if it is its mesh's first reference,
//      work items, first-reference flag, draws), summed per block, the block sums
//      scanned by one block, the totals read back to size the outputs;
//   3. per slot the block-local scan plus its block's base gives its positions: it
//      writes its instance and work items, and a first reference writes its mesh's
//      base and rank;
//   4. per used slot its object record (the LOD offsets need its mesh's base);
//   5. one warp per used mesh copies its descriptors to its base.
// Counts, draws and LOD offsets are checked against u32 where the reference's
// checked arithmetic panics; the call then fails with HELIO_ERR_INVALID_ARG.

#include <algorithm>
#include <cstring>
#include <new>

#include "common.cuh"
#include "host_util.h"

namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kVals = 5;  // used, descriptors, work items, first references, draws
constexpr uint32_t kSub = 4;   // 256-slot sub-blocks per scan block
constexpr uint32_t kScanBlock = kSub * kThreads;  // slots per block of the slot scan
constexpr uint32_t kErrPool = 1u;    // a used mesh's descriptors leave the pool
constexpr uint32_t kErrOffset = 2u;  // an LOD descriptor offset exceeds u32

struct SlotVals {
    uint32_t v[kVals];
    uint32_t mesh;
    bool used, first;
};

// Mesh records are read as 16-byte words (the API requires them 16-byte aligned): a
// warp's lanes usually name different meshes, so every load instruction touches up to
// 32 lines, and wide loads keep the number of such instructions down.
__device__ __forceinline__ uint4 mesh_word(const HelioVgMeshRecord* meshes, uint32_t m, int k) {
    return __ldg(reinterpret_cast<const uint4*>(meshes + m) + k);
}

// Word 0 of the record: first_meshlet, meshlet_count, lod_count, max_meshlet_count.
__device__ __forceinline__ bool head_used(uint4 h) { return h.y > 0u && h.z > 0u; }

__device__ __forceinline__ bool mesh_used(const HelioVgMeshRecord* meshes, uint32_t mesh_count, uint32_t m) {
    return m < mesh_count && head_used(mesh_word(meshes, m, 0));
}

__device__ __forceinline__ SlotVals slot_vals(const helio_vg_build_inputs& in, const uint32_t* first_ref, uint32_t o) {
    SlotVals s{};
    s.mesh = HELIO_VG_NO_MESH;
    if (o >= in.slot_count) return s;
    const uint32_t m = in.slot_mesh[o];
    if (m >= in.mesh_count) return s;
    const uint4 h = mesh_word(in.meshes, m, 0);
    if (!head_used(h)) return s;
    s.mesh = m;
    s.used = true;
    s.first = first_ref[m] == o;
    s.v[0] = 1u;
    s.v[1] = s.first ? h.y : 0u;
    s.v[2] = (uint32_t)(((uint64_t)h.w + HELIO_VG_MESHLETS_PER_WORK_ITEM - 1u) / HELIO_VG_MESHLETS_PER_WORK_ITEM);
    s.v[3] = s.first ? 1u : 0u;
    s.v[4] = h.w;
    return s;
}

constexpr uint32_t kSharedMeshes = 8192;  // libraries up to this size take the shared min-table
constexpr uint32_t kCopies = 32;          // global copies of a small library's table

// first_ref[m] = the smallest used slot of mesh m. Block b takes the contiguous slots
// [b * chunk, (b + 1) * chunk). A small library (at most kSharedMeshes meshes) would
// pile the atomics of the whole grid onto the few L2 lines of its table, so each block
// takes the minimum per mesh in a shared table first and pushes its distinct meshes to
// copy b % kCopies of the global table (first_ref then holds kCopies tables, which
// min_copies_kernel folds); a larger library spreads its atomics by itself and goes
// straight to the one table. A global atomic is skipped when the table already holds
// an earlier slot.
__global__ void __launch_bounds__(kThreads) first_ref_kernel(helio_vg_build_inputs in, uint32_t chunk,
                                                             uint32_t* first_ref, uint32_t* error) {
    __shared__ uint32_t s_first[kSharedMeshes];
    const bool local = in.mesh_count <= kSharedMeshes;
    if (local)
        for (uint32_t k = threadIdx.x; k < in.mesh_count; k += kThreads) s_first[k] = 0xFFFFFFFFu;
    __syncthreads();
    const uint32_t o0 = blockIdx.x * chunk, o1 = (uint32_t)min((uint64_t)o0 + chunk, (uint64_t)in.slot_count);
    for (uint32_t o = o0 + threadIdx.x; o < o1; o += kThreads) {
        const uint32_t m = in.slot_mesh[o];
        if (m >= in.mesh_count) continue;
        const uint4 h = mesh_word(in.meshes, m, 0);
        if (!head_used(h)) continue;
        if ((uint64_t)h.x + h.y > in.pool_count) atomicOr(error, kErrPool);
        if (local) atomicMin(s_first + m, o);
        else if (__ldcg(first_ref + m) > o) atomicMin(first_ref + m, o);
    }
    if (!local) return;
    __syncthreads();
    uint32_t* copy = first_ref + (size_t)(blockIdx.x % kCopies) * in.mesh_count;
    for (uint32_t k = threadIdx.x; k < in.mesh_count; k += kThreads) {
        const uint32_t f = s_first[k];
        if (f != 0xFFFFFFFFu && __ldcg(copy + k) > f) atomicMin(copy + k, f);
    }
}

// Small libraries: first_ref[m] = the minimum of the kCopies tables (copy 0 is first_ref).
__global__ void min_copies_kernel(uint32_t* first_ref, uint32_t mesh_count) {
    for (uint32_t m = blockIdx.x * blockDim.x + threadIdx.x; m < mesh_count; m += gridDim.x * blockDim.x) {
        uint32_t f = first_ref[m];
#pragma unroll 8
        for (uint32_t c = 1; c < kCopies; ++c) f = min(f, first_ref[(size_t)c * mesh_count + m]);
        first_ref[m] = f;
    }
}

// Position of the r-th (0-based) set bit of x; x has more than r set bits, so the
// result is in 0..31.
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t x, uint32_t r) {
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

// Inclusive scans of the kVals values x[k] over a block of T threads at once (one
// exchange through shared memory s[kVals][T / 32]); total[k] gets the block sums.
template <uint32_t T>
__device__ void block_scan5(uint64_t (&x)[kVals], uint64_t (*s)[T / 32], uint64_t (&total)[kVals]) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
    for (uint32_t d = 1; d < 32u; d <<= 1)
#pragma unroll
        for (uint32_t k = 0; k < kVals; ++k) {
            const uint64_t t = __shfl_up_sync(0xffffffffu, x[k], d);
            if (lane >= d) x[k] += t;
        }
    if (lane == 31u)
#pragma unroll
        for (uint32_t k = 0; k < kVals; ++k) s[k][warp] = x[k];
    __syncthreads();
#pragma unroll
    for (uint32_t k = 0; k < kVals; ++k) {
        uint64_t before = 0, sum = 0;
        for (uint32_t w = 0; w < T / 32u; ++w) {
            const uint64_t t = s[k][w];
            if (w < warp) before += t;
            sum += t;
        }
        x[k] += before;
        total[k] = sum;
    }
    __syncthreads();
}

// Sums of the five counts over each block of kScanBlock slots.
__global__ void __launch_bounds__(kThreads) block_sums_kernel(helio_vg_build_inputs in, const uint32_t* first_ref,
                                                              uint64_t* block_tot) {
    __shared__ uint64_t s[kVals][kThreads / 32];
    uint64_t x[kVals] = {0, 0, 0, 0, 0}, total[kVals];
#pragma unroll
    for (uint32_t j = 0; j < kSub; ++j) {
        const SlotVals v = slot_vals(in, first_ref, blockIdx.x * kScanBlock + j * kThreads + threadIdx.x);
#pragma unroll
        for (uint32_t k = 0; k < kVals; ++k) x[k] += v.v[k];
    }
    block_scan5<kThreads>(x, s, total);
    if (threadIdx.x == 0)
#pragma unroll
        for (uint32_t k = 0; k < kVals; ++k) block_tot[(size_t)blockIdx.x * kVals + k] = total[k];
}

// One block: exclusive scan of the block sums of every value; totals[k] = the sums.
// Round r scans blocks [r T, (r + 1) T) (consecutive threads read consecutive blocks)
// and carries its sums into the next round.
constexpr uint32_t kScanThreads = 512;

__global__ void __launch_bounds__(kScanThreads) scan_blocks_kernel(const uint64_t* block_tot, uint32_t blocks,
                                                                   uint64_t* block_base, uint64_t* totals) {
    __shared__ uint64_t s[kVals][kScanThreads / 32];
    uint64_t carry[kVals] = {0, 0, 0, 0, 0};
    for (uint32_t b0 = 0; b0 < blocks; b0 += kScanThreads) {
        const uint32_t b = b0 + threadIdx.x;
        uint64_t x[kVals], own[kVals], total[kVals];
#pragma unroll
        for (uint32_t k = 0; k < kVals; ++k) own[k] = x[k] = b < blocks ? block_tot[(size_t)b * kVals + k] : 0u;
        block_scan5<kScanThreads>(x, s, total);
#pragma unroll
        for (uint32_t k = 0; k < kVals; ++k) {
            if (b < blocks) block_base[(size_t)b * kVals + k] = carry[k] + x[k] - own[k];
            carry[k] += total[k];
        }
    }
    if (threadIdx.x == 0)
#pragma unroll
        for (uint32_t k = 0; k < kVals; ++k) totals[k] = carry[k];
}

struct BuildOut {
    HelioGpuMeshletEntry* meshlets;
    HelioGpuVgObject* objects;
    HelioGpuInstanceData* instances;
    HelioGpuVgWorkItem* items;
    uint32_t* obj_of_slot;  // [slot_count]: object index of a used slot
    uint32_t* mesh_base;    // [mesh_count]: first descriptor of a used mesh in the output
    uint32_t* mesh_order;   // [used meshes]: mesh of each first reference, in slot order
    const uint64_t* totals;  // the scan's kVals totals, then the error word
    uint64_t cap_objects, cap_meshlets, cap_items;  // records the output buffers hold
};

// The output passes are launched before the host has read the scan's totals, with the
// buffers the builder holds. They write only when the totals fit those buffers and the
// reference would not have stopped (a used mesh's descriptors leave the pool, or a count
// exceeds u32); otherwise every thread leaves at once and the host, after reading the
// totals, grows the buffers and runs the passes again (or reports the error).
__device__ __forceinline__ bool outputs_fit(const BuildOut& o) {
    const uint64_t objects = __ldcg(o.totals + 0), descs = __ldcg(o.totals + 1), items = __ldcg(o.totals + 2);
    const uint64_t draws = __ldcg(o.totals + 4);
    const uint32_t err = __ldcg(reinterpret_cast<const uint32_t*>(o.totals + kVals));
    return (err & kErrPool) == 0u && descs <= 0xFFFFFFFFull && items <= 0xFFFFFFFFull && draws <= 0xFFFFFFFFull &&
           objects <= o.cap_objects && descs <= o.cap_meshlets && items <= o.cap_items;
}

// A block of kScanBlock slots, as kSub sub-blocks of 256 in slot order: each sub-block's
// scan plus the block's base and the earlier sub-blocks' sums gives every slot its
// positions.
__global__ void __launch_bounds__(kThreads) place_kernel(helio_vg_build_inputs in, const uint32_t* first_ref,
                                                         const uint64_t* block_base, BuildOut out) {
    __shared__ uint64_t s[kVals][kThreads / 32];
    if (!outputs_fit(out)) return;  // uniform over the grid
    uint64_t carry[kVals];
#pragma unroll
    for (uint32_t k = 0; k < kVals; ++k) carry[k] = block_base[(size_t)blockIdx.x * kVals + k];
    for (uint32_t j = 0; j < kSub; ++j) {
        const uint32_t o = blockIdx.x * kScanBlock + j * kThreads + threadIdx.x;
        const SlotVals v = slot_vals(in, first_ref, o);
        uint64_t x[kVals], total[kVals];
#pragma unroll
        for (uint32_t k = 0; k < kVals; ++k) x[k] = v.v[k];
        block_scan5<kThreads>(x, s, total);  // uniform over the block: every thread takes part
        uint32_t at[kVals];
#pragma unroll
        for (uint32_t k = 0; k < kVals; ++k) {  // the totals fit in u32 (outputs_fit)
            at[k] = (uint32_t)(carry[k] + x[k] - v.v[k]);
            carry[k] += total[k];
        }
        if (v.used) {
            out.obj_of_slot[o] = at[0];
            for (uint32_t i = 0; i < v.v[2]; ++i)
                out.items[at[2] + i] = HelioGpuVgWorkItem{at[0], i * HELIO_VG_MESHLETS_PER_WORK_ITEM};
            if (v.first) {
                out.mesh_base[v.mesh] = at[1];
                out.mesh_order[at[3]] = v.mesh;
            }
        }
    }
}

// One thread per slot. A warp's used slots have consecutive object indices, so the
// warp copies their instances and writes their records as contiguous runs of 16-byte
// words. For the records, lane t of round r
// takes word w = t % 8 of the warp's k-th used slot (k = (32 r + t) / 8), reads that
// word of its mesh record (four whole records per load instruction) and stores it in
// place. The object record is the mesh record with word 0 replaced (object index,
// lod_count, max_meshlet_count, 0) and the LOD firsts (words 4, 5) offset by the
// mesh's base.
__global__ void __launch_bounds__(kThreads) objects_kernel(helio_vg_build_inputs in, BuildOut out, uint32_t* error) {
    static_assert(sizeof(HelioGpuVgObject) == 128 && sizeof(HelioVgMeshRecord) == 128, "record layouts");
    if (!outputs_fit(out)) return;  // uniform over the grid
    const uint32_t o = blockIdx.x * kThreads + threadIdx.x, lane = threadIdx.x & 31u;
    const uint32_t m = o < in.slot_count ? in.slot_mesh[o] : HELIO_VG_NO_MESH;
    const bool used = o < in.slot_count && mesh_used(in.meshes, in.mesh_count, m);
    const uint32_t used_mask = __ballot_sync(0xffffffffu, used);
    if (!used_mask) return;
    const uint32_t lead = __ffs(used_mask) - 1u;
    const uint32_t obj0 = __shfl_sync(0xffffffffu, used ? out.obj_of_slot[o] : 0u, lead);
    const uint32_t n_used = __popc(used_mask);
    // The warp's instances, copied by the whole warp as 16-byte words in order (coalesced
    // reads and writes); done here rather than after the placement scan, whose block
    // barriers would hold the loads back.
    {
        constexpr uint32_t kW = sizeof(HelioGpuInstanceData) / 16;  // 9 words per instance
        const uint32_t slot0 = o - lane;
        const uint4* src = reinterpret_cast<const uint4*>(in.slot_instances);
        uint4* idst = reinterpret_cast<uint4*>(out.instances + obj0);
        const uint32_t words = n_used * kW;
        for (uint32_t w = lane; w < words; w += 32u) {
            const uint32_t k = w / kW;  // k-th used lane of the warp
            idst[w] = src[(size_t)(slot0 + nth_set_bit(used_mask, k)) * kW + (w - k * kW)];
        }
    }
    uint4* dst = reinterpret_cast<uint4*>(out.objects + obj0);
    bool over = false;
    const uint32_t rounds = (n_used * 8u + 31u) / 32u;  // the same for every lane of the warp
    for (uint32_t r = 0; r < rounds; ++r) {
        const uint32_t t = r * 32u + lane, k = min(t >> 3, n_used - 1u), w = t & 7u;
        const uint32_t mk = __shfl_sync(0xffffffffu, m, nth_set_bit(used_mask, k));
        if (t >= n_used * 8u) continue;
        uint4 x = mesh_word(in.meshes, mk, (int)w);
        if (w == 0u) {
            x = make_uint4(obj0 + k, x.z, x.w, 0u);
        } else if (w == 4u || w == 5u) {
            const uint64_t base = out.mesh_base[mk];
            const uint64_t a = base + x.x, b = base + x.y, c = base + x.z, d = base + x.w;
            over |= (a | b | c | d) > 0xFFFFFFFFull;
            x = make_uint4((uint32_t)a, (uint32_t)b, (uint32_t)c, (uint32_t)d);
        }
        dst[t] = x;
    }
    if (over) atomicOr(error, kErrOffset);
}

// One warp per used mesh, in first-reference order: its descriptors, 4 x 16 bytes each.
// The grid is sized for every mesh of the library; the used ones are counted by the scan.
__global__ void copy_descriptors_kernel(helio_vg_build_inputs in, BuildOut out) {
    if (!outputs_fit(out)) return;  // uniform over the grid
    const uint32_t used_meshes = (uint32_t)__ldcg(out.totals + 3);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, W = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = w0; r < used_meshes; r += W) {
        const uint32_t m = out.mesh_order[r];
        const HelioVgMeshRecord& rec = in.meshes[m];
        const uint4* src = reinterpret_cast<const uint4*>(in.pool + rec.first_meshlet);
        uint4* dst = reinterpret_cast<uint4*>(out.meshlets + out.mesh_base[m]);
        const uint64_t words = (uint64_t)rec.meshlet_count * 4u;
        for (uint64_t i = lane; i < words; i += 32u) dst[i] = src[i];
    }
}

uint32_t grid_for(uint64_t n, uint32_t per_block) {
    const uint64_t g = (n + per_block - 1) / per_block;
    return (uint32_t)(g < 1 ? 1 : (g > 65535u * 8u ? 65535u * 8u : g));
}

}  // namespace

using helio::DevBuf;

struct helio_vg_builder {
    DevBuf first_ref, block_tot, block_base, totals, obj_of_slot, mesh_base, mesh_order;
    DevBuf meshlets, objects, instances, items;
    uint32_t meshlet_count = 0, object_count = 0, item_count = 0, max_draw_count = 0;
    uint64_t runs = 0;
    bool valid = false;
};

extern "C" {

int32_t helio_vg_builder_create(helio_vg_builder** out) {
    HELIO_ARG(out, "null pointer");
    *out = new (std::nothrow) helio_vg_builder();
    if (!*out) return helio_fail(HELIO_ERR_RESOURCE, "out of host memory");
    return HELIO_OK;
}

int32_t helio_vg_builder_run(helio_vg_builder* b, const helio_vg_build_inputs* in, void* stream) {
    HELIO_ARG(b && in, "null pointer");
    HELIO_ARG(in->slot_count == 0 || (in->slot_mesh && in->slot_instances), "slot arrays missing");
    HELIO_ARG(in->mesh_count == 0 || in->meshes, "mesh records missing");
    HELIO_ARG(in->pool_count == 0 || in->pool, "descriptor pool missing");
    HELIO_ARG((reinterpret_cast<uintptr_t>(in->pool) & 15u) == 0 &&
                  (reinterpret_cast<uintptr_t>(in->meshes) & 15u) == 0 &&
                  (reinterpret_cast<uintptr_t>(in->slot_instances) & 15u) == 0,
              "pool, meshes and slot_instances must be 16-byte aligned");
    cudaStream_t s = helio::as_stream(stream);
    b->valid = false;
    const uint32_t S = in->slot_count, M = in->mesh_count;
    const uint32_t blocks = S ? (uint32_t)(((uint64_t)S + kScanBlock - 1) / kScanBlock) : 1u;  // slot-scan blocks
    const bool copies = M <= kSharedMeshes;  // first_ref_kernel's small-library form
    HELIO_CK(b->first_ref.ensure((size_t)M * 4 * (copies ? kCopies : 1u)));
    HELIO_CK(b->block_tot.ensure((size_t)blocks * kVals * 8));
    HELIO_CK(b->block_base.ensure((size_t)blocks * kVals * 8));
    HELIO_CK(b->totals.ensure(kVals * 8 + 8));  // totals, then the error word
    HELIO_CK(b->obj_of_slot.ensure((size_t)S * 4));
    HELIO_CK(b->mesh_base.ensure((size_t)M * 4));
    HELIO_CK(b->mesh_order.ensure((size_t)M * 4));
    uint32_t* error = reinterpret_cast<uint32_t*>(b->totals.as<uint64_t>() + kVals);
    if (M) HELIO_CK(cudaMemsetAsync(b->first_ref.ptr, 0xFF, (size_t)M * 4 * (copies ? kCopies : 1u), s));
    HELIO_CK(cudaMemsetAsync(b->totals.ptr, 0, kVals * 8 + 8, s));
    // Launch accounting and the event profiler see one "vg_build" entry per run with
    // slots: helio_launch_end counts the first kernel, helio_launch_note each later one.
    const bool any = S > 0;
    if (any) helio_launch_begin("vg_build", s);
    if (S) {
        const uint32_t chunk = (uint32_t)std::max<uint64_t>(kThreads * 8u, ((uint64_t)S + 1183u) / 1184u);
        first_ref_kernel<<<(uint32_t)(((uint64_t)S + chunk - 1) / chunk), kThreads, 0, s>>>(
            *in, chunk, b->first_ref.as<uint32_t>(), error);
        if (copies && M) {
            min_copies_kernel<<<grid_for(M, kThreads), kThreads, 0, s>>>(b->first_ref.as<uint32_t>(), M);
            helio_launch_note();
        }
        block_sums_kernel<<<blocks, kThreads, 0, s>>>(*in, b->first_ref.as<uint32_t>(), b->block_tot.as<uint64_t>());
        helio_launch_note();
        scan_blocks_kernel<<<1, kScanThreads, 0, s>>>(b->block_tot.as<uint64_t>(), blocks, b->block_base.as<uint64_t>(),
                                                  b->totals.as<uint64_t>());
        helio_launch_note();
    }
    // The output passes with the buffers held now (a first run, or a larger library, finds
    // them too small: the passes then leave at once and run again below, once sized).
    auto outputs = [&]() {
        BuildOut o{b->meshlets.as<HelioGpuMeshletEntry>(), b->objects.as<HelioGpuVgObject>(),
                   b->instances.as<HelioGpuInstanceData>(), b->items.as<HelioGpuVgWorkItem>(),
                   b->obj_of_slot.as<uint32_t>(), b->mesh_base.as<uint32_t>(), b->mesh_order.as<uint32_t>(),
                   b->totals.as<uint64_t>(), 0, 0, 0};
        o.cap_objects = std::min(b->objects.bytes / sizeof(HelioGpuVgObject),
                                 b->instances.bytes / sizeof(HelioGpuInstanceData));
        o.cap_meshlets = b->meshlets.bytes / sizeof(HelioGpuMeshletEntry);
        o.cap_items = b->items.bytes / sizeof(HelioGpuVgWorkItem);
        return o;
    };
    auto launch_outputs = [&](const BuildOut& o) {
        if (!S) return;
        place_kernel<<<blocks, kThreads, 0, s>>>(*in, b->first_ref.as<uint32_t>(), b->block_base.as<uint64_t>(), o);
        helio_launch_note();
        objects_kernel<<<(uint32_t)(((uint64_t)S + kThreads - 1) / kThreads), kThreads, 0, s>>>(*in, o, error);
        helio_launch_note();
        if (M) {
            copy_descriptors_kernel<<<grid_for((uint64_t)M * 32u, kThreads), kThreads, 0, s>>>(*in, o);
            helio_launch_note();
        }
    };
    const BuildOut held = outputs();
    launch_outputs(held);
    // The bracket ends with the last launch, before the read-back (later launches of a run
    // that had to grow its outputs are counted, not timed).
    if (any) helio_launch_end(s);
    cudaError_t e = cudaGetLastError();
    uint64_t tot[kVals + 1] = {0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(tot, b->totals.ptr, sizeof(tot), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    uint32_t err = 0;
    std::memcpy(&err, &tot[kVals], 4);
    const char* why = e != cudaSuccess         ? cudaGetErrorString(e)
                      : (err & kErrPool)       ? "a mesh's descriptor range leaves the pool"
                      : tot[1] > 0xFFFFFFFFull ? "virtual geometry exceeds the u32 descriptor address space"
                      : tot[2] > 0xFFFFFFFFull ? "virtual geometry exceeds the u32 work-item address space"
                      : tot[4] > 0xFFFFFFFFull ? "virtual geometry indirect draw capacity exceeds u32"
                                               : nullptr;
    if (why) return helio_fail(e != cudaSuccess ? HELIO_ERR_CUDA : HELIO_ERR_INVALID_ARG, "%s", why);
    const uint64_t objects = tot[0], descriptors = tot[1], items = tot[2];
    if (objects > held.cap_objects || descriptors > held.cap_meshlets || items > held.cap_items) {
        if ((e = b->meshlets.ensure(descriptors * sizeof(HelioGpuMeshletEntry))) == cudaSuccess &&
            (e = b->objects.ensure(objects * sizeof(HelioGpuVgObject))) == cudaSuccess &&
            (e = b->instances.ensure(objects * sizeof(HelioGpuInstanceData))) == cudaSuccess)
            e = b->items.ensure(items * sizeof(HelioGpuVgWorkItem));
        if (e != cudaSuccess) return helio_fail(HELIO_ERR_CUDA, "vg_build outputs: %s", cudaGetErrorString(e));
        launch_outputs(outputs());
        HELIO_CK(cudaGetLastError());
        HELIO_CK(cudaMemcpyAsync(&err, error, 4, cudaMemcpyDeviceToHost, s));
        HELIO_CK(cudaStreamSynchronize(s));
    }
    HELIO_ARG(!(err & kErrOffset), "virtual geometry descriptor offset overflow");
    b->object_count = (uint32_t)objects;
    b->meshlet_count = (uint32_t)descriptors;
    b->item_count = (uint32_t)items;
    b->max_draw_count = (uint32_t)tot[4];
    b->runs += 1;
    b->valid = true;
    return HELIO_OK;
}

int32_t helio_vg_builder_frame_data(const helio_vg_builder* b, helio_vg_frame_data* out) {
    HELIO_ARG(b && out, "null pointer");
    HELIO_ARG(b->valid, "no successful run");
    std::memset(out, 0, sizeof(*out));
    out->meshlets = b->meshlets.as<HelioGpuMeshletEntry>();
    out->objects = b->objects.as<HelioGpuVgObject>();
    out->instances = b->instances.as<HelioGpuInstanceData>();
    out->work_items = b->items.as<HelioGpuVgWorkItem>();
    out->meshlet_count = b->meshlet_count;
    out->object_count = b->object_count;
    out->work_item_count = b->item_count;
    out->max_draw_count = b->max_draw_count;
    out->buffer_version = b->runs;
    out->instance_version = b->runs;
    out->memory = HELIO_MEM_DEVICE;
    return HELIO_OK;
}

void helio_vg_builder_destroy(helio_vg_builder* b) { delete b; }

}  // extern "C"
