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

#include <cstring>
#include <new>

#include "common.cuh"
#include "host_util.h"

namespace {

constexpr uint32_t kThreads = 256;
constexpr uint32_t kVals = 5;  // used, descriptors, work items, first references, draws
constexpr uint32_t kErrPool = 1u;    // a used mesh's descriptors leave the pool
constexpr uint32_t kErrOffset = 2u;  // an LOD descriptor offset exceeds u32

struct SlotVals {
    uint32_t v[kVals];
    uint32_t mesh;
    bool used, first;
};

__device__ __forceinline__ bool mesh_used(const HelioVgMeshRecord* meshes, uint32_t mesh_count, uint32_t m) {
    return m < mesh_count && meshes[m].meshlet_count > 0u && meshes[m].lod_count > 0u;
}

__device__ __forceinline__ SlotVals slot_vals(const helio_vg_build_inputs& in, const uint32_t* first_ref, uint32_t o) {
    SlotVals s{};
    s.mesh = HELIO_VG_NO_MESH;
    if (o >= in.slot_count) return s;
    const uint32_t m = in.slot_mesh[o];
    if (!mesh_used(in.meshes, in.mesh_count, m)) return s;
    const HelioVgMeshRecord& r = in.meshes[m];
    s.mesh = m;
    s.used = true;
    s.first = first_ref[m] == o;
    s.v[0] = 1u;
    s.v[1] = s.first ? r.meshlet_count : 0u;
    s.v[2] = (uint32_t)(((uint64_t)r.max_meshlet_count + HELIO_VG_MESHLETS_PER_WORK_ITEM - 1u) /
                        HELIO_VG_MESHLETS_PER_WORK_ITEM);
    s.v[3] = s.first ? 1u : 0u;
    s.v[4] = r.max_meshlet_count;
    return s;
}

__global__ void first_ref_kernel(helio_vg_build_inputs in, uint32_t* first_ref, uint32_t* error) {
    for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < in.slot_count; o += gridDim.x * blockDim.x) {
        const uint32_t m = in.slot_mesh[o];
        if (!mesh_used(in.meshes, in.mesh_count, m)) continue;
        const HelioVgMeshRecord& r = in.meshes[m];
        if ((uint64_t)r.first_meshlet + r.meshlet_count > in.pool_count) atomicOr(error, kErrPool);
        atomicMin(first_ref + m, o);
    }
}

// Inclusive scan of a u64 over the block (256 threads); total gets the block sum.
__device__ uint64_t block_inclusive64(uint64_t x, uint64_t* s, uint64_t& total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
    for (uint32_t d = 1; d < 32u; d <<= 1) {
        const uint64_t t = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += t;
    }
    if (lane == 31u) s[warp] = x;
    __syncthreads();
    uint64_t before = 0;
    total = 0;
#pragma unroll
    for (uint32_t w = 0; w < kThreads / 32u; ++w) {
        const uint64_t t = s[w];
        if (w < warp) before += t;
        total += t;
    }
    __syncthreads();
    return before + x;
}

__global__ void __launch_bounds__(kThreads) block_sums_kernel(helio_vg_build_inputs in, const uint32_t* first_ref,
                                                              uint64_t* block_tot) {
    __shared__ uint64_t s[kThreads / 32];
    const SlotVals v = slot_vals(in, first_ref, blockIdx.x * kThreads + threadIdx.x);
    for (uint32_t k = 0; k < kVals; ++k) {
        uint64_t total;
        block_inclusive64(v.v[k], s, total);
        if (threadIdx.x == 0) block_tot[(size_t)blockIdx.x * kVals + k] = total;
    }
}

// One block: exclusive scan of the block sums of every value; totals[k] = the sums.
__global__ void __launch_bounds__(kThreads) scan_blocks_kernel(const uint64_t* block_tot, uint32_t blocks,
                                                               uint64_t* block_base, uint64_t* totals) {
    __shared__ uint64_t s[kThreads / 32];
    for (uint32_t k = 0; k < kVals; ++k) {
        uint64_t carry = 0;
        for (uint32_t b0 = 0; b0 < blocks; b0 += kThreads) {
            const uint32_t b = b0 + threadIdx.x;
            const uint64_t x = b < blocks ? block_tot[(size_t)b * kVals + k] : 0u;
            uint64_t total;
            const uint64_t inc = block_inclusive64(x, s, total);
            if (b < blocks) block_base[(size_t)b * kVals + k] = carry + inc - x;
            carry += total;
        }
        if (threadIdx.x == 0) totals[k] = carry;
    }
}

struct BuildOut {
    HelioGpuMeshletEntry* meshlets;
    HelioGpuVgObject* objects;
    HelioGpuInstanceData* instances;
    HelioGpuVgWorkItem* items;
    uint32_t* obj_of_slot;  // [slot_count]: object index of a used slot
    uint32_t* mesh_base;    // [mesh_count]: first descriptor of a used mesh in the output
    uint32_t* mesh_order;   // [used meshes]: mesh of each first reference, in slot order
};

__global__ void __launch_bounds__(kThreads) place_kernel(helio_vg_build_inputs in, const uint32_t* first_ref,
                                                         const uint64_t* block_base, BuildOut out) {
    __shared__ uint64_t s[kThreads / 32];
    const uint32_t o = blockIdx.x * kThreads + threadIdx.x;
    const SlotVals v = slot_vals(in, first_ref, o);
    uint32_t at[kVals];
    for (uint32_t k = 0; k < kVals; ++k) {
        uint64_t total;
        const uint64_t inc = block_inclusive64(v.v[k], s, total);
        // The totals fit in u32 (checked on the host before this launch).
        at[k] = (uint32_t)(block_base[(size_t)blockIdx.x * kVals + k] + inc - v.v[k]);
    }
    if (!v.used) return;
    out.obj_of_slot[o] = at[0];
    {
        const uint4* src = reinterpret_cast<const uint4*>(in.slot_instances + o);
        uint4* dst = reinterpret_cast<uint4*>(out.instances + at[0]);
#pragma unroll
        for (int w = 0; w < (int)(sizeof(HelioGpuInstanceData) / 16); ++w) dst[w] = src[w];
    }
    for (uint32_t i = 0; i < v.v[2]; ++i)
        out.items[at[2] + i] = HelioGpuVgWorkItem{at[0], i * HELIO_VG_MESHLETS_PER_WORK_ITEM};
    if (v.first) {
        out.mesh_base[v.mesh] = at[1];
        out.mesh_order[at[3]] = v.mesh;
    }
}

__global__ void objects_kernel(helio_vg_build_inputs in, BuildOut out, uint32_t* error) {
    for (uint32_t o = blockIdx.x * blockDim.x + threadIdx.x; o < in.slot_count; o += gridDim.x * blockDim.x) {
        const uint32_t m = in.slot_mesh[o];
        if (!mesh_used(in.meshes, in.mesh_count, m)) continue;
        const HelioVgMeshRecord& r = in.meshes[m];
        const uint32_t idx = out.obj_of_slot[o], base = out.mesh_base[m];
        HelioGpuVgObject ob;
        ob.instance_index = idx;
        ob.lod_count = r.lod_count;
        ob.max_meshlet_count = r.max_meshlet_count;
        ob.reserved = 0u;
        for (int k = 0; k < 4; ++k) ob.local_bounds[k] = r.local_bounds[k];
        for (int l = 0; l < HELIO_VG_LOD_LEVELS; ++l) {
            const uint64_t first = (uint64_t)base + r.lod_first_meshlets[l];
            if (first > 0xFFFFFFFFull) atomicOr(error, kErrOffset);
            ob.lod_errors[l] = r.lod_errors[l];
            ob.lod_first_meshlets[l] = (uint32_t)first;
            ob.lod_meshlet_counts[l] = r.lod_meshlet_counts[l];
        }
        out.objects[idx] = ob;
    }
}

// One warp per used mesh, in first-reference order: its descriptors, 4 x 16 bytes each.
__global__ void copy_descriptors_kernel(helio_vg_build_inputs in, BuildOut out, uint32_t used_meshes) {
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
                  (reinterpret_cast<uintptr_t>(in->slot_instances) & 15u) == 0,
              "pool and slot_instances must be 16-byte aligned");
    cudaStream_t s = helio::as_stream(stream);
    b->valid = false;
    const uint32_t S = in->slot_count, M = in->mesh_count;
    const uint32_t blocks = S ? (S + kThreads - 1) / kThreads : 1u;
    HELIO_CK(b->first_ref.ensure((size_t)M * 4));
    HELIO_CK(b->block_tot.ensure((size_t)blocks * kVals * 8));
    HELIO_CK(b->block_base.ensure((size_t)blocks * kVals * 8));
    HELIO_CK(b->totals.ensure(kVals * 8 + 8));  // totals, then the error word
    HELIO_CK(b->obj_of_slot.ensure((size_t)S * 4));
    HELIO_CK(b->mesh_base.ensure((size_t)M * 4));
    HELIO_CK(b->mesh_order.ensure((size_t)M * 4));
    uint32_t* error = reinterpret_cast<uint32_t*>(b->totals.as<uint64_t>() + kVals);
    if (M) HELIO_CK(cudaMemsetAsync(b->first_ref.ptr, 0xFF, (size_t)M * 4, s));
    HELIO_CK(cudaMemsetAsync(b->totals.ptr, 0, kVals * 8 + 8, s));
    if (S) first_ref_kernel<<<grid_for(S, kThreads), kThreads, 0, s>>>(*in, b->first_ref.as<uint32_t>(), error);
    HELIO_CK(cudaGetLastError());
    if (S) {
        block_sums_kernel<<<blocks, kThreads, 0, s>>>(*in, b->first_ref.as<uint32_t>(), b->block_tot.as<uint64_t>());
        HELIO_CK(cudaGetLastError());
        scan_blocks_kernel<<<1, kThreads, 0, s>>>(b->block_tot.as<uint64_t>(), blocks, b->block_base.as<uint64_t>(),
                                                  b->totals.as<uint64_t>());
        HELIO_CK(cudaGetLastError());
    }
    uint64_t tot[kVals + 1] = {0};
    HELIO_CK(cudaMemcpyAsync(tot, b->totals.ptr, sizeof(tot), cudaMemcpyDeviceToHost, s));
    HELIO_CK(cudaStreamSynchronize(s));
    uint32_t err = 0;
    std::memcpy(&err, &tot[kVals], 4);
    HELIO_ARG(!(err & kErrPool), "a mesh's descriptor range leaves the pool");
    HELIO_ARG(tot[1] <= 0xFFFFFFFFull, "virtual geometry exceeds the u32 descriptor address space");
    HELIO_ARG(tot[2] <= 0xFFFFFFFFull, "virtual geometry exceeds the u32 work-item address space");
    HELIO_ARG(tot[4] <= 0xFFFFFFFFull, "virtual geometry indirect draw capacity exceeds u32");
    const uint64_t objects = tot[0], descriptors = tot[1], items = tot[2], used_meshes = tot[3];
    HELIO_CK(b->meshlets.ensure(descriptors * sizeof(HelioGpuMeshletEntry)));
    HELIO_CK(b->objects.ensure(objects * sizeof(HelioGpuVgObject)));
    HELIO_CK(b->instances.ensure(objects * sizeof(HelioGpuInstanceData)));
    HELIO_CK(b->items.ensure(items * sizeof(HelioGpuVgWorkItem)));
    BuildOut o{b->meshlets.as<HelioGpuMeshletEntry>(), b->objects.as<HelioGpuVgObject>(),
               b->instances.as<HelioGpuInstanceData>(), b->items.as<HelioGpuVgWorkItem>(),
               b->obj_of_slot.as<uint32_t>(), b->mesh_base.as<uint32_t>(), b->mesh_order.as<uint32_t>()};
    if (S) {
        place_kernel<<<blocks, kThreads, 0, s>>>(*in, b->first_ref.as<uint32_t>(), b->block_base.as<uint64_t>(), o);
        HELIO_CK(cudaGetLastError());
        objects_kernel<<<grid_for(S, kThreads), kThreads, 0, s>>>(*in, o, error);
        HELIO_CK(cudaGetLastError());
    }
    if (used_meshes) {
        copy_descriptors_kernel<<<grid_for(used_meshes * 32u, kThreads), kThreads, 0, s>>>(*in, o,
                                                                                          (uint32_t)used_meshes);
        HELIO_CK(cudaGetLastError());
    }
    HELIO_CK(cudaMemcpyAsync(&err, error, 4, cudaMemcpyDeviceToHost, s));
    HELIO_CK(cudaStreamSynchronize(s));
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
