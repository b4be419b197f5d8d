// tma.cuh — Tensor Memory Accelerator (TMA) tile loads into shared memory, completed
// on an mbarrier, for sm_100a (PTX ISA: cp.async.bulk.tensor, mbarrier).
//
// Only plain tiled loads of this GPU's own global memory are used: no cluster
// multicast form of any load appears in this library.
#pragma once

#include <cuda.h>  // CUtensorMap (the 128-byte opaque descriptor)
#include <stdint.h>

namespace helio {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Initialises an mbarrier for `count` arrivals (one thread), then makes the
// initialisation visible to the async proxy that completes the transactions.
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also announces `bytes` of transactions still to land.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// True once the phase with parity `parity` has completed (one bounded hardware wait).
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}

// Waits for the phase, giving up after `limit` polls (returns false then).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if (i >= 16) __nanosleep(64);
    }
    return false;
}

// 2-D tiled load of the box at element coordinates (x, y) of `map` into shared
// memory at `dst` (128-byte aligned), completing `bytes` of transactions on `bar`.
// x * element size must be a multiple of 16 bytes; y may be anything (rows outside
// the tensor are filled with zeros).
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int32_t x, int32_t y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// Brings a descriptor that lives in global memory (written by the host before the
// launch) into the tensormap proxy's view; once per CTA before its first use.
__device__ __forceinline__ void tma_descriptor_acquire(const CUtensorMap* map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(reinterpret_cast<uint64_t>(map))
                 : "memory");
}

}  // namespace helio
