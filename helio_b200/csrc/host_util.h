// host_util.h — host-side helpers shared by the C-ABI implementation files.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/helio_cull.h"

// Formats `fmt` into the calling thread's helio_last_error() and returns `code`.
int32_t helio_fail(int32_t code, const char* fmt, ...);

#define HELIO_CK(call)                                                                                 \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return helio_fail(HELIO_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

#define HELIO_ARG(cond, msg)                                            \
    do {                                                                \
        if (!(cond)) return helio_fail(HELIO_ERR_INVALID_ARG, "%s", msg); \
    } while (0)

namespace helio {

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Owned device allocation with grow-only semantics.
// Bytes to hold for `need` when `held` bytes are allocated: a buffer that must grow takes at
// least 1.5x what it held, so that a buffer which keeps growing (a server's batches of
// changing shapes) is reallocated a logarithmic number of times (cudaFree synchronises the
// whole device). A first allocation takes exactly `need`.
inline size_t grow_capacity(size_t need, size_t held) {
    if (need <= held) return held;
    if (held == 0) return need;
    const size_t g = held + held / 2;
    return need > g ? need : g;
}

struct DevBuf {
    void* ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    cudaError_t ensure(size_t need) {
        if (need <= bytes && ptr) return cudaSuccess;
        if (need == 0) need = 16;
        const size_t cap = grow_capacity(need, ptr ? bytes : 0);
        release();
        cudaError_t e = cudaMalloc(&ptr, cap);
        if (e == cudaSuccess) bytes = cap;
        return e;
    }
    template <typename T>
    T* as() const {
        return reinterpret_cast<T*>(ptr);
    }
};

inline uint32_t host_mip_levels(uint32_t w, uint32_t h) {
    uint32_t m = w > h ? w : h, bits = 0;
    while (m) {
        ++bits;
        m >>= 1;
    }
    return bits ? bits : 1u;
}

}  // namespace helio
