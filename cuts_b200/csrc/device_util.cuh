// device_util.cuh -- device-side helpers shared by the level kernels and the
// batched engine.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cuts {

constexpr uint32_t kFullMask = 0xffffffffu;

// Kernel view of the resident data graph (see DeviceGraph).
struct DevView {
    const uint2 *out_info;
    const uint2 *in_info;
    const uint32_t *adj;
    uint32_t n;
};


__device__ __forceinline__ uint32_t lbound(const uint32_t *__restrict__ a, uint32_t len,
                                           uint32_t x) {
    uint32_t lo = 0;
    while (len > 0) {
        uint32_t half = len >> 1;
        if (__ldg(a + lo + half) < x) { lo += half + 1; len -= half + 1; }
        else len = half;
    }
    return lo;
}

__device__ __forceinline__ bool contains(const uint32_t *__restrict__ a, uint32_t len, uint32_t x) {
    uint32_t p = lbound(a, len, x);
    return p < len && __ldg(a + p) == x;
}

// Lower bound of x in a[from, len), searching forward from a position known
// to be <= the answer: exponential steps, then a binary search in the last
// step's interval (galloping; Bentley & Yao 1976).
__device__ __forceinline__ uint32_t lbound_from(const uint32_t *__restrict__ a, uint32_t len,
                                                uint32_t from, uint32_t x) {
    if (from >= len || __ldg(a + from) >= x) return from;
    uint32_t lo = from + 1, step = 1;
    while (lo + step <= len && __ldg(a + lo + step - 1) < x) {
        lo += step;
        step <<= 1;
    }
    uint32_t n = min(step, len - lo);
    while (n > 0) {
        const uint32_t half = n >> 1;
        if (__ldg(a + lo + half) < x) { lo += half + 1; n -= half + 1; }
        else n = half;
    }
    return lo;
}

__device__ __forceinline__ uint32_t warp_min(uint32_t v) {
    #pragma unroll
    for (int s = 16; s; s >>= 1) v = min(v, __shfl_xor_sync(kFullMask, v, s));
    return v;
}


// %globaltimer: nanoseconds, comparable across the SMs of one GPU.
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

}  // namespace cuts
