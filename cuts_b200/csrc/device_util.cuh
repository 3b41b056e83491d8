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
    // per vertex: entries of its out- (in-) list below the vertex itself
    // (may be null: the lists are searched instead)
    const uint32_t *bwd_out;
    const uint32_t *bwd_in;
    // dense core of a symmetric graph: the kCore vertices of highest id
    // (the hubs, ids being degree ranks), from core0 up; row d - core0 of
    // core_bits (kCore / 32 words) has bit u - core0 set when d lists u.
    // Null when absent.
    const uint32_t *core_bits;
    uint32_t core0;
};

constexpr uint32_t kCore = 1024;  // vertices in the dense core

// The kernels' view of a resident graph (a DeviceGraph).
template <class G>
inline DevView graph_view(const G &g) {
    return DevView{g.out_info, g.in_info, g.adj, g.n, g.bwd_out, g.bwd_in, g.core_bits, g.core0};
}

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

// Lower bound of x in the list of vertex u (direction in_dir), where the
// list's window often starts or ends at u itself (x == u + 1 or x == u, the
// ordering conditions of symmetry breaking on degree-ranked ids): those two
// are read from the per-vertex count of entries below u instead of searched.
// `loops`: the graph has self-loops, so u may list itself.
__device__ __forceinline__ uint32_t lbound_own(const DevView &g, bool in_dir, uint32_t u,
                                               const uint32_t *__restrict__ list, uint32_t len, uint32_t x,
                                               bool loops) {
    const uint32_t *bw = in_dir ? g.bwd_in : g.bwd_out;
    if (bw && (x == u || x == u + 1)) {
        uint32_t b = __ldg(bw + u);
        if (x == u + 1 && loops && b < len && __ldg(list + b) == u) ++b;
        return b;
    }
    return lbound(list, len, x);
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
