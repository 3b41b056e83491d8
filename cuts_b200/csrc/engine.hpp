// engine.hpp -- device-resident data graph and the counting driver.
#pragma once
#include <cuda_runtime.h>

#include "host.hpp"

namespace cuts {

// Data graph in HBM.  Each adjacency list starts on a 16-byte boundary
// (offsets are multiples of 4 words) and is padded with 0xFFFFFFFF up to the
// next boundary, so lists can be staged with 128-bit loads.  info[v] =
// {word offset, length}; for a symmetric graph in_info aliases out_info.
struct DeviceGraph {
    int device = 0;
    uint32_t n = 0;
    uint64_t arcs = 0;
    bool symmetric = false;
    uint32_t max_deg = 0;
    uint2 *out_info = nullptr;
    uint2 *in_info = nullptr;
    uint32_t *adj = nullptr;
    uint64_t adj_words = 0;
    cudaStream_t stream = nullptr;

    // trie-level arena, carved per query
    void *arena = nullptr;
    size_t arena_bytes = 0;
    uint64_t level_cap_req = 0;   // 0 = automatic

    // small device scratch and pinned host mirrors
    uint32_t *d_u32 = nullptr;             // counters / cursors / flags
    unsigned long long *d_u64 = nullptr;   // count accumulators
    void *d_plan = nullptr;                // Plan
    uint64_t *d_tiles = nullptr;           // planner tile sums
    uint32_t *d_bounds = nullptr;          // planner chunk boundaries
    size_t tiles_cap = 0;
    uint32_t *h_u32 = nullptr;             // pinned
    unsigned long long *h_u64 = nullptr;   // pinned
    void *h_plan = nullptr;                // pinned
    uint32_t *h_bounds = nullptr;          // pinned
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

int device_graph_upload(const HostGraph &g, int device, DeviceGraph **out);
void device_graph_free(DeviceGraph *g);

struct CountResult {
    uint64_t count = 0;
    float ms = 0.f;
    uint64_t level_sizes[kMaxK] = {};
    uint64_t launches = 0;
    uint64_t chunks = 0;
    uint64_t last_level_bytes = 0;
};

// Counts embeddings of q (order already set) in g.  chunks >= 1 slices the
// root level like the reference's trunks.  want_bytes adds an untimed pass
// computing the last-level kernel's algorithmic traffic.
int device_count(DeviceGraph &g, const Query &q, uint32_t chunks, uint32_t flags,
                 bool want_bytes, CountResult &res);

// Enumerates every embedding and writes ans.txt lines (util.cpp:53-74).
int device_dump(DeviceGraph &g, const Query &q, const char *path, uint64_t *lines);

}  // namespace cuts
