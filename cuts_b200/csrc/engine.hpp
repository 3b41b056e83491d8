// engine.hpp -- device-resident data graph and the counting driver.
#pragma once
#include <cuda_runtime.h>

#include "host.hpp"
#include "order_search.hpp"

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
    bool loops = false;  // some vertex lists itself (a self-loop arc)
    uint2 *out_info = nullptr;
    uint2 *in_info = nullptr;
    uint32_t *adj = nullptr;
    uint64_t adj_words = 0;
    // per vertex: entries of its out- (in-) list below itself; bwd_in
    // aliases bwd_out for a symmetric graph
    uint32_t *bwd_out = nullptr;
    uint32_t *bwd_in = nullptr;
    // adjacency bitmap of the highest-id vertices (symmetric graphs): row
    // d - core0, bit u - core0 (kCore x kCore bits)
    uint32_t *core_bits = nullptr;
    uint32_t core0 = 0;
    cudaStream_t stream = nullptr;

    // trie-level arena, carved per query
    void *arena = nullptr;
    size_t arena_bytes = 0;
    size_t arena_default = 0;
    uint64_t level_cap_req = 0;   // 0 = automatic
    uint32_t fuse_split = 0;      // fused count: |S| above which a parent is split (0 = default)

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
    DegreeStats stats;                     // degree tails, for order features
    std::vector<uint32_t> h_out_deg, h_in_deg;  // by device id
    std::vector<uint32_t> orig;            // device id -> host vertex (empty: the same)

    // batched engine: vertices in out-degree order and task prefix sums
    uint32_t *batch_vsorted = nullptr;
    unsigned long long *batch_pref = nullptr;
    std::vector<unsigned long long> batch_pref_host;
    uint32_t batch_grain = 0;
};

int device_graph_upload(const HostGraph &g, int device, DeviceGraph **out);
// The same from CSR arrays in host memory (validated and checked for
// symmetry on the device; in-lists may be null for a symmetric graph).
int device_graph_from_csr(uint32_t n, const uint64_t *out_off, const uint32_t *out_adj, const uint64_t *in_off,
                          const uint32_t *in_adj, int device, DeviceGraph **out);
// Builds g's device layout (layout.cu): sym_hint 1 symmetric, 0 directed
// (in-lists given), -1 decide; validate checks offsets and list order.
int device_layout(uint32_t n, const uint64_t *out_off, const uint32_t *out_adj, const uint64_t *in_off,
                  const uint32_t *in_adj, int sym_hint, bool validate, DeviceGraph &g);
void device_graph_free(DeviceGraph *g);

struct CountResult {
    uint64_t count = 0;
    float ms = 0.f;
    uint64_t level_sizes[kMaxK] = {};
    uint64_t launches = 0;
    uint64_t chunks = 0;
    uint64_t last_level_bytes = 0;
    // per-kernel device time when profiling (CUDA events around each launch)
    double last_level_ms = 0, expand_ms = 0;
    uint64_t last_level_launches = 0, expand_launches = 0;
};

// Run options beyond the query.
struct CountOptions {
    uint32_t chunks = 1;      // root slices (the reference's trunks)
    uint32_t flags = 0;       // CUTS_FLAG_*
    uint32_t shard = 0;       // roots u with u % nshards == shard
    uint32_t nshards = 1;
    bool want_bytes = false;  // untimed pass for the last-level traffic model
    bool profile = false;     // event pairs around every level launch
    double budget_ms = 0;     // > 0: stop launching chunks after this much time
};

// Counts embeddings of q (order already set) in g.  chunks >= 1 slices the
// root level like the reference's trunks.  want_bytes adds an untimed pass
// computing the last-level kernel's algorithmic traffic.
int device_count(DeviceGraph &g, const Query &q, const CountOptions &opt, CountResult &res);

// Enumerates every embedding and writes ans.txt lines (util.cpp:53-74).
// shard / nshards: only the roots u with u % nshards == shard (device ids).
int device_dump(DeviceGraph &g, const Query &q, const char *path, uint64_t *lines, uint32_t shard = 0,
                uint32_t nshards = 1);

}  // namespace cuts
