// batch.hpp -- batched counting of many queries in one persistent launch.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "engine.hpp"

namespace cuts {

constexpr int kBatchMaxK = 10;  // query vertices handled inside the batched kernel
constexpr int kBatchMaxJ = 8;   // joined lists per level inside the batched kernel

// One level of a batched query (a compact LevelPlan).
struct BLevel {
    uint32_t nj, qin, qout, check_sig, gt_mask, lt_mask, closed_form, fold, guar_mask, pad[3];
    uint8_t jpos[kBatchMaxJ];
    uint8_t jdir[kBatchMaxJ];
};

struct BQuery {
    BLevel lv[kBatchMaxK];
    uint32_t k;
    uint32_t type;      // level-1 candidate list: 0 out, 1 in, 2 the shorter
    uint32_t root_cnt;  // roots = the first root_cnt vertices in out-degree order
    uint32_t pad;
};

// Launch shape picked by the autotuner (0 = default).
struct BatchTuning {
    uint32_t grain = 64;          // level-1 candidates per task
    uint32_t tasks_per_grab = 1;  // tasks taken per work-counter atomic
    uint32_t blocks_per_sm = 0;   // cap on resident blocks per SM (0 = occupancy)
};

// Per-graph structures shared by every batch: vertices in out-degree order and
// prefix sums of per-root task counts for each list type.
int batch_prepare_graph(DeviceGraph &g, uint32_t grain);

struct Batch {
    DeviceGraph *g = nullptr;
    uint32_t flags = 0;
    BatchTuning tune;
    std::vector<const Query *> queries;
    uint32_t nq = 0;                 // all queries
    uint32_t nb = 0;                 // queries in the launch
    std::vector<uint32_t> index;     // launch slot -> query
    std::vector<int> eligible;       // 1 in the launch, 2 no root, 0 level engine
    bool route_level = true;         // fused / orbit-folded queries of 4+ vertices to the level engine
    bool route_all = false;          // every query of 4+ vertices to the level engine
    std::vector<uint64_t> aut;       // count multiplier per query
    std::vector<unsigned long long> qbase_host;
    unsigned long long total_tasks = 0;
    BQuery *d_queries = nullptr;
    unsigned long long *d_qbase = nullptr, *d_counts = nullptr, *d_ctr = nullptr;
    uint32_t *d_aborted = nullptr;
    unsigned long long *d_qtime = nullptr;  // warp-ns spent per query (per-query limit)
    double query_budget_ms = 0;             // per-query limit in whole-GPU ms (0 = none)
    unsigned long long *h_counts = nullptr, *h_ctr = nullptr;
    uint32_t *h_aborted = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long captured_budget = ~0ull;
    double captured_query_budget = -1;
    uint32_t shard = 0, nshards = 1;  // tasks t with t % nshards == shard (one GPU of several)
    uint32_t captured_shard = 0, captured_nshards = 0;
    uint32_t launch_blocks = 0;

    int create(DeviceGraph &g, const std::vector<const Query *> &qs, uint32_t flags,
               const BatchTuning &tune);
    // budget_ms > 0 stops the launch after that much device time; queries not
    // finished report CUTS_ERR_BUDGET.
    int run(double budget_ms, std::vector<uint64_t> &counts, std::vector<int> &status, float *ms);
    // Each query may use query_budget_ms of the whole GPU (its warp time,
    // summed over the launch's warps, up to query_budget_ms x warps); a query
    // past it reports CUTS_ERR_BUDGET and the others carry on.  0 = no limit.
    void set_query_budget(double ms) { query_budget_ms = ms; }
    // This launch takes only the tasks t with t % nshards == shard, so
    // nshards launches (one per GPU) partition every query's count.
    void set_shard(uint32_t s, uint32_t n) { shard = s; nshards = n; }
    void destroy();

  private:
    int capture(unsigned long long budget_ns);
};

// The allocation-free count (cuts_count_noalloc): graph and counts in the
// caller's device memory, engine scratch in a fixed device array.
int count_noalloc(const uint32_t *info_out, const uint32_t *info_in, const uint32_t *adj, uint32_t n,
                  int symmetric, const Query *const *qs, uint32_t nq, uint32_t flags,
                  unsigned long long *counts, cudaStream_t stream);

}  // namespace cuts
