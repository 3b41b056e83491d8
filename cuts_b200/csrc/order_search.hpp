// order_search.hpp -- learned matching order (features, search, fallback).
#pragma once
#include <cstdint>
#include <vector>

#include "host.hpp"

namespace cuts {

struct Mlp;

constexpr int kFeatures = 16;

// Degree tails of the data graph: *_ge[d] = vertices with degree >= d.
struct DegreeStats {
    uint64_t n = 0;
    std::vector<uint64_t> out_ge, in_ge;
};
DegreeStats degree_stats(const HostGraph &g);

// Features of order position i given the prefix order[0..i] and
// parent_log = log(1 + |L_{i-1}|).
void step_features(const Query &q, const DegreeStats &ds, const uint32_t *order, uint32_t i,
                   float parent_log, float *f);

// Relative cost per parent of a closed-form last level (counted, not scanned).
constexpr double kClosedFormCost = 0.1;

// sum_{i<k-1} (exp(pred_i) - 1) * cost of level i+1 per parent: 1 + its
// joined lists, or kClosedFormCost for a closed-form last level
double predicted_work(const Query &q, const uint32_t *order, const float *pred);

struct OrderSearchOptions {
    size_t beam = 0;      // 0 = exhaustive
    double margin = 1.25; // learned order must promise this much less work
    size_t top = 0;       // also return this many complete orders, least predicted work first
};

struct OrderChoice {
    std::vector<uint32_t> order, score_order;
    std::vector<float> pred, score_pred;
    double best_work = 0, score_work = 0;
    size_t candidates = 0;
    bool used_learned = false;
    std::vector<std::vector<uint32_t>> top;  // opt.top best complete orders
    std::vector<double> top_work;
};

int learned_order(const Query &q, const DegreeStats &ds, Mlp &mlp, const OrderSearchOptions &opt,
                  OrderChoice &out);

}  // namespace cuts
