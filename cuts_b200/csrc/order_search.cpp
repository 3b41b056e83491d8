// order_search.cpp -- learned matching order: per-step features, the
// order search over connected-prefix orders, and the score-order fallback.
//
// The reference picks one order greedily (graph.cpp:62-93).  Here every
// connected-prefix order is a candidate (beam search above 8 query
// vertices); the MLP predicts log(1 + |L_i|) step by step, feeding its own
// prediction of the parent level back as a feature, and the predicted work
//     W(order) = sum_{i < k-1} exp(pred_i) * (1 + joins at level i+1)
// ranks the candidates.  The score order stays the fallback: it is used
// when no model is given, and kept unless the best candidate's predicted
// work is at least `margin` times smaller.  Order never changes the count.
#include <algorithm>
#include <cmath>
#include <numeric>

#include "mlp.hpp"
#include "order_search.hpp"

namespace cuts {

DegreeStats degree_stats(const HostGraph &g) {
    DegreeStats s;
    s.n = g.n;
    const uint32_t md = g.max_degree();
    s.out_ge.assign(size_t(md) + 2, 0);
    s.in_ge.assign(size_t(md) + 2, 0);
    for (uint32_t v = 0; v < g.n; ++v) {
        s.out_ge[g.out_deg(v)]++;
        s.in_ge[g.in_deg(v)]++;
    }
    for (int64_t d = int64_t(md); d >= 0; --d) {
        s.out_ge[d] += s.out_ge[d + 1];
        s.in_ge[d] += s.in_ge[d + 1];
    }
    return s;
}

static double frac_ge(const std::vector<uint64_t> &ge, uint64_t n, uint32_t d) {
    if (n == 0) return 0.0;
    if (d >= ge.size()) return 0.0;
    return double(ge[d]) / double(n);
}

static float logf20(double x) { return float(std::log(std::max(x, 1e-12)) / 20.0); }

// Undirected neighbour masks and degrees of the query (self-loops excluded).
struct QMasks {
    uint32_t nb[kMaxK];
    uint32_t deg[kMaxK];
};
static QMasks masks_of(const Query &q) {
    QMasks m{};
    for (uint32_t v = 0; v < q.k; ++v) {
        for (uint32_t w : q.out[v]) if (w != v) m.nb[v] |= 1u << w;
        for (uint32_t w : q.in[v]) if (w != v) m.nb[v] |= 1u << w;
    }
    for (uint32_t v = 0; v < q.k; ++v) m.deg[v] = uint32_t(__builtin_popcount(m.nb[v]));
    return m;
}

static void features_masked(const Query &q, const QMasks &M, const DegreeStats &ds,
                            const uint32_t *order, uint32_t i, float parent_log, float *f) {
    const uint32_t v = order[i];
    std::fill(f, f + kFeatures, 0.f);
    uint32_t prefix = 0;
    for (uint32_t j = 0; j < i; ++j) prefix |= 1u << order[j];
    const uint32_t joined = M.nb[v] & prefix;
    const uint32_t nj = uint32_t(__builtin_popcount(joined));
    uint32_t minjdeg = 1000;
    for (uint32_t msk = joined; msk; msk &= msk - 1) minjdeg = std::min(minjdeg, M.deg[__builtin_ctz(msk)]);
    uint32_t inner = 0;  // undirected query edges within positions 0..i
    const uint32_t upto = prefix | (1u << v);
    for (uint32_t msk = upto; msk; msk &= msk - 1)
        inner += uint32_t(__builtin_popcount(M.nb[__builtin_ctz(msk)] & upto));
    inner /= 2;
    const double surv = std::min(frac_ge(ds.out_ge, ds.n, uint32_t(q.out[v].size())),
                                 frac_ge(ds.in_ge, ds.n, uint32_t(q.in[v].size())));
    f[0] = M.deg[v] / 8.f;
    f[1] = nj / 4.f;
    f[2] = i / 8.f;
    f[3] = q.k / 8.f;
    f[4] = parent_log / 20.f;
    f[5] = i == 0 ? 1.f : 0.f;
    f[6] = logf20(surv);
    f[7] = inner / 16.f;
    f[8] = (nj ? minjdeg : 0) / 8.f;
    f[9] = float(std::log1p(double(ds.n)) / 20.0);
    for (int b = 1; b <= 6; ++b) f[9 + b] = logf20(frac_ge(ds.out_ge, ds.n, 1u << (2 * b)));
}

// Features of position i of `order` (prefix order[0..i]); parent_log =
// log(1 + |L_{i-1}|) (true sizes when training, predictions when searching).
void step_features(const Query &q, const DegreeStats &ds, const uint32_t *order, uint32_t i,
                   float parent_log, float *f) {
    features_masked(q, masks_of(q), ds, order, i, parent_log, f);
}

static uint32_t joins_at(const Query &q, const uint32_t *order, uint32_t i) {
    uint32_t nj = 0;
    const uint32_t v = order[i];
    for (uint32_t j = 0; j < i; ++j)
        nj += (q.has_arc(v, order[j]) || q.has_arc(order[j], v)) ? 1 : 0;
    return nj;
}

// Work of level i+1 per entry of L_i: one probe sequence per joined list,
// except a last level with a single joined list and no self-loop, which the
// engine counts by list arithmetic (and folds into the level before).
static double level_cost(const Query &q, const uint32_t *order, uint32_t i) {
    const uint32_t nj = joins_at(q, order, i + 1);
    if (i + 2 == q.k && nj == 1 && !q.self_loop(order[i + 1])) return kClosedFormCost;
    return 1.0 + nj;
}

double predicted_work(const Query &q, const uint32_t *order, const float *pred) {
    double w = 0;
    for (uint32_t i = 0; i + 1 < q.k; ++i)
        w += std::expm1(double(std::max(pred[i], 0.f))) * level_cost(q, order, i);
    return w;
}

namespace {
struct Cand {
    std::vector<uint32_t> order;  // prefix
    std::vector<float> pred;      // predicted log sizes so far
    uint32_t used = 0;            // bitmask of placed vertices
};
}  // namespace

int learned_order(const Query &q, const DegreeStats &ds, Mlp &mlp, const OrderSearchOptions &opt,
                  OrderChoice &out) {
    const uint32_t k = q.k;
    out = OrderChoice();
    std::vector<uint32_t> score;
    int rc = score_order(q, score);
    if (rc) return rc;
    out.score_order = score;
    out.order = score;
    if (k <= 2) return CUTS_OK;
    const size_t beam = opt.beam ? opt.beam : 100000;
    const QMasks M = masks_of(q);
    std::vector<Cand> cur;
    for (uint32_t v = 0; v < k; ++v) {
        Cand c;
        c.order = {v};
        c.used = 1u << v;
        cur.push_back(c);
    }
    // the score order is always evaluated, whatever the beam keeps
    Cand score_c;
    bool track_score = true;
    std::vector<float> feats;
    for (uint32_t i = 0; i < k; ++i) {
        // predict step i for every candidate (and the score order's prefix)
        std::vector<Cand *> rows;
        for (auto &c : cur) rows.push_back(&c);
        Cand sc;
        if (track_score) {
            sc.order.assign(score.begin(), score.begin() + i + 1);
            sc.pred = score_c.pred;
            rows.push_back(&sc);
        }
        feats.assign(rows.size() * kFeatures, 0.f);
        for (size_t r = 0; r < rows.size(); ++r) {
            const float parent = i ? rows[r]->pred[i - 1] : 0.f;
            features_masked(q, M, ds, rows[r]->order.data(), i, parent, &feats[r * kFeatures]);
        }
        std::vector<float> y(rows.size());
        rc = mlp.predict(feats.data(), int(rows.size()), y.data());
        if (rc) return rc;
        for (size_t r = 0; r < rows.size(); ++r) rows[r]->pred.push_back(std::max(y[r], 0.f));
        if (track_score) score_c = sc;
        if (i + 1 == k) break;
        // extend by every vertex joined to the prefix
        std::vector<Cand> next;
        for (auto &c : cur) {
            for (uint32_t v = 0; v < k; ++v) {
                if (c.used >> v & 1) continue;
                if (!(M.nb[v] & c.used)) continue;
                Cand n2 = c;
                n2.order.push_back(v);
                n2.used |= 1u << v;
                next.push_back(std::move(n2));
            }
        }
        if (next.size() > beam) {
            // keep the prefixes with the least predicted work so far
            std::vector<std::pair<double, size_t>> key(next.size());
            for (size_t r = 0; r < next.size(); ++r) {
                double w = 0;
                for (float p : next[r].pred) w += std::expm1(double(p));
                key[r] = {w, r};
            }
            std::nth_element(key.begin(), key.begin() + beam, key.end());
            std::vector<Cand> kept;
            for (size_t r = 0; r < beam; ++r) kept.push_back(std::move(next[key[r].second]));
            next.swap(kept);
        }
        cur.swap(next);
    }
    out.candidates = cur.size();
    out.score_work = predicted_work(q, score_c.order.data(), score_c.pred.data());
    out.score_pred = score_c.pred;
    size_t best = 0;
    double bw = 1e300;
    for (size_t r = 0; r < cur.size(); ++r) {
        if (cur[r].order.size() != k) continue;
        const double w = predicted_work(q, cur[r].order.data(), cur[r].pred.data());
        if (w < bw) { bw = w; best = r; }
    }
    out.best_work = bw;
    if (opt.top) {
        std::vector<std::pair<double, size_t>> key;
        for (size_t r = 0; r < cur.size(); ++r)
            if (cur[r].order.size() == k)
                key.push_back({predicted_work(q, cur[r].order.data(), cur[r].pred.data()), r});
        std::sort(key.begin(), key.end());
        for (size_t r = 0; r < key.size() && r < opt.top; ++r) {
            out.top.push_back(cur[key[r].second].order);
            out.top_work.push_back(key[r].first);
        }
    }
    if (!cur.empty() && bw * opt.margin < out.score_work) {
        out.order = cur[best].order;
        out.pred = cur[best].pred;
        out.used_learned = true;
    } else {
        out.pred = score_c.pred;
    }
    return CUTS_OK;
}

}  // namespace cuts
