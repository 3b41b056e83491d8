// capi.cpp -- the extern "C" surface declared in include/cuts_b200.h.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <memory>
#include <cmath>
#include <new>

#include "batch.hpp"
#include "engine.hpp"
#include "host.hpp"
#include "mlp.hpp"
#include "order_search.hpp"

struct cuts_graph_s {
    cuts::DeviceGraph *dev = nullptr;
};
struct cuts_query_s {
    cuts::Query q;
};
struct cuts_hgraph_s {
    cuts::HostGraph g;
};
struct cuts_batch_s {
    cuts::Batch b;
    ~cuts_batch_s() { b.destroy(); }
};
struct cuts_mlp_s {
    cuts::Mlp m;
    ~cuts_mlp_s() { m.destroy(); }
};

using namespace cuts;

#define GUARD(expr)                                                     \
    try {                                                               \
        return (expr);                                                  \
    } catch (const std::bad_alloc &) {                                  \
        return set_error(CUTS_ERR_NOMEM, "host allocation failed");     \
    } catch (const std::exception &ex) {                                \
        return set_error(CUTS_ERR_ARG, ex.what());                      \
    }

extern "C" {

const char *cuts_last_error(void) { return last_error(); }
const char *cuts_version(void) { return "cuts_b200 0.1"; }

// ---- host graph ---------------------------------------------------------

int cuts_hgraph_load(const char *path, cuts_hgraph *out) {
    if (!path || !out) return set_error(CUTS_ERR_ARG, "null argument");
    *out = nullptr;
    GUARD(([&]() {
        auto h = std::make_unique<cuts_hgraph_s>();
        int rc = load_graph_text(path, h->g);
        if (rc) return rc;
        *out = h.release();
        return CUTS_OK;
    })());
}

int cuts_hgraph_gen_er(uint32_t n, double p, uint64_t seed, cuts_hgraph *out) {
    if (!out || p < 0 || p > 1) return set_error(CUTS_ERR_ARG, "bad argument");
    *out = nullptr;
    GUARD(([&]() {
        auto h = std::make_unique<cuts_hgraph_s>();
        gen_erdos_renyi(n, p, seed, h->g);
        *out = h.release();
        return CUTS_OK;
    })());
}

int cuts_hgraph_gen_chung_lu(uint32_t n, uint64_t m, double gamma, double wmin, double cap,
                             uint64_t seed, cuts_hgraph *out) {
    if (!out) return set_error(CUTS_ERR_ARG, "null argument");
    *out = nullptr;
    GUARD(([&]() {
        auto h = std::make_unique<cuts_hgraph_s>();
        int rc = gen_chung_lu(n, m, gamma, wmin, cap, seed, h->g);
        if (rc) return rc;
        *out = h.release();
        return CUTS_OK;
    })());
}

int cuts_hgraph_info(cuts_hgraph h, uint32_t *n, uint64_t *arcs, int *symmetric,
                     uint32_t *max_degree) {
    if (!h) return set_error(CUTS_ERR_ARG, "null graph");
    if (n) *n = h->g.n;
    if (arcs) *arcs = h->g.arcs;
    if (symmetric) *symmetric = h->g.symmetric;
    if (max_degree) *max_degree = h->g.max_degree();
    return CUTS_OK;
}

int cuts_hgraph_csr(cuts_hgraph h, uint64_t *out_off, uint32_t *out_adj, uint64_t *in_off,
                    uint32_t *in_adj) {
    if (!h) return set_error(CUTS_ERR_ARG, "null graph");
    const HostGraph &g = h->g;
    if (out_off) std::memcpy(out_off, g.out_off.data(), sizeof(uint64_t) * (size_t(g.n) + 1));
    if (out_adj && g.arcs) std::memcpy(out_adj, g.out_adj.data(), sizeof(uint32_t) * g.arcs);
    if (!g.symmetric) {
        if (in_off) std::memcpy(in_off, g.in_off.data(), sizeof(uint64_t) * (size_t(g.n) + 1));
        if (in_adj && g.arcs) std::memcpy(in_adj, g.in_adj.data(), sizeof(uint32_t) * g.arcs);
    }
    return CUTS_OK;
}

int cuts_hgraph_write(cuts_hgraph h, const char *path) {
    if (!h || !path) return set_error(CUTS_ERR_ARG, "null argument");
    GUARD(write_graph_text(path, h->g));
}

int cuts_hgraph_save_binary(cuts_hgraph h, const char *path) {
    if (!h || !path) return set_error(CUTS_ERR_ARG, "null argument");
    GUARD(save_graph_binary(path, h->g));
}

int cuts_hgraph_load_binary(const char *path, cuts_hgraph *out) {
    if (!path || !out) return set_error(CUTS_ERR_ARG, "null argument");
    *out = nullptr;
    GUARD(([&]() {
        auto h = std::make_unique<cuts_hgraph_s>();
        int rc = load_graph_binary(path, h->g);
        if (rc) return rc;
        *out = h.release();
        return CUTS_OK;
    })());
}

int cuts_graph_upload(cuts_hgraph h, int device, cuts_graph *out) {
    if (!h || !out) return set_error(CUTS_ERR_ARG, "null argument");
    *out = nullptr;
    GUARD(([&]() {
        auto gh = std::make_unique<cuts_graph_s>();
        int rc = device_graph_upload(h->g, device, &gh->dev);
        if (rc) return rc;
        *out = gh.release();
        return CUTS_OK;
    })());
}

void cuts_hgraph_free(cuts_hgraph h) { delete h; }

int cuts_gen_random_query(uint32_t k, double p, uint64_t seed, uint32_t *narcs, uint32_t *src,
                          uint32_t *dst) {
    if (!narcs || !src || !dst || k == 0 || k > CUTS_MAX_QUERY)
        return set_error(CUTS_ERR_ARG, "bad argument");
    GUARD(([&]() {
        std::vector<uint32_t> s, d;
        gen_random_query(k, p, seed, s, d);
        *narcs = uint32_t(s.size());
        std::copy(s.begin(), s.end(), src);
        std::copy(d.begin(), d.end(), dst);
        return CUTS_OK;
    })());
}

// ---- device graph ---------------------------------------------------------

int cuts_graph_load(const char *path, int device, cuts_graph *out) {
    if (!path || !out) return set_error(CUTS_ERR_ARG, "null argument");
    *out = nullptr;
    GUARD(([&]() {
        HostGraph g;
        int rc = load_graph_text(path, g);
        if (rc) return rc;
        auto gh = std::make_unique<cuts_graph_s>();
        rc = device_graph_upload(g, device, &gh->dev);
        if (rc) return rc;
        *out = gh.release();
        return CUTS_OK;
    })());
}

int cuts_graph_from_csr(uint32_t n, const uint64_t *out_off, const uint32_t *out_adj,
                        const uint64_t *in_off, const uint32_t *in_adj, int device,
                        cuts_graph *out) {
    if (!out) return set_error(CUTS_ERR_ARG, "null argument");
    *out = nullptr;
    GUARD(([&]() {
        auto gh = std::make_unique<cuts_graph_s>();
        int rc = device_graph_from_csr(n, out_off, out_adj, in_off, in_adj, device, &gh->dev);
        if (rc) return rc;
        *out = gh.release();
        return CUTS_OK;
    })());
}

int cuts_graph_info(cuts_graph g, uint32_t *n, uint64_t *arcs, int *symmetric,
                    uint32_t *max_degree) {
    if (!g || !g->dev) return set_error(CUTS_ERR_ARG, "null graph");
    if (n) *n = g->dev->n;
    if (arcs) *arcs = g->dev->arcs;
    if (symmetric) *symmetric = g->dev->symmetric;
    if (max_degree) *max_degree = g->dev->max_deg;
    return CUTS_OK;
}

int cuts_graph_set_level_cap(cuts_graph g, uint64_t entries) {
    if (!g || !g->dev) return set_error(CUTS_ERR_ARG, "null graph");
    g->dev->level_cap_req = entries;
    return CUTS_OK;
}

int cuts_graph_set_fuse_split(cuts_graph g, uint32_t split) {
    if (!g || !g->dev) return set_error(CUTS_ERR_ARG, "null graph");
    g->dev->fuse_split = split;
    return CUTS_OK;
}

int cuts_graph_set_arena_bytes(cuts_graph g, uint64_t bytes) {
    if (!g || !g->dev) return set_error(CUTS_ERR_ARG, "null graph");
    DeviceGraph &d = *g->dev;
    cudaSetDevice(d.device);
    if (d.arena) cudaFreeAsync(d.arena, d.stream);
    cudaStreamSynchronize(d.stream);
    d.arena = nullptr;
    d.arena_bytes = bytes ? size_t(bytes) : d.arena_default;
    return CUTS_OK;
}

void cuts_graph_free(cuts_graph g) {
    if (!g) return;
    device_graph_free(g->dev);
    delete g;
}

// ---- query ------------------------------------------------------------------

int cuts_query_load(const char *path, cuts_query *out) {
    if (!path || !out) return set_error(CUTS_ERR_ARG, "null argument");
    *out = nullptr;
    GUARD(([&]() {
        auto qh = std::make_unique<cuts_query_s>();
        int rc = load_query_text(path, qh->q);
        if (rc) return rc;
        *out = qh.release();
        return CUTS_OK;
    })());
}

int cuts_query_from_arcs(uint32_t k, uint32_t narcs, const uint32_t *src, const uint32_t *dst,
                         cuts_query *out) {
    if (!out || (narcs && (!src || !dst))) return set_error(CUTS_ERR_ARG, "null argument");
    *out = nullptr;
    GUARD(([&]() {
        auto qh = std::make_unique<cuts_query_s>();
        int rc = query_from_arcs(k, src, dst, narcs, qh->q);
        if (rc) return rc;
        *out = qh.release();
        return CUTS_OK;
    })());
}

int cuts_query_info(cuts_query q, uint32_t *k, uint32_t *order) {
    if (!q) return set_error(CUTS_ERR_ARG, "null query");
    if (k) *k = q->q.k;
    if (order) std::copy(q->q.order.begin(), q->q.order.end(), order);
    return CUTS_OK;
}

int cuts_query_joins(cuts_query q, uint32_t *p_off, uint32_t *p, uint32_t *c_off, uint32_t *c) {
    if (!q || !p_off || !p || !c_off || !c) return set_error(CUTS_ERR_ARG, "null argument");
    const Query &Q = q->q;
    p_off[0] = c_off[0] = 0;
    for (uint32_t i = 0; i < Q.k; ++i) {
        p_off[i + 1] = p_off[i];
        for (uint32_t j : Q.P[i]) p[p_off[i + 1]++] = j;
        c_off[i + 1] = c_off[i];
        for (uint32_t j : Q.C[i]) c[c_off[i + 1]++] = j;
    }
    return CUTS_OK;
}

int cuts_query_set_order(cuts_query q, const uint32_t *order) {
    if (!q || !order) return set_error(CUTS_ERR_ARG, "null argument");
    GUARD(([&]() {
        Query tmp = q->q;
        int rc = set_order(tmp, std::vector<uint32_t>(order, order + q->q.k));
        if (rc) return rc;
        q->q = std::move(tmp);
        return CUTS_OK;
    })());
}

int cuts_query_prefix(cuts_query q, uint32_t j, cuts_query *out) {
    if (!q || !out) return set_error(CUTS_ERR_ARG, "null argument");
    *out = nullptr;
    GUARD(([&]() {
        auto h = std::make_unique<cuts_query_s>();
        int rc = query_prefix(q->q, j, h->q);
        if (rc) return rc;
        *out = h.release();
        return CUTS_OK;
    })());
}

int cuts_query_plan_levels(cuts_query q, int data_symmetric, uint32_t flags, uint32_t *out,
                           uint64_t *aut) {
    if (!q || !out) return set_error(CUTS_ERR_ARG, "null argument");
    GUARD(([&]() {
        Plan p;
        int rc = build_plan(q->q, data_symmetric != 0, flags, p);
        if (rc) return rc;
        for (uint32_t i = 0; i < q->q.k; ++i) {
            const LevelPlan &L = p.lv[i];
            uint32_t *o = out + 12 * i;
            o[0] = L.nj; o[1] = L.check_sig; o[2] = L.closed_form; o[3] = L.fold;
            o[4] = L.guar_mask; o[5] = L.gt_mask; o[6] = L.lt_mask; o[7] = L.fuse; o[8] = L.ofold;
            o[9] = L.qin; o[10] = L.qout; o[11] = L.fold2;
        }
        if (aut) *aut = p.aut;
        return CUTS_OK;
    })());
}

int cuts_query_automorphisms(cuts_query q, uint64_t *count) {
    if (!q || !count) return set_error(CUTS_ERR_ARG, "null argument");
    *count = automorphism_count(q->q);
    return CUTS_OK;
}

void cuts_query_free(cuts_query q) { delete q; }

// ---- counting -----------------------------------------------------------------

static int count_impl(cuts_graph g, cuts_query q, const CountOptions &opt, uint64_t *count,
                      float *ms, uint64_t *level_sizes, uint64_t *stats) {
    if (!g || !g->dev || !q) return set_error(CUTS_ERR_ARG, "null handle");
    GUARD(([&]() {
        CountResult r;
        int rc = device_count(*g->dev, q->q, opt, r);
        if (rc) return rc;
        if (count) *count = r.count;
        if (ms) *ms = r.ms;
        if (level_sizes) std::copy(r.level_sizes, r.level_sizes + q->q.k, level_sizes);
        if (stats) {
            stats[0] = r.launches;
            stats[1] = r.chunks;
            stats[2] = r.last_level_bytes;
            stats[3] = uint64_t(r.last_level_ms * 1e6);
            stats[4] = uint64_t(r.expand_ms * 1e6);
            stats[5] = r.last_level_launches;
            stats[6] = r.expand_launches;
            stats[7] = 0;
        }
        return CUTS_OK;
    })());
}

int cuts_count_ex(cuts_graph g, cuts_query q, uint32_t chunks, uint32_t flags, uint64_t *count,
                  float *ms, uint64_t *level_sizes, uint64_t *stats) {
    CountOptions opt;
    opt.chunks = chunks;
    opt.flags = flags;
    opt.want_bytes = stats && stats[2] != 0;
    opt.profile = stats && stats[3] != 0;
    return count_impl(g, q, opt, count, ms, level_sizes, stats);
}

int cuts_count_sharded(cuts_graph g, cuts_query q, uint32_t chunks, uint32_t flags,
                       uint32_t shard, uint32_t nshards, uint64_t *count, float *ms,
                       uint64_t *level_sizes) {
    CountOptions opt;
    opt.chunks = chunks;
    opt.flags = flags;
    opt.shard = shard;
    opt.nshards = nshards;
    return count_impl(g, q, opt, count, ms, level_sizes, nullptr);
}

int cuts_count_sharded_ex(cuts_graph g, cuts_query q, uint32_t chunks, uint32_t flags, uint32_t shard,
                          uint32_t nshards, uint64_t *count, float *ms, uint64_t *level_sizes, uint64_t *stats) {
    CountOptions opt;
    opt.chunks = chunks;
    opt.flags = flags;
    opt.shard = shard;
    opt.nshards = nshards;
    opt.want_bytes = stats && stats[2] != 0;
    opt.profile = stats && stats[3] != 0;
    return count_impl(g, q, opt, count, ms, level_sizes, stats);
}

int cuts_count(cuts_graph g, cuts_query q, uint32_t chunks, uint32_t flags, uint64_t *count,
               float *ms) {
    return cuts_count_ex(g, q, chunks, flags, count, ms, nullptr, nullptr);
}

int cuts_count_budget(cuts_graph g, cuts_query q, uint32_t chunks, uint32_t flags,
                      double budget_ms, uint64_t *count, float *ms, uint64_t *level_sizes) {
    CountOptions opt;
    opt.chunks = chunks;
    opt.flags = flags;
    opt.budget_ms = budget_ms;
    return count_impl(g, q, opt, count, ms, level_sizes, nullptr);
}

int cuts_count_sample(cuts_graph g, cuts_query q, uint32_t shard, uint32_t nshards,
                      uint32_t flags, double budget_ms, uint64_t *count, float *ms,
                      uint64_t *level_sizes) {
    CountOptions opt;
    opt.flags = flags;
    opt.shard = shard;
    opt.nshards = nshards;
    opt.budget_ms = budget_ms;
    return count_impl(g, q, opt, count, ms, level_sizes, nullptr);
}

int cuts_dump(cuts_graph g, cuts_query q, const char *path, uint64_t *count) {
    if (!g || !g->dev || !q || !path) return set_error(CUTS_ERR_ARG, "null argument");
    GUARD(device_dump(*g->dev, q->q, path, count));
}

int cuts_dump_sharded(cuts_graph g, cuts_query q, uint32_t shard, uint32_t nshards, const char *path,
                      uint64_t *count) {
    if (!g || !g->dev || !q || !path) return set_error(CUTS_ERR_ARG, "null argument");
    GUARD(device_dump(*g->dev, q->q, path, count, shard, nshards));
}

static std::string base_name(const std::string &s) {
    // common.cpp:19-26: the part after the last '/', or "" without one
    size_t i = s.rfind('/');
    return i == std::string::npos ? std::string() : s.substr(i + 1);
}

int cuts_search(const char *query_file, const char *data_file, int write_to_disk,
                uint32_t trunks, uint64_t *count, float *ms) {
    if (!query_file || !data_file) return set_error(CUTS_ERR_ARG, "null argument");
    GUARD(([&]() {
        std::cout << "start loading graph file from disk to memory..." << std::endl;
        Query q;
        int rc = load_query_text(query_file, q);
        if (rc) return rc;
        HostGraph hg;
        rc = load_graph_text(data_file, hg);
        if (rc) return rc;
        std::cout << "graph loading complete..." << std::endl;
        std::cout << "start copying graph to gpu..." << std::endl;
        DeviceGraph *dg = nullptr;
        rc = device_graph_upload(hg, 0, &dg);
        if (rc) return rc;
        std::unique_ptr<DeviceGraph, void (*)(DeviceGraph *)> hold(dg, device_graph_free);
        std::cout << (trunks ? "finish copying graph to gpu..." : "end copying graph to gpu...")
                  << std::endl;
        CountResult r;
        CountOptions opt;
        opt.chunks = trunks ? trunks : 1;
        // the same count, found once per automorphism class (exact; a query
        // with self-loops is enumerated plainly); CUTS_PLAIN=1 enumerates
        // every embedding as the reference does
        const char *plain = std::getenv("CUTS_PLAIN");
        if (!(plain && plain[0] == '1')) opt.flags = CUTS_FLAG_SYMMETRY_BREAK;
        rc = device_count(*dg, q, opt, r);
        if (rc) return rc;
        std::cout << base_name(data_file) << "," << base_name(query_file) << "," << r.ms << "ms,"
                  << r.count << std::endl;
        if (write_to_disk) {
            std::cout << "start writting matching results to disk,ans.txt" << std::endl;
            uint64_t lines = 0;
            rc = device_dump(*dg, q, "ans.txt", &lines);
            if (rc) return rc;
            std::cout << "finish writting matching results to disk,ans.txt" << std::endl;
        }
        if (count) *count = r.count;
        if (ms) *ms = r.ms;
        return CUTS_OK;
    })());
}

// ---- learned order ------------------------------------------------------------

int cuts_mlp_create(uint32_t in_dim, uint64_t seed, int device, cuts_mlp *out) {
    if (!out) return set_error(CUTS_ERR_ARG, "null argument");
    *out = nullptr;
    GUARD(([&]() {
        auto h = std::make_unique<cuts_mlp_s>();
        int rc = h->m.create(int(in_dim), seed, device);
        if (rc) return rc;
        *out = h.release();
        return CUTS_OK;
    })());
}

int cuts_mlp_param_count(cuts_mlp m, uint32_t *n) {
    if (!m || !n) return set_error(CUTS_ERR_ARG, "null argument");
    *n = uint32_t(mlp_param_count(m->m.in));
    return CUTS_OK;
}

int cuts_mlp_get_params(cuts_mlp m, float *params) {
    if (!m || !params) return set_error(CUTS_ERR_ARG, "null argument");
    return m->m.get_params(params);
}

int cuts_mlp_set_params(cuts_mlp m, const float *params) {
    if (!m || !params) return set_error(CUTS_ERR_ARG, "null argument");
    return m->m.set_params(params);
}

int cuts_mlp_loss_grad(cuts_mlp m, const float *X, const float *y, uint32_t n, float *loss,
                       float *grad) {
    if (!m || !X || !y || n == 0) return set_error(CUTS_ERR_ARG, "bad argument");
    GUARD(m->m.loss_grad(X, y, int(n), loss, grad));
}

int cuts_mlp_train(cuts_mlp m, const float *X, const float *y, uint32_t n, uint32_t epochs,
                   uint32_t batch, float lr, float *final_loss) {
    if (!m || !X || !y || n == 0) return set_error(CUTS_ERR_ARG, "bad argument");
    GUARD(m->m.train(X, y, int(n), int(epochs), int(batch), lr, final_loss));
}

int cuts_mlp_predict(cuts_mlp m, const float *X, uint32_t n, float *y) {
    if (!m || !X || !y) return set_error(CUTS_ERR_ARG, "null argument");
    if (n == 0) return CUTS_OK;
    GUARD(m->m.predict(X, int(n), y));
}

void cuts_mlp_free(cuts_mlp m) { delete m; }

int cuts_query_features(cuts_query q, cuts_graph g, const uint32_t *order,
                        const uint64_t *level_sizes, float *features) {
    if (!q || !g || !g->dev || !order || !features) return set_error(CUTS_ERR_ARG, "null argument");
    GUARD(([&]() {
        const Query &Q = q->q;
        for (uint32_t i = 0; i < Q.k; ++i) {
            const float parent = (i && level_sizes) ? float(std::log1p(double(level_sizes[i - 1]))) : 0.f;
            step_features(Q, g->dev->stats, order, i, parent, features + size_t(i) * kFeatures);
        }
        return CUTS_OK;
    })());
}

int cuts_plan(cuts_query q, cuts_graph g, int mode, cuts_mlp m, uint32_t beam, double margin,
              uint32_t *order_out, double *pred_work, double *score_work) {
    if (!q || !g || !g->dev) return set_error(CUTS_ERR_ARG, "null argument");
    GUARD(([&]() {
        Query &Q = q->q;
        std::vector<uint32_t> order;
        double pw = 0, sw = 0;
        if (mode == CUTS_ORDER_LEARNED && m) {
            OrderSearchOptions opt;
            opt.beam = beam;
            opt.margin = margin > 0 ? margin : 1.25;
            OrderChoice ch;
            int rc = learned_order(Q, g->dev->stats, m->m, opt, ch);
            if (rc) return rc;
            order = ch.order;
            pw = ch.used_learned ? ch.best_work : ch.score_work;
            sw = ch.score_work;
        } else if (mode == CUTS_ORDER_SCORE || mode == CUTS_ORDER_LEARNED) {
            int rc = score_order(Q, order);  // fallback when no model is given
            if (rc) return rc;
        } else {
            return set_error(CUTS_ERR_ARG, "unknown order mode");
        }
        int rc = set_order(Q, order);
        if (rc) return rc;
        if (order_out) std::copy(order.begin(), order.end(), order_out);
        if (pred_work) *pred_work = pw;
        if (score_work) *score_work = sw;
        return CUTS_OK;
    })());
}

int cuts_plan_candidates(cuts_query q, cuts_graph g, cuts_mlp m, uint32_t beam, uint32_t max_orders,
                         uint32_t *orders_out, double *work_out, uint32_t *n_out) {
    if (!q || !g || !g->dev || !m || !orders_out || !n_out) return set_error(CUTS_ERR_ARG, "null argument");
    GUARD(([&]() {
        const Query &Q = q->q;
        OrderSearchOptions opt;
        opt.beam = beam;
        opt.top = max_orders;
        OrderChoice ch;
        int rc = learned_order(Q, g->dev->stats, m->m, opt, ch);
        if (rc) return rc;
        *n_out = uint32_t(ch.top.size());
        for (size_t r = 0; r < ch.top.size(); ++r) {
            std::copy(ch.top[r].begin(), ch.top[r].end(), orders_out + r * Q.k);
            if (work_out) work_out[r] = ch.top_work[r];
        }
        return CUTS_OK;
    })());
}

int cuts_batch_create(cuts_graph g, const cuts_query *qs, uint32_t nq, uint32_t flags,
                      const uint32_t *tune, cuts_batch *out) {
    if (!g || !g->dev || !out || (nq && !qs)) return set_error(CUTS_ERR_ARG, "null argument");
    *out = nullptr;
    GUARD(([&]() {
        std::vector<const Query *> v;
        for (uint32_t i = 0; i < nq; ++i) {
            if (!qs[i]) return set_error(CUTS_ERR_ARG, "null query in batch");
            v.push_back(&qs[i]->q);
        }
        BatchTuning t;
        if (tune) {
            if (tune[0]) t.grain = tune[0];
            if (tune[1]) t.tasks_per_grab = tune[1];
            t.blocks_per_sm = tune[2];
        }
        auto h = std::make_unique<cuts_batch_s>();
        int rc = h->b.create(*g->dev, v, flags, t);
        if (rc) return rc;
        *out = h.release();
        return CUTS_OK;
    })());
}

int cuts_batch_run(cuts_batch b, double budget_ms, uint64_t *counts, int *status, float *ms) {
    if (!b) return set_error(CUTS_ERR_ARG, "null batch");
    GUARD(([&]() {
        std::vector<uint64_t> c;
        std::vector<int> st;
        int rc = b->b.run(budget_ms, c, st, ms);
        if (rc) return rc;
        if (counts) std::copy(c.begin(), c.end(), counts);
        if (status) std::copy(st.begin(), st.end(), status);
        return CUTS_OK;
    })());
}

int cuts_batch_set_query_budget(cuts_batch b, double ms) {
    if (!b || !(ms >= 0)) return set_error(CUTS_ERR_ARG, "bad batch or budget");
    b->b.set_query_budget(ms);
    return CUTS_OK;
}

int cuts_batch_set_shard(cuts_batch b, uint32_t shard, uint32_t nshards) {
    if (!b || nshards == 0 || shard >= nshards) return set_error(CUTS_ERR_ARG, "bad batch or shard");
    b->b.set_shard(shard, nshards);
    return CUTS_OK;
}

int cuts_batch_info(cuts_batch b, uint64_t *tasks, uint32_t *blocks) {
    if (!b) return set_error(CUTS_ERR_ARG, "null batch");
    if (tasks) *tasks = b->b.total_tasks;
    if (blocks) *blocks = b->b.launch_blocks;
    return CUTS_OK;
}

void cuts_batch_free(cuts_batch b) { delete b; }

int cuts_count_batch(cuts_graph g, const cuts_query *qs, uint32_t nq, uint32_t flags,
                     uint64_t *counts, int *status, float *ms) {
    cuts_batch b = nullptr;
    int rc = cuts_batch_create(g, qs, nq, flags, nullptr, &b);
    if (rc) return rc;
    rc = cuts_batch_run(b, 0, counts, status, ms);
    cuts_batch_free(b);
    return rc;
}

int cuts_count_noalloc(const uint32_t *info_out, const uint32_t *info_in, const uint32_t *adj,
                       uint32_t n, const cuts_query *qs, uint32_t nq, uint32_t flags,
                       uint64_t *counts, void *stream) {
    const Query *ptrs[64];
    if (nq > 64) return set_error(CUTS_ERR_LIMIT, "cuts_count_noalloc: more than 64 queries in one call");
    if (nq && !qs) return set_error(CUTS_ERR_ARG, "cuts_count_noalloc: null query array");
    for (uint32_t i = 0; i < nq; ++i) ptrs[i] = qs[i] ? &qs[i]->q : nullptr;
    return count_noalloc(info_out, info_in, adj, n, info_in == nullptr, ptrs, nq, flags,
                         reinterpret_cast<unsigned long long *>(counts),
                         static_cast<cudaStream_t>(stream));
}

}  // extern "C"
