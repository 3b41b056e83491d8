// host.hpp -- host-side types of the cuts_b200 engine (graphs, queries,
// matching order, query plan).  Shared by the C ABI, the CLI and the CUDA
// driver.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/cuts_b200.h"

namespace cuts {

// Thread-local error message behind cuts_last_error().
int set_error(int code, const std::string &msg);
const char *last_error();

// Host CSR with both directions.  When `symmetric`, in_off/in_adj are
// empty and the out-lists serve both directions.
struct HostGraph {
    uint32_t n = 0;
    uint64_t arcs = 0;
    bool symmetric = false;
    std::vector<uint64_t> out_off, in_off;
    std::vector<uint32_t> out_adj, in_adj;

    uint32_t out_deg(uint32_t v) const { return uint32_t(out_off[v + 1] - out_off[v]); }
    uint32_t in_deg(uint32_t v) const {
        return symmetric ? out_deg(v) : uint32_t(in_off[v + 1] - in_off[v]);
    }
    const uint32_t *out_list(uint32_t v) const { return out_adj.data() + out_off[v]; }
    const uint32_t *in_list(uint32_t v) const {
        return symmetric ? out_list(v) : in_adj.data() + in_off[v];
    }
    uint32_t max_degree() const;
};

// Parses the reference text format (util.cpp:19-52): line 1 = V via
// std::stoi semantics, then one arc per line as "s<TAB>t"; lines without a
// TAB are skipped; duplicate arcs collapse; self-loops are kept.
int load_graph_text(const std::string &path, HostGraph &g);
// Builds the CSR from arcs (sorted, deduplicated); detects symmetry.
int graph_from_arcs(uint32_t n, std::vector<uint32_t> &src, std::vector<uint32_t> &dst,
                    HostGraph &g);
// Adopts caller CSR arrays (validates sortedness and ranges).
int graph_from_csr(uint32_t n, const uint64_t *out_off, const uint32_t *out_adj,
                   const uint64_t *in_off, const uint32_t *in_adj, HostGraph &g);
// Writes the reference text format.
int write_graph_text(const std::string &path, const HostGraph &g);
// Binary CSR cache (skips parsing and sorting on reload).
int save_graph_binary(const std::string &path, const HostGraph &g);
int load_graph_binary(const std::string &path, HostGraph &g);

// Query graph with its matching order and P/C join lists over level
// positions (graph.cpp:94-133).
struct Query {
    uint32_t k = 0;
    std::vector<std::vector<uint32_t>> out, in;  // sorted per vertex
    std::vector<uint32_t> order;                 // order[pos] = query vertex
    std::vector<std::vector<uint32_t>> P, C;     // per position: earlier positions
    // A prefix of a larger query keeps that query's degree signatures and
    // tests them at every level (empty: the signatures are the degrees here)
    std::vector<uint32_t> sig_in, sig_out;
    bool has_arc(uint32_t a, uint32_t b) const;
    bool self_loop(uint32_t v) const { return has_arc(v, v); }
    bool loop_free() const;
    bool weakly_connected() const;
};

int query_from_arcs(uint32_t k, const uint32_t *src, const uint32_t *dst, uint32_t narcs,
                    Query &q);
int load_query_text(const std::string &path, Query &q);

// Greedy score order of graph.cpp:62-93 / score.cpp:18-99 (first vertex =
// max out-degree, then lexicographic (score1, score2, score3), lowest id on
// ties) and its P/C lists.
int score_order(const Query &q, std::vector<uint32_t> &order);
// The first j positions of q's order as a query of their own (order kept,
// q's signatures kept): its trie levels are exactly q's first j levels, so
// their sizes can be logged at a fraction of the full run's cost.
int query_prefix(const Query &q, uint32_t j, Query &out);
// Fills q.P / q.C for q.order; rejects orders with an unjoined prefix.
int set_order(Query &q, const std::vector<uint32_t> &order);

// |Aut(Q)|: number of arc-preserving permutations of the query.
uint64_t automorphism_count(const Query &q);
// Symmetry-breaking pairs (a, b) meaning f(a) < f(b), one embedding per
// orbit of Aut(Q) (Grochow & Kellis 2007, "Network motif discovery using
// subgraph enumeration and symmetry-breaking", RECOMB).
std::vector<std::pair<uint32_t, uint32_t>> symmetry_conditions(const Query &q);

// ---- device plan ------------------------------------------------------

constexpr int kMaxK = CUTS_MAX_QUERY;
constexpr int kMaxJ = 32;

// One level of the plan as the kernels read it.
struct LevelPlan {
    uint32_t nj;              // distinct joined lists
    uint32_t qin, qout;       // signature of order[i] (in, out degree)
    uint32_t check_sig;       // apply the signature filter at this level
    uint32_t gt_mask;         // c > m_j required for positions j in mask
    uint32_t lt_mask;         // c < m_j required for positions j in mask
    uint32_t closed_form;     // last level: count by list arithmetic
    uint32_t fold;            // level k-2: also counts level k-1 (closed form
                              // independent of this level's vertex)
    uint32_t guar_mask;       // last level: positions whose vertex the query's
                              // own arcs guarantee to be in the joined list
    uint32_t fuse;            // counted level c: count it from level c-1's
                              // candidate sets (see build_plan)
    uint32_t fuse_extra;      // mask of c's joins beyond c-1's joins and (c-1)
    uint32_t fuse_tp;         // index of c's join on position c-1
    uint32_t ofold;           // last level, orbit fold: positions x of the
                              // pendant's attachment orbit (0 = plain fold)
    uint32_t fold2;           // level k-3: also counts levels k-2 and k-1,
                              // two pendants on earlier positions (1: no
                              // condition between them, 2: one list and
                              // window, the second above / below the first)
    uint32_t guar1;           // level k-2 of a pendant pair: positions whose
                              // vertex the query guarantees in its list
    uint32_t oguar[kMaxK];    // orbit fold: positions j with m_j guaranteed
                              // in the list of m_x, per orbit position x
    uint8_t jpos[kMaxJ];      // joined position j
    uint8_t jdir[kMaxJ];      // 0: out-list of m_j (P join), 1: in-list (C join)
};

struct Plan {
    uint32_t k;
    uint32_t symmetric;       // data graph symmetric: in-lists == out-lists
    uint64_t aut;             // multiplier applied to the count (1 or |Aut|)
    uint32_t data_loops;      // the data graph has self-loops (set by the engine)
    LevelPlan lv[kMaxK];
};

// Builds the plan for q.order on a graph with the given symmetry.
int build_plan(const Query &q, bool data_symmetric, uint32_t flags, Plan &plan);

// ---- seeded generators ------------------------------------------------

// Undirected G(n, p) by geometric skipping (Batagelj & Brandes 2005), both
// arcs per edge, no loops.
void gen_erdos_renyi(uint32_t n, double p, uint64_t seed, HostGraph &g);
// Undirected Chung-Lu graph: weights w_i = min(cap, wmin * U^(-1/(gamma-1))),
// endpoints drawn proportional to w (alias method), loops and duplicates
// rejected, exactly m distinct edges (the first m distinct edges of the
// seeded draw stream).
int gen_chung_lu(uint32_t n, uint64_t m, double gamma, double wmin, double cap,
                 uint64_t seed, HostGraph &g);
// Random connected undirected query: random spanning tree (vertex i attaches
// to a uniform earlier vertex), then each remaining pair with probability p.
void gen_random_query(uint32_t k, double p, uint64_t seed, std::vector<uint32_t> &src,
                      std::vector<uint32_t> &dst);

// splitmix64 (Steele, Lea & Flood 2014) used by every generator.
inline uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
inline double u01(uint64_t h) { return double((h >> 11) + 1) * (1.0 / 9007199254740993.0); }

}  // namespace cuts
