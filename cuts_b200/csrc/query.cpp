// query.cpp -- query graphs, the greedy score order, symmetry conditions and
// the per-level plan the kernels execute.
#include <algorithm>
#include <functional>

#include "host.hpp"

namespace cuts {

bool Query::has_arc(uint32_t a, uint32_t b) const {
    return std::binary_search(out[a].begin(), out[a].end(), b);
}

bool Query::loop_free() const {
    for (uint32_t v = 0; v < k; ++v)
        if (self_loop(v)) return false;
    return true;
}

bool Query::weakly_connected() const {
    if (k == 0) return false;
    std::vector<char> seen(k, 0);
    std::vector<uint32_t> st{0};
    seen[0] = 1;
    uint32_t cnt = 1;
    while (!st.empty()) {
        uint32_t v = st.back();
        st.pop_back();
        for (auto *lst : {&out[v], &in[v]})
            for (uint32_t w : *lst)
                if (!seen[w]) { seen[w] = 1; ++cnt; st.push_back(w); }
    }
    return cnt == k;
}

int query_from_arcs(uint32_t k, const uint32_t *src, const uint32_t *dst, uint32_t narcs,
                    Query &q) {
    if (k == 0) return set_error(CUTS_ERR_QUERY, "query has no vertices");
    if (k > uint32_t(kMaxK))
        return set_error(CUTS_ERR_QUERY, "query has more than " + std::to_string(kMaxK) + " vertices");
    q = Query();
    q.k = k;
    q.out.assign(k, {});
    q.in.assign(k, {});
    for (uint32_t i = 0; i < narcs; ++i) {
        if (src[i] >= k || dst[i] >= k) return set_error(CUTS_ERR_ARG, "query arc out of range");
        q.out[src[i]].push_back(dst[i]);
        q.in[dst[i]].push_back(src[i]);
    }
    for (uint32_t v = 0; v < k; ++v) {
        for (auto *l : {&q.out[v], &q.in[v]}) {
            std::sort(l->begin(), l->end());
            l->erase(std::unique(l->begin(), l->end()), l->end());
        }
    }
    if (k > 1 && !q.weakly_connected())
        return set_error(CUTS_ERR_QUERY,
                         "query is not connected (the reference's order repeats a vertex there)");
    std::vector<uint32_t> order;
    int rc = score_order(q, order);
    if (rc) return rc;
    return set_order(q, order);
}

int load_query_text(const std::string &path, Query &q) {
    HostGraph g;
    int rc = load_graph_text(path, g);
    if (rc) return rc;
    if (g.n > uint32_t(kMaxK))
        return set_error(CUTS_ERR_QUERY, "query has more than " + std::to_string(kMaxK) + " vertices");
    std::vector<uint32_t> s, d;
    for (uint32_t u = 0; u < g.n; ++u)
        for (uint64_t a = g.out_off[u]; a < g.out_off[u + 1]; ++a) {
            s.push_back(u);
            d.push_back(g.out_adj[a]);
        }
    return query_from_arcs(g.n, s.data(), d.data(), uint32_t(s.size()), q);
}

// ---- score order: graph.cpp:62-93, score.cpp:18-99 -------------------

static bool in_prefix(uint32_t v, const std::vector<uint32_t> &sel, size_t len) {
    for (size_t i = 0; i < len; ++i)
        if (sel[i] == v) return true;
    return false;
}

// arcs between v and the ordered set, counted from both sides (score.cpp:18-35)
static uint32_t score1(const Query &q, const std::vector<uint32_t> &sel, size_t len, uint32_t v) {
    uint32_t s = 0;
    for (size_t i = 0; i < len; ++i) s += q.has_arc(sel[i], v);
    for (uint32_t w : q.out[v]) s += in_prefix(w, sel, len);
    return s;
}
// v's out-neighbours among the unordered out-neighbours of the ordered set (score.cpp:36-54)
static uint32_t score2(const Query &q, const std::vector<uint32_t> &sel, size_t len, uint32_t v) {
    std::vector<char> mark(q.k, 0);
    for (size_t i = 0; i < len; ++i)
        for (uint32_t w : q.out[sel[i]])
            if (!in_prefix(w, sel, len)) mark[w] = 1;
    uint32_t s = 0;
    for (uint32_t w = 0; w < q.k; ++w) s += mark[w] && q.has_arc(v, w);
    return s;
}
// v's out-neighbours outside the ordered set and its out-neighbourhood (score.cpp:56-80)
static uint32_t score3(const Query &q, const std::vector<uint32_t> &sel, size_t len, uint32_t v) {
    std::vector<char> reach(q.k, 0);
    for (size_t i = 0; i < len; ++i) {
        reach[sel[i]] = 1;
        for (uint32_t w : q.out[sel[i]]) reach[w] = 1;
    }
    uint32_t s = 0;
    for (uint32_t w = 0; w < q.k; ++w) s += !reach[w] && q.has_arc(v, w);
    return s;
}

int score_order(const Query &q, std::vector<uint32_t> &order) {
    order.assign(q.k, 0);
    uint32_t maxd = 0, idx = 0;
    for (uint32_t v = 0; v < q.k; ++v)
        if (maxd < q.out[v].size()) { maxd = uint32_t(q.out[v].size()); idx = v; }
    order[0] = idx;
    for (size_t ins = 1; ins < q.k; ++ins) {
        uint32_t b1 = 0, b2 = 0, b3 = 0;
        for (uint32_t v = 0; v < q.k; ++v) {
            if (in_prefix(v, order, ins)) continue;
            uint32_t s1 = score1(q, order, ins, v), s2 = score2(q, order, ins, v),
                     s3 = score3(q, order, ins, v);
            // strict lexicographic '>' (score.cpp:81-99): lowest id wins ties
            if (s1 > b1 || (s1 == b1 && (s2 > b2 || (s2 == b2 && s3 > b3)))) {
                b1 = s1; b2 = s2; b3 = s3; idx = v;
            }
        }
        order[ins] = idx;
    }
    return CUTS_OK;
}

int query_prefix(const Query &q, uint32_t j, Query &out) {
    if (q.order.size() != q.k || j < 1 || j > q.k) return set_error(CUTS_ERR_ARG, "bad prefix length");
    std::vector<int> pos(q.k, -1);
    for (uint32_t i = 0; i < j; ++i) pos[q.order[i]] = int(i);
    Query p;
    p.k = j;
    p.out.assign(j, {});
    p.in.assign(j, {});
    p.sig_in.resize(j);
    p.sig_out.resize(j);
    for (uint32_t i = 0; i < j; ++i) {
        const uint32_t v = q.order[i];
        for (uint32_t w : q.out[v])
            if (pos[w] >= 0) p.out[i].push_back(uint32_t(pos[w]));
        for (uint32_t w : q.in[v])
            if (pos[w] >= 0) p.in[i].push_back(uint32_t(pos[w]));
        std::sort(p.out[i].begin(), p.out[i].end());
        std::sort(p.in[i].begin(), p.in[i].end());
        p.sig_in[i] = uint32_t(q.in[v].size());
        p.sig_out[i] = uint32_t(q.out[v].size());
    }
    std::vector<uint32_t> ident(j);
    for (uint32_t i = 0; i < j; ++i) ident[i] = i;
    int rc = set_order(p, ident);
    if (rc) return rc;
    out = std::move(p);
    return CUTS_OK;
}

int set_order(Query &q, const std::vector<uint32_t> &order) {
    if (order.size() != q.k) return set_error(CUTS_ERR_ARG, "order length != k");
    std::vector<char> seen(q.k, 0);
    for (uint32_t v : order) {
        if (v >= q.k || seen[v]) return set_error(CUTS_ERR_ARG, "order is not a permutation");
        seen[v] = 1;
    }
    q.order = order;
    q.P.assign(q.k, {});
    q.C.assign(q.k, {});
    for (uint32_t i = 1; i < q.k; ++i) {
        uint32_t v = order[i];
        for (uint32_t j = 0; j < i; ++j) {
            uint32_t t = order[j];
            if (q.has_arc(v, t)) q.C[i].push_back(j);   // arc v -> order[j]
            if (q.has_arc(t, v)) q.P[i].push_back(j);   // arc order[j] -> v
        }
        if (q.P[i].empty() && q.C[i].empty())
            return set_error(CUTS_ERR_QUERY, "order position " + std::to_string(i) +
                                                 " has no arc to an earlier position");
    }
    return CUTS_OK;
}

// ---- automorphisms ------------------------------------------------------

// Finds one arc-preserving permutation with perm[fixed[i]] = fixed[i] and
// perm[v] = w, by backtracking over vertices in id order.
static bool find_automorphism(const Query &q, const std::vector<uint32_t> &fixed, uint32_t v,
                              uint32_t w) {
    const uint32_t k = q.k;
    std::vector<int> img(k, -1), used(k, 0);
    for (uint32_t f : fixed) { img[f] = int(f); used[f] = 1; }
    if (img[v] >= 0 && img[v] != int(w)) return false;
    if (img[v] < 0) {
        if (used[w]) return false;
        img[v] = int(w);
        used[w] = 1;
    }
    auto consistent = [&](uint32_t a) {
        uint32_t fa = uint32_t(img[a]);
        if (q.out[a].size() != q.out[fa].size() || q.in[a].size() != q.in[fa].size()) return false;
        for (uint32_t b = 0; b < k; ++b) {
            if (img[b] < 0) continue;
            uint32_t fb = uint32_t(img[b]);
            if (q.has_arc(a, b) != q.has_arc(fa, fb)) return false;
            if (q.has_arc(b, a) != q.has_arc(fb, fa)) return false;
        }
        return true;
    };
    for (uint32_t a = 0; a < k; ++a)
        if (img[a] >= 0 && !consistent(a)) return false;
    std::function<bool(uint32_t)> rec = [&](uint32_t a) -> bool {
        if (a == k) return true;
        if (img[a] >= 0) return rec(a + 1);
        for (uint32_t c = 0; c < k; ++c) {
            if (used[c]) continue;
            img[a] = int(c);
            used[c] = 1;
            if (consistent(a) && rec(a + 1)) return true;
            used[c] = 0;
            img[a] = -1;
        }
        return false;
    };
    return rec(0);
}

// Stabiliser chain: repeatedly take the earliest-ordered vertex with a
// nontrivial orbit under the current stabiliser, require f(v) < f(w) for the
// rest of its orbit, then fix v.  |Aut| = product of the orbit sizes.
static void stabiliser_chain(const Query &q, std::vector<std::pair<uint32_t, uint32_t>> *conds,
                             uint64_t *aut) {
    std::vector<uint32_t> fixed;
    uint64_t total = 1;
    std::vector<uint32_t> by_pos = q.order.empty() ? std::vector<uint32_t>() : q.order;
    if (by_pos.empty())
        for (uint32_t v = 0; v < q.k; ++v) by_pos.push_back(v);
    while (true) {
        bool any = false;
        for (uint32_t v : by_pos) {
            if (std::find(fixed.begin(), fixed.end(), v) != fixed.end()) continue;
            std::vector<uint32_t> orbit;
            for (uint32_t w = 0; w < q.k; ++w)
                if (w == v || find_automorphism(q, fixed, v, w)) orbit.push_back(w);
            if (orbit.size() > 1) {
                for (uint32_t w : orbit)
                    if (w != v && conds) conds->push_back({v, w});
                total *= orbit.size();
                fixed.push_back(v);
                any = true;
                break;
            }
        }
        if (!any) break;
    }
    if (aut) *aut = total;
}

std::vector<std::pair<uint32_t, uint32_t>> symmetry_conditions(const Query &q) {
    std::vector<std::pair<uint32_t, uint32_t>> c;
    stabiliser_chain(q, &c, nullptr);
    return c;
}

uint64_t automorphism_count(const Query &q) {
    uint64_t a = 1;
    stabiliser_chain(q, nullptr, &a);
    return a;
}

// ---- plan ---------------------------------------------------------------

// Orbit fold.  When the last vertex e of the order is a pendant on vertex a
// (its level is a closed form over a's list L), every embedding of Q is an
// embedding psi of the core C = Q - e plus one vertex of L(psi(a)) outside
// psi(C).  Summing over the |Aut(C)| embeddings psi = phi o sigma of one
// class, psi(a) = phi(x) runs over the orbit O of a under Aut(C), each x
// |Aut(C)| / |O| times, so
//   count(Q) = |Aut(C)| / |O| x sum over one phi per class of
//              sum_{x in O} ( |L(phi(x))| - |L(phi(x)) n phi(C)| ).
// The core's own symmetry is broken (its stabiliser chain), which leaves
// |O| times fewer core embeddings to enumerate than breaking Q's.  The
// weight is evaluated at level k-2 (a fold); the memberships that involve
// the level k-2 vertex must be implied by the query's arcs, so that the
// per-candidate weight needs no list search.  Returns false (plan untouched)
// when the query does not have that shape or the orbit is trivial.
// The query vertex at order position jp.
static inline uint32_t a_of(const Query &q, uint32_t jp) { return q.order[jp]; }

static bool orbit_fold_plan(const Query &q, bool data_symmetric, Plan &plan) {
    const uint32_t k = q.k, c = k - 2;
    LevelPlan &F = plan.lv[k - 1];
    if (k < 3 || !F.closed_form || F.nj != 1) return false;
    const uint32_t jf = F.jpos[0], dir = F.jdir[0];
    const uint32_t e = q.order[k - 1];
    std::vector<uint32_t> pos(k);
    for (uint32_t i = 0; i < k; ++i) pos[q.order[i]] = i;
    // the core, relabelled by position
    Query C;
    C.k = k - 1;
    C.out.assign(k - 1, {});
    C.in.assign(k - 1, {});
    for (uint32_t i = 0; i + 1 < k; ++i) {
        const uint32_t v = q.order[i];
        for (uint32_t w : q.out[v])
            if (w != e) C.out[i].push_back(pos[w]);
        for (uint32_t w : q.in[v])
            if (w != e) C.in[i].push_back(pos[w]);
        std::sort(C.out[i].begin(), C.out[i].end());
        std::sort(C.in[i].begin(), C.in[i].end());
    }
    for (uint32_t i = 0; i + 1 < k; ++i) C.order.push_back(i);
    uint32_t omask = 1u << jf;
    for (uint32_t x = 0; x + 1 < k; ++x)
        if (x != jf && find_automorphism(C, {}, jf, x)) omask |= 1u << x;
    if (__builtin_popcount(omask) < 2) return false;
    // m_j is in the list of m_x whenever the query has the arc that list stands for
    uint32_t oguar[kMaxK] = {};
    for (uint32_t x = 0; x + 1 < k; ++x) {
        if (!((omask >> x) & 1u)) continue;
        for (uint32_t j = 0; j + 1 < k; ++j) {
            if (j == x) continue;
            const uint32_t a = q.order[x], b = q.order[j];
            const bool fwd = dir == 0 ? q.has_arc(a, b) : q.has_arc(b, a);
            const bool rev = dir == 0 ? q.has_arc(b, a) : q.has_arc(a, b);
            if (fwd || (data_symmetric && rev)) oguar[x] |= 1u << j;
        }
    }
    for (uint32_t x = 0; x < c; ++x)
        if (((omask >> x) & 1u) && !((oguar[x] >> c) & 1u)) return false;
    if (((omask >> c) & 1u) && (oguar[c] & ((1u << c) - 1)) != ((1u << c) - 1)) return false;
    std::vector<std::pair<uint32_t, uint32_t>> conds;
    uint64_t autc = 1;
    stabiliser_chain(C, &conds, &autc);
    for (auto &cd : conds) {  // f(a) < f(b), positions
        const uint32_t pa = cd.first, pb = cd.second;
        if (pb > pa) plan.lv[pb].gt_mask |= 1u << pa;
        else plan.lv[pa].lt_mask |= 1u << pb;
    }
    plan.aut = autc / uint64_t(__builtin_popcount(omask));
    // the core's positions are filtered by their degrees in the core: an
    // orbit vertex other than a carries no pendant arc, and the class
    // representative may put any orbit vertex at a's position
    for (uint32_t i = 0; i + 1 < k; ++i) {
        plan.lv[i].qin = uint32_t(C.in[i].size());
        plan.lv[i].qout = uint32_t(C.out[i].size());
    }
    F.ofold = omask;
    for (uint32_t x = 0; x < kMaxK; ++x) F.oguar[x] = oguar[x];
    plan.lv[k - 2].fold = 1;
    return true;
}

int build_plan(const Query &q, bool data_symmetric, uint32_t flags, Plan &plan) {
    plan = Plan();
    plan.k = q.k;
    plan.symmetric = data_symmetric;
    plan.aut = 1;
    const uint32_t k = q.k;
    for (uint32_t i = 0; i < k; ++i) {
        LevelPlan &L = plan.lv[i];
        const uint32_t v = q.order[i];
        L.qin = q.sig_in.empty() ? uint32_t(q.in[v].size()) : q.sig_in[v];
        L.qout = q.sig_out.empty() ? uint32_t(q.out[v].size()) : q.sig_out[v];
        uint32_t nj = 0;
        auto add = [&](uint32_t pos, uint32_t dir) {
            if (data_symmetric) dir = 0;  // in-list == out-list: one list per position
            for (uint32_t t = 0; t < nj; ++t)
                if (L.jpos[t] == pos && L.jdir[t] == dir) return;
            L.jpos[nj] = uint8_t(pos);
            L.jdir[nj] = uint8_t(dir);
            ++nj;
        };
        if (i > 0) {
            for (uint32_t j : q.P[i]) add(j, 0);  // candidate in out-list of m_j
            for (uint32_t j : q.C[i]) add(j, 1);  // candidate in in-list of m_j
        }
        L.nj = nj;
        // At the last level every arc of order[k-1] is a join, so a
        // candidate that passes the joins and injectivity already has the
        // degrees the signature asks for -- unless the query vertex has a
        // self-loop, which the joins never check but the signature counts.
        L.check_sig = (i + 1 < k) || q.self_loop(v) || !q.sig_in.empty();
        L.closed_form = (k >= 2 && i + 1 == k && nj == 1 && !L.check_sig &&
                         !(flags & CUTS_FLAG_NO_CLOSED_FORM));
        if (L.closed_form) {
            // m_j lies in the joined list whenever the query has the arc the
            // list stands for (or its reverse on a symmetric data graph)
            const uint32_t jp = L.jpos[0], a = q.order[jp];
            for (uint32_t j = 0; j < i; ++j) {
                if (j == jp) continue;  // a query self-loop is not a data constraint
                const uint32_t b = q.order[j];
                const bool fwd = L.jdir[0] == 0 ? q.has_arc(a, b) : q.has_arc(b, a);
                const bool rev = L.jdir[0] == 0 ? q.has_arc(b, a) : q.has_arc(a, b);
                if (fwd || (data_symmetric && rev)) L.guar_mask |= 1u << j;
            }
        }
    }
    // symmetry breaking needs the query's own automorphisms, which a prefix
    // with a larger query's signatures does not have: prefixes count plainly
    const bool sym = (flags & CUTS_FLAG_SYMMETRY_BREAK) && q.loop_free() && q.sig_in.empty();
    const bool orbit = sym && !(flags & CUTS_FLAG_NO_ORBIT_FOLD) && k >= 3 &&
                       orbit_fold_plan(q, data_symmetric, plan);
    if (sym && k >= 2 && !orbit) {
        std::vector<uint32_t> pos(k);
        for (uint32_t i = 0; i < k; ++i) pos[q.order[i]] = i;
        std::vector<std::pair<uint32_t, uint32_t>> conds;
        uint64_t aut = 1;
        stabiliser_chain(q, &conds, &aut);
        for (auto &c : conds) {  // f(a) < f(b)
            uint32_t pa = pos[c.first], pb = pos[c.second];
            if (pb > pa) plan.lv[pb].gt_mask |= 1u << pa;
            else plan.lv[pa].lt_mask |= 1u << pb;
        }
        plan.aut = aut;
    }
    // Fold the last level into level k-2 when its closed form does not
    // depend on the vertex chosen at k-2: the joined list is an earlier
    // position's and no symmetry condition involves position k-2.  Each
    // level k-2 candidate then contributes the closed form directly.
    if (k >= 3 && plan.lv[k - 1].closed_form) {
        const LevelPlan &F = plan.lv[k - 1];
        const uint32_t pen = 1u << (k - 2);
        if (F.jpos[0] != k - 2 && !(F.gt_mask & pen) && !(F.lt_mask & pen)) plan.lv[k - 2].fold = 1;
    }
    // Pendant pair: the last two vertices are both pendants on earlier
    // positions (each joins one list of a position below k-2, every query
    // arc of theirs goes there, no self-loop -- so the joins imply their
    // signatures) and both join the same list.  Their pairs (t1, t2) have a
    // closed form per level k-3 candidate: with no condition between them,
    // |A'| |B'| - |A' n B'| (A', B' the two windows of that list minus the
    // matched vertices; A' n B' a window difference); with t2 above (or
    // below) t1 on the same window, |A'| choose 2.  Level k-3 then counts
    // both levels (plain orbit-free plans only).  Pendants on two different
    // lists stay unfolded: |A' n B'| would be a serial intersection in one
    // lane, over hub lists as long as the largest degree.
    if (k >= 4 && !(flags & CUTS_FLAG_NO_PAIR_FOLD) && plan.lv[k - 1].closed_form && !plan.lv[k - 1].ofold) {
        LevelPlan &L1 = plan.lv[k - 2];
        const LevelPlan &L2 = plan.lv[k - 1];
        const uint32_t p1 = k - 2, pen = 1u << p1;
        const uint32_t v1 = q.order[p1];
        bool ok = L1.nj == 1 && L1.jpos[0] < p1 && L2.jpos[0] == L1.jpos[0] &&
                  L2.jdir[0] == L1.jdir[0] && !q.self_loop(v1) && q.sig_in.empty();
        if (ok) {  // every arc of v1 goes to the vertex its list belongs to
            const uint32_t a = q.order[L1.jpos[0]];
            for (uint32_t w : q.out[v1]) ok = ok && w == a;
            for (uint32_t w : q.in[v1]) ok = ok && w == a;
        }
        if (ok && !(L1.gt_mask & pen) && !(L1.lt_mask & pen)) {
            const bool cond = ((L2.gt_mask | L2.lt_mask) & pen) != 0;
            uint32_t kind = 0;
            if (!cond) {
                kind = 1;
            } else if (((L2.gt_mask & pen) != 0) != ((L2.lt_mask & pen) != 0) &&
                       L1.gt_mask == (L2.gt_mask & ~pen) &&
                       L1.lt_mask == (L2.lt_mask & ~pen)) {
                kind = 2;
            }
            if (kind) {
                // matched vertices the query's arcs put in v1's list
                const uint32_t jp = L1.jpos[0];
                L1.guar1 = 0;
                for (uint32_t j = 0; j < p1; ++j) {
                    if (j == jp) continue;
                    const uint32_t b = q.order[j];
                    const bool fwd = L1.jdir[0] == 0 ? q.has_arc(a_of(q, jp), b) : q.has_arc(b, a_of(q, jp));
                    const bool rev = L1.jdir[0] == 0 ? q.has_arc(b, a_of(q, jp)) : q.has_arc(a_of(q, jp), b);
                    if (fwd || (data_symmetric && rev)) L1.guar1 |= 1u << j;
                }
                plan.lv[k - 3].fold2 = kind;
                plan.lv[k - 2].fold = 0;
            }
        }
    }
    // Fuse the counted level c with level p = c-1 when c's candidates are a
    // subset of p's: every list p joins is joined at c too, c also joins p's
    // own vertex, p's signature is no stricter than c's, and p's symmetry
    // window is no narrower than c's (p's conditions are among c's).  Then,
    // for one parent at level p-1, p's candidate set S serves every vertex s
    // chosen at p: c's candidates are the t in S that lie in s's list.
    if (k >= 3 && !(flags & CUTS_FLAG_NO_FUSE) && !(k >= 4 && plan.lv[k - 3].fold2)) {
        const uint32_t c = (plan.lv[k - 2].fold) ? k - 2 : k - 1;
        const uint32_t p = c - 1;
        LevelPlan &Lc = plan.lv[c];
        const LevelPlan &Lp = plan.lv[p];
        bool ok = p >= 1 && !Lc.closed_form && Lp.check_sig && Lc.qin >= Lp.qin && Lc.qout >= Lp.qout;
        const uint32_t below = (1u << p) - 1;
        ok = ok && (Lp.gt_mask & below & ~Lc.gt_mask) == 0 && (Lp.lt_mask & below & ~Lc.lt_mask) == 0;
        uint32_t tp = kMaxJ, covered = 0;
        for (uint32_t t = 0; ok && t < Lc.nj; ++t)
            if (Lc.jpos[t] == p && tp == kMaxJ) { tp = t; covered |= 1u << t; }
        ok = ok && tp != kMaxJ;
        for (uint32_t u = 0; ok && u < Lp.nj; ++u) {
            bool found = false;
            for (uint32_t t = 0; t < Lc.nj; ++t)
                if (Lc.jpos[t] == Lp.jpos[u] && Lc.jdir[t] == Lp.jdir[u]) { found = true; covered |= 1u << t; }
            ok = found;
        }
        if (ok) {
            Lc.fuse = 1;
            Lc.fuse_tp = tp;
            Lc.fuse_extra = ((Lc.nj >= 32) ? ~0u : ((1u << Lc.nj) - 1)) & ~covered;
        }
    }
    return CUTS_OK;
}

}  // namespace cuts
