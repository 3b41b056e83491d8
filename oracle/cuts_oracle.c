/*
 * cuts_oracle.c -- CPU oracle (test infrastructure only; see cuts_oracle.h).
 *
 * Plain C11 + OpenMP restatement of the reference's counting path:
 *   loader            util.cpp:19-52
 *   CSR + signatures  graph.cpp:18-61
 *   order + P/C       graph.cpp:62-134, score.cpp:18-99, common.cpp:27-42
 *   level semantics   device_funcs.cu:57-100 (candidates from the smallest
 *                     joined list, not yet matched, signature-OK),
 *                     device_funcs.cu:128-232 (membership in every other
 *                     joined list: a P join uses the matched vertex's
 *                     out-list, a C join its in-list),
 *                     device_funcs.cu:267-279 (level 0 signature scan),
 *                     host_funcs.cu:115-171 (count only at iter == k-1 >= 1).
 */
#include "cuts_oracle.h"

#include <ctype.h>
#include <errno.h>
#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ */
/* graph construction                                                  */
/* ------------------------------------------------------------------ */

static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

/* Build one CSR from (key, val) pairs packed as key<<32|val; sorts and
 * dedups in place (the reference inserts into std::set, util.cpp:46-47). */
static int build_csr(uint32_t n, uint64_t narcs, uint64_t *packed,
                     uint64_t **off_out, uint32_t **adj_out, uint64_t *nuniq) {
    qsort(packed, (size_t)narcs, sizeof(uint64_t), cmp_u64);
    uint64_t u = 0;
    for (uint64_t i = 0; i < narcs; ++i)
        if (i == 0 || packed[i] != packed[i - 1]) packed[u++] = packed[i];
    uint64_t *off = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    uint32_t *adj = (uint32_t *)malloc((size_t)(u ? u : 1) * sizeof(uint32_t));
    if (!off || !adj) { free(off); free(adj); return OR_ERR_NOMEM; }
    for (uint64_t i = 0; i < u; ++i) {
        off[(packed[i] >> 32) + 1]++;
        adj[i] = (uint32_t)(packed[i] & 0xffffffffu);
    }
    for (uint32_t v = 0; v < n; ++v) off[v + 1] += off[v];
    *off_out = off; *adj_out = adj; *nuniq = u;
    return OR_OK;
}

int or_graph_from_arcs(uint32_t n, uint64_t narcs, const uint32_t *src,
                       const uint32_t *dst, or_graph *g) {
    memset(g, 0, sizeof(*g));
    uint64_t *pk = (uint64_t *)malloc((size_t)(narcs ? narcs : 1) * sizeof(uint64_t));
    if (!pk) return OR_ERR_NOMEM;
    for (uint64_t i = 0; i < narcs; ++i) {
        if (src[i] >= n || dst[i] >= n) { free(pk); return OR_ERR_RANGE; }
        pk[i] = ((uint64_t)src[i] << 32) | dst[i];
    }
    uint64_t u1 = 0, u2 = 0;
    int rc = build_csr(n, narcs, pk, &g->out_off, &g->out_adj, &u1);
    if (rc) { free(pk); return rc; }
    for (uint64_t i = 0; i < narcs; ++i) pk[i] = ((uint64_t)dst[i] << 32) | src[i];
    rc = build_csr(n, narcs, pk, &g->in_off, &g->in_adj, &u2);
    free(pk);
    if (rc) { or_free_graph(g); return rc; }
    g->n = n;
    g->arcs = u1;
    return OR_OK;
}

void or_free_graph(or_graph *g) {
    free(g->out_off); free(g->out_adj); free(g->in_off); free(g->in_adj);
    memset(g, 0, sizeof(*g));
}

int or_is_symmetric(const or_graph *g) {
    if (memcmp(g->out_off, g->in_off, ((size_t)g->n + 1) * sizeof(uint64_t))) return 0;
    return memcmp(g->out_adj, g->in_adj, (size_t)g->arcs * sizeof(uint32_t)) == 0;
}

/* std::stoi prefix semantics: skip leading whitespace, optional sign,
 * at least one digit, stop at the first non-digit.  Returns 0 on success. */
static int parse_int_prefix(const char *s, const char *end, long long *out) {
    while (s < end && isspace((unsigned char)*s)) ++s;
    int neg = 0;
    if (s < end && (*s == '+' || *s == '-')) { neg = (*s == '-'); ++s; }
    if (s >= end || !isdigit((unsigned char)*s)) return OR_ERR_PARSE;
    long long v = 0;
    while (s < end && isdigit((unsigned char)*s)) {
        v = v * 10 + (*s - '0');
        if (v > INT_MAX + 1LL) return OR_ERR_PARSE; /* stoi throws out_of_range */
        ++s;
    }
    v = neg ? -v : v;
    if (v > INT_MAX || v < INT_MIN) return OR_ERR_PARSE;
    *out = v;
    return OR_OK;
}

int or_load_graph(const char *path, or_graph *g) {
    memset(g, 0, sizeof(*g));
    FILE *f = fopen(path, "rb");
    if (!f) return OR_ERR_IO;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    char *buf = (char *)malloc((size_t)sz + 1);
    if (!buf) { fclose(f); return OR_ERR_NOMEM; }
    if (sz > 0 && fread(buf, 1, (size_t)sz, f) != (size_t)sz) { free(buf); fclose(f); return OR_ERR_IO; }
    fclose(f);
    buf[sz] = 0;
    const char *p = buf, *end = buf + sz;
    /* line 1: V = stoi(line) */
    const char *nl = memchr(p, '\n', (size_t)(end - p));
    const char *le = nl ? nl : end;
    long long V;
    if (parse_int_prefix(p, le, &V) || V < 0) { free(buf); return OR_ERR_PARSE; }
    p = nl ? nl + 1 : end;
    uint64_t cap = 1024, na = 0;
    uint32_t *src = (uint32_t *)malloc(cap * 4), *dst = (uint32_t *)malloc(cap * 4);
    int rc = OR_OK;
    while (p < end && rc == OR_OK) {
        nl = memchr(p, '\n', (size_t)(end - p));
        le = nl ? nl : end;
        const char *tab = memchr(p, '\t', (size_t)(le - p));
        if (tab) { /* lines without a TAB are skipped (util.cpp:40-43) */
            long long s, t;
            if (parse_int_prefix(p, tab, &s) || parse_int_prefix(tab + 1, le, &t)) rc = OR_ERR_PARSE;
            else if (s < 0 || t < 0 || s >= V || t >= V) rc = OR_ERR_RANGE;
            else {
                if (na == cap) {
                    cap *= 2;
                    src = (uint32_t *)realloc(src, cap * 4);
                    dst = (uint32_t *)realloc(dst, cap * 4);
                }
                src[na] = (uint32_t)s; dst[na] = (uint32_t)t; ++na;
            }
        }
        p = nl ? nl + 1 : end;
    }
    free(buf);
    if (rc == OR_OK) rc = or_graph_from_arcs((uint32_t)V, na, src, dst, g);
    free(src); free(dst);
    return rc;
}

/* ------------------------------------------------------------------ */
/* order (graph.cpp:62-134, score.cpp:18-99)                           */
/* ------------------------------------------------------------------ */

/* common.cpp:27-34 -- named binary_search, actually a linear scan. */
static int lin_has(uint32_t v, const uint32_t *a, uint64_t s, uint64_t e) {
    for (uint64_t i = s; i < e; ++i) if (a[i] == v) return 1;
    return 0;
}

static uint32_t score1(const or_graph *q, const uint32_t *sel, uint32_t len, uint32_t v) {
    uint32_t dout = 0, din = 0;
    for (uint32_t i = 0; i < len; ++i)
        if (lin_has(v, q->out_adj, q->out_off[sel[i]], q->out_off[sel[i] + 1])) dout++;
    for (uint64_t i = q->out_off[v]; i < q->out_off[v + 1]; ++i)
        if (lin_has(q->out_adj[i], sel, 0, len)) din++;
    return dout + din;
}

static uint32_t score2(const or_graph *q, const uint32_t *sel, uint32_t len, uint32_t v) {
    char mark[OR_MAX_QUERY] = {0};
    for (uint32_t i = 0; i < len; ++i)
        for (uint64_t a = q->out_off[sel[i]]; a < q->out_off[sel[i] + 1]; ++a) {
            uint32_t w = q->out_adj[a];
            if (!lin_has(w, sel, 0, len)) mark[w] = 1;
        }
    uint32_t s = 0;
    for (uint32_t w = 0; w < q->n; ++w)
        if (mark[w] && lin_has(w, q->out_adj, q->out_off[v], q->out_off[v + 1])) s++;
    return s;
}

static uint32_t score3(const or_graph *q, const uint32_t *sel, uint32_t len, uint32_t v) {
    char reach[OR_MAX_QUERY] = {0};
    for (uint32_t i = 0; i < len; ++i) {
        reach[sel[i]] = 1;
        for (uint64_t a = q->out_off[sel[i]]; a < q->out_off[sel[i] + 1]; ++a) reach[q->out_adj[a]] = 1;
    }
    uint32_t s = 0;
    for (uint32_t w = 0; w < q->n; ++w)
        if (!reach[w] && lin_has(w, q->out_adj, q->out_off[v], q->out_off[v + 1])) s++;
    return s;
}

int or_joins_for_order(const or_graph *q, const uint32_t *order, uint32_t *p_off,
                       uint32_t *p, uint32_t *c_off, uint32_t *c) {
    uint32_t k = q->n, np = 0, nc = 0;
    p_off[0] = c_off[0] = 0;
    /* level 0 has no joins; levels i>=1 join earlier positions j (graph.cpp:94-113) */
    for (uint32_t i = 0; i < k; ++i) {
        if (i > 0) {
            uint32_t v = order[i];
            for (uint32_t j = 0; j < i; ++j) {
                uint32_t t = order[j];
                if (lin_has(t, q->out_adj, q->out_off[v], q->out_off[v + 1])) c[nc++] = j;
                if (lin_has(t, q->in_adj, q->in_off[v], q->in_off[v + 1])) p[np++] = j;
            }
        }
        p_off[i + 1] = np;
        c_off[i + 1] = nc;
    }
    return OR_OK;
}

int or_order(const or_graph *q, uint32_t *order, uint32_t *p_off, uint32_t *p,
             uint32_t *c_off, uint32_t *c) {
    uint32_t k = q->n;
    if (k == 0 || k > OR_MAX_QUERY) return OR_ERR_QUERY;
    /* first vertex: max out-degree, lowest id on ties (graph.cpp:68-75).
     * idx is uninitialised in the reference when every out-degree is 0;
     * the oracle takes vertex 0 there. */
    uint32_t maxd = 0, idx = 0;
    for (uint32_t v = 0; v < k; ++v) {
        uint32_t d = (uint32_t)(q->out_off[v + 1] - q->out_off[v]);
        if (maxd < d) { maxd = d; idx = v; }
    }
    order[0] = idx;
    uint32_t ins = 1;
    while (ins < k) { /* graph.cpp:77-93: strict '>' keeps the lowest id; idx
                         stays stale when nothing beats (0,0,0) */
        uint32_t b1 = 0, b2 = 0, b3 = 0;
        for (uint32_t v = 0; v < k; ++v) {
            if (lin_has(v, order, 0, ins)) continue;
            uint32_t s1 = score1(q, order, ins, v);
            uint32_t s2 = score2(q, order, ins, v);
            uint32_t s3 = score3(q, order, ins, v);
            int better = (s1 > b1) || (s1 == b1 && (s2 > b2 || (s2 == b2 && s3 > b3)));
            if (better) { b1 = s1; b2 = s2; b3 = s3; idx = v; }
        }
        order[ins++] = idx;
    }
    return or_joins_for_order(q, order, p_off, p, c_off, c);
}

/* ------------------------------------------------------------------ */
/* counting                                                            */
/* ------------------------------------------------------------------ */

typedef struct {
    const or_graph *d;
    uint32_t k;
    uint32_t qin[OR_MAX_QUERY], qout[OR_MAX_QUERY];   /* per level position */
    uint32_t nj[OR_MAX_QUERY];                        /* joins per level */
    uint32_t jpos[OR_MAX_QUERY][2 * OR_MAX_QUERY];
    uint8_t jout[OR_MAX_QUERY][2 * OR_MAX_QUERY];     /* 1 = P join (out-list) */
    int symmetric;
    /* ordering conditions: at level i the candidate must exceed M[j] for
     * j in gt[i] and lie below M[j] for j in lt[i] (0 = no condition) */
    uint32_t gt[OR_MAX_QUERY], lt[OR_MAX_QUERY];
    /* count the last level by list arithmetic when it joins one list */
    int closed_last;
    int last_single;      /* the last level's joins name one list */
    int last_loop_free;   /* the last query vertex has no self-loop */
} plan_t;

typedef struct {
    uint64_t lvl[OR_MAX_QUERY];
    uint64_t bytes;
    or_match_cb cb;
    void *user;
    const uint32_t *order;
} acc_t;

static int sig_ok(const plan_t *P, uint32_t i, uint32_t u) {
    const or_graph *d = P->d;
    uint64_t din = d->in_off[u + 1] - d->in_off[u];
    uint64_t dout = d->out_off[u + 1] - d->out_off[u];
    return din >= P->qin[i] && dout >= P->qout[i];  /* common.cpp:35-42 */
}

static int bsearch_u32(const uint32_t *a, uint64_t s, uint64_t e, uint32_t x) {
    while (s < e) {
        uint64_t m = s + (e - s) / 2;
        if (a[m] < x) s = m + 1; else if (a[m] > x) e = m; else return 1;
    }
    return 0;
}

static void list_of(const plan_t *P, uint32_t i, uint32_t t, const uint32_t *M,
                     const uint32_t **lst, uint64_t *len) {
    const or_graph *d = P->d;
    uint32_t u = M[P->jpos[i][t]];
    if (P->jout[i][t]) { *lst = d->out_adj + d->out_off[u]; *len = d->out_off[u + 1] - d->out_off[u]; }
    else { *lst = d->in_adj + d->in_off[u]; *len = d->in_off[u + 1] - d->in_off[u]; }
}

/* Streaming bytes for expanding one parent at level i (distinct lists). */
static uint64_t parent_bytes(const plan_t *P, uint32_t i, const uint32_t *M) {
    uint64_t b = 8;
    for (uint32_t t = 0; t < P->nj[i]; ++t) {
        int dup = 0;
        for (uint32_t s = 0; s < t; ++s) {
            int same_list = P->symmetric || P->jout[i][s] == P->jout[i][t];
            if (P->jpos[i][s] == P->jpos[i][t] && same_list) { dup = 1; break; }
        }
        if (dup) continue;
        const uint32_t *l; uint64_t len;
        list_of(P, i, t, M, &l, &len);
        b += 4 * len + 8;
    }
    return b;
}

static void emit(const plan_t *P, acc_t *A, const uint32_t *M) {
    uint32_t by_q[OR_MAX_QUERY];
    for (uint32_t j = 0; j < P->k; ++j) by_q[A->order[j]] = M[j];
    A->cb(by_q, P->k, A->user);
}

static uint64_t lower_bound_u32(const uint32_t *a, uint64_t len, uint32_t x) {
    uint64_t lo = 0, hi = len;
    while (lo < hi) {
        uint64_t m = lo + (hi - lo) / 2;
        if (a[m] < x) lo = m + 1; else hi = m;
    }
    return lo;
}

/* Candidate window [lo, hi) of level i from the ordering conditions. */
static void cond_window(const plan_t *P, uint32_t i, const uint32_t *M, uint32_t *lo, uint32_t *hi) {
    uint32_t a = 0, b = UINT32_MAX;
    for (uint32_t j = 0; j < i; ++j) {
        if (((P->gt[i] >> j) & 1u) && M[j] + 1 > a) a = M[j] + 1;
        if (((P->lt[i] >> j) & 1u) && M[j] < b) b = M[j];
    }
    *lo = a; *hi = b;
}

/* Expand the partial match M[0..i-1] at level i. */
static void extend(const plan_t *P, acc_t *A, uint32_t i, uint32_t *M) {
    A->bytes += parent_bytes(P, i, M);
    uint32_t nj = P->nj[i];
    /* smallest joined list (device_funcs.cu:233-266) */
    uint32_t best = 0; uint64_t blen = UINT64_MAX; const uint32_t *bl = NULL;
    for (uint32_t t = 0; t < nj; ++t) {
        const uint32_t *l; uint64_t len;
        list_of(P, i, t, M, &l, &len);
        if (len < blen) { blen = len; best = t; bl = l; }
    }
    uint32_t lo = 0, hi = UINT32_MAX;
    if (P->gt[i] | P->lt[i]) cond_window(P, i, M, &lo, &hi);
    if (P->closed_last && i + 1 == P->k && P->last_single && P->last_loop_free && !A->cb) {
        /* one list, every query neighbour of the last vertex already
         * matched: each list element in the window that is not matched yet
         * extends (the joins imply the signature) */
        uint64_t s0 = lo ? lower_bound_u32(bl, blen, lo) : 0;
        uint64_t e0 = hi != UINT32_MAX ? lower_bound_u32(bl, blen, hi) : blen;
        if (e0 > s0) {
            uint64_t c = e0 - s0;
            for (uint32_t j = 0; j < i; ++j)
                if (M[j] >= lo && M[j] < hi && bsearch_u32(bl, 0, blen, M[j])) --c;
            A->lvl[i] += c;
        }
        return;
    }
    for (uint64_t x = 0; x < blen; ++x) {
        uint32_t c = bl[x];
        if (c < lo) continue;
        if (c >= hi) break;
        int used = 0;
        for (uint32_t j = 0; j < i; ++j) if (M[j] == c) { used = 1; break; }
        if (used || !sig_ok(P, i, c)) continue;
        int ok = 1;
        for (uint32_t t = 0; t < nj && ok; ++t) {
            if (t == best) continue;
            const uint32_t *l; uint64_t len;
            list_of(P, i, t, M, &l, &len);
            ok = bsearch_u32(l, 0, len, c);
        }
        if (!ok) continue;
        A->lvl[i]++;
        M[i] = c;
        if (i + 1 < P->k) extend(P, A, i + 1, M);
        else if (A->cb) emit(P, A, M);
    }
}

static int make_plan(const or_graph *d, const or_graph *q, const uint32_t *order_in,
                     plan_t *P, uint32_t *order) {
    uint32_t k = q->n;
    if (k == 0 || k > OR_MAX_QUERY) return OR_ERR_QUERY;
    uint32_t p_off[OR_MAX_QUERY + 1], c_off[OR_MAX_QUERY + 1];
    uint32_t p[OR_MAX_QUERY * OR_MAX_QUERY], c[OR_MAX_QUERY * OR_MAX_QUERY];
    if (order_in) {
        char seen[OR_MAX_QUERY] = {0};
        for (uint32_t i = 0; i < k; ++i) {
            if (order_in[i] >= k || seen[order_in[i]]) return OR_ERR_QUERY;
            seen[order_in[i]] = 1;
            order[i] = order_in[i];
        }
        or_joins_for_order(q, order, p_off, p, c_off, c);
    } else {
        or_order(q, order, p_off, p, c_off, c);
    }
    memset(P, 0, sizeof(*P));
    P->d = d;
    P->k = k;
    P->symmetric = or_is_symmetric(d);
    for (uint32_t i = 0; i < k; ++i) {
        uint32_t v = order[i];
        P->qin[i] = (uint32_t)(q->in_off[v + 1] - q->in_off[v]);
        P->qout[i] = (uint32_t)(q->out_off[v + 1] - q->out_off[v]);
        uint32_t n = 0;
        for (uint32_t a = p_off[i]; a < p_off[i + 1]; ++a) { P->jpos[i][n] = p[a]; P->jout[i][n] = 1; n++; }
        for (uint32_t a = c_off[i]; a < c_off[i + 1]; ++a) { P->jpos[i][n] = c[a]; P->jout[i][n] = 0; n++; }
        P->nj[i] = n;
        /* a level with no join has undefined behaviour in the reference
         * (device_funcs.cu:233-266 reads an unset join); only reachable
         * for disconnected queries, which the oracle rejects */
        if (i > 0 && n == 0) return OR_ERR_QUERY;
    }
    {
        uint32_t i = k - 1, v = order[i];
        P->last_single = k >= 2;
        for (uint32_t t = 1; t < P->nj[i]; ++t) {
            int same = P->jpos[i][t] == P->jpos[i][0] && (P->symmetric || P->jout[i][t] == P->jout[i][0]);
            if (!same) P->last_single = 0;
        }
        P->last_loop_free = !lin_has(v, q->out_adj, q->out_off[v], q->out_off[v + 1]);
    }
    return OR_OK;
}

static int count_impl(const or_graph *d, const or_graph *q, const uint32_t *order_in,
                      uint32_t root_begin, uint32_t root_end, uint32_t shard, uint32_t nshards,
                      const uint32_t *conds, uint32_t ncond, uint32_t opts,
                      int nthreads, uint64_t *count, uint64_t *level_sizes, uint64_t *alg_bytes);

int or_count(const or_graph *d, const or_graph *q, const uint32_t *order_in,
             uint32_t root_begin, uint32_t root_end, int nthreads,
             uint64_t *count, uint64_t *level_sizes, uint64_t *alg_bytes) {
    return count_impl(d, q, order_in, root_begin, root_end, 0, 1, NULL, 0, 0, nthreads, count,
                      level_sizes, alg_bytes);
}

int or_count_striped(const or_graph *d, const or_graph *q, const uint32_t *order,
                     uint32_t shard, uint32_t nshards, int nthreads, uint64_t *count,
                     uint64_t *level_sizes) {
    if (nshards == 0 || shard >= nshards) return OR_ERR_QUERY;
    return count_impl(d, q, order, 0, UINT32_MAX, shard, nshards, NULL, 0, 0, nthreads, count,
                      level_sizes, NULL);
}

int or_count_ex(const or_graph *d, const or_graph *q, const uint32_t *order,
                const uint32_t *conds, uint32_t ncond, uint32_t shard, uint32_t nshards,
                uint32_t opts, int nthreads, uint64_t *count, uint64_t *level_sizes) {
    if (nshards == 0 || shard >= nshards) return OR_ERR_QUERY;
    if (ncond && !conds) return OR_ERR_QUERY;
    return count_impl(d, q, order, 0, UINT32_MAX, shard, nshards, conds, ncond, opts, nthreads,
                      count, level_sizes, NULL);
}

static int count_impl(const or_graph *d, const or_graph *q, const uint32_t *order_in,
                      uint32_t root_begin, uint32_t root_end, uint32_t shard, uint32_t nshards,
                      const uint32_t *conds, uint32_t ncond, uint32_t opts,
                      int nthreads, uint64_t *count, uint64_t *level_sizes, uint64_t *alg_bytes) {
    plan_t P;
    uint32_t order[OR_MAX_QUERY];
    int rc = make_plan(d, q, order_in, &P, order);
    if (rc) return rc;
    uint32_t k = P.k;
    for (uint32_t c = 0; c < ncond; ++c) {  /* M[a] < M[b], checked at the later position */
        uint32_t a = conds[2 * c], b = conds[2 * c + 1];
        if (a >= k || b >= k || a == b) return OR_ERR_QUERY;
        if (a < b) P.gt[b] |= 1u << a; else P.lt[a] |= 1u << b;
    }
    P.closed_last = (opts & OR_OPT_CLOSED_LAST) != 0;
    /* level 0 (device_funcs.cu:267-279), in vertex-id order */
    uint32_t *roots = (uint32_t *)malloc(((size_t)d->n + 1) * sizeof(uint32_t));
    if (!roots) return OR_ERR_NOMEM;
    uint64_t nr = 0;
    for (uint32_t u = 0; u < d->n; ++u)
        if (u % nshards == shard && sig_ok(&P, 0, u)) roots[nr++] = u;
    uint64_t rb = root_begin < nr ? root_begin : nr;
    uint64_t re = root_end < nr ? root_end : nr;
    uint64_t lvl[OR_MAX_QUERY] = {0};
    uint64_t bytes = 8ull * d->n + 4ull * (re - rb);
    lvl[0] = re - rb;
    if (k >= 2) {
#ifdef _OPENMP
        if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
        uint64_t nroots = re - rb;
        #pragma omp parallel
        {
            acc_t A;
            memset(&A, 0, sizeof(A));
            uint32_t M[OR_MAX_QUERY];
            /* one task per root, handed out dynamically so hub roots do
               not serialise a static partition */
            #pragma omp for schedule(dynamic, 1) nowait
            for (uint64_t r = 0; r < nroots; ++r) {
                M[0] = roots[rb + r];
                extend(&P, &A, 1, M);
            }
            #pragma omp critical
            {
                for (uint32_t i = 1; i < k; ++i) lvl[i] += A.lvl[i];
                bytes += A.bytes;
            }
        }
        for (uint32_t i = 1; i + 1 < k; ++i) bytes += 8 * lvl[i];
    }
    free(roots);
    /* a 1-vertex query reports 0: the count is only added at iter == k-1 >= 1 */
    if (count) *count = k >= 2 ? lvl[k - 1] : 0;
    if (level_sizes) for (uint32_t i = 0; i < k; ++i) level_sizes[i] = lvl[i];
    if (alg_bytes) *alg_bytes = bytes;
    return OR_OK;
}

int or_enumerate(const or_graph *d, const or_graph *q, const uint32_t *order_in,
                 or_match_cb cb, void *user) {
    plan_t P;
    uint32_t order[OR_MAX_QUERY];
    int rc = make_plan(d, q, order_in, &P, order);
    if (rc) return rc;
    if (P.k < 2) return OR_OK;
    acc_t A;
    memset(&A, 0, sizeof(A));
    A.cb = cb; A.user = user; A.order = order;
    uint32_t M[OR_MAX_QUERY];
    for (uint32_t u = 0; u < d->n; ++u) {
        if (!sig_ok(&P, 0, u)) continue;
        M[0] = u;
        extend(&P, &A, 1, M);
    }
    return OR_OK;
}

/* ------------------------------------------------------------------ */
/* seeded Chung-Lu generator and degree relabelling                    */
/* ------------------------------------------------------------------ */

/* splitmix64 (Steele, Lea & Flood 2014) */
static uint64_t sm64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

static double unit_open(uint64_t h) { return (double)((h >> 11) + 1) * (1.0 / 9007199254740993.0); }

typedef struct {
    float *prob;
    uint32_t *alias;
    uint32_t n;
} alias_t;

/* Vose's alias method over weights w[0..n) (double arithmetic, float
 * probabilities, LIFO work lists). */
static int alias_build(const double *w, uint32_t n, alias_t *A) {
    A->n = n;
    A->prob = (float *)calloc(n, sizeof(float));
    A->alias = (uint32_t *)calloc(n, sizeof(uint32_t));
    double *sc = (double *)malloc((size_t)n * sizeof(double));
    uint32_t *small = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
    uint32_t *large = (uint32_t *)malloc((size_t)n * sizeof(uint32_t));
    if (!A->prob || !A->alias || !sc || !small || !large) {
        free(A->prob); free(A->alias); free(sc); free(small); free(large);
        return OR_ERR_NOMEM;
    }
    double sum = 0;
    for (uint32_t i = 0; i < n; ++i) sum += w[i];
    uint32_t ns = 0, nl = 0;
    for (uint32_t i = 0; i < n; ++i) {
        sc[i] = w[i] * n / sum;
        if (sc[i] < 1.0) small[ns++] = i; else large[nl++] = i;
    }
    while (ns && nl) {
        uint32_t s = small[--ns], l = large[nl - 1];
        A->prob[s] = (float)sc[s];
        A->alias[s] = l;
        sc[l] = (sc[l] + sc[s]) - 1.0;
        if (sc[l] < 1.0) { --nl; small[ns++] = l; }
    }
    for (uint32_t i = 0; i < nl; ++i) { A->prob[large[i]] = 1.f; A->alias[large[i]] = large[i]; }
    for (uint32_t i = 0; i < ns; ++i) { A->prob[small[i]] = 1.f; A->alias[small[i]] = small[i]; }
    free(sc); free(small); free(large);
    return OR_OK;
}

static uint32_t alias_draw(const alias_t *A, uint64_t h) {
    uint32_t col = (uint32_t)(((h >> 32) * (uint64_t)A->n) >> 32);
    float coin = (float)(uint32_t)h * (1.0f / 4294967296.0f);
    return coin < A->prob[col] ? col : A->alias[col];
}

int or_gen_chung_lu(uint32_t n, uint64_t m, double gamma, double wmin, double cap,
                    uint64_t seed, or_graph *g) {
    memset(g, 0, sizeof(*g));
    if (n < 2 || gamma <= 1.0 || wmin <= 0) return OR_ERR_QUERY;
    if (m > (uint64_t)n * (n - 1) / 2) return OR_ERR_QUERY;
    const uint64_t ws = sm64(seed ^ 0x574549474854ull), es = sm64(seed ^ 0x45444745ull);
    double *w = (double *)malloc((size_t)n * sizeof(double));
    if (!w) return OR_ERR_NOMEM;
    const double ex = -1.0 / (gamma - 1.0);
    for (uint32_t i = 0; i < n; ++i) {
        double x = wmin * pow(unit_open(sm64(ws + (uint64_t)i)), ex);
        w[i] = x < cap ? x : cap;
    }
    alias_t A;
    int rc = alias_build(w, n, &A);
    free(w);
    if (rc) return rc;
    /* the first m distinct non-loop pairs of the stream t = 0, 1, 2, ...
     * (open-addressing set of packed pairs; 0 never occurs: it is a loop) */
    uint64_t cap_h = 1;
    while (cap_h < 2 * m + 16) cap_h <<= 1;
    uint64_t *set = (uint64_t *)calloc((size_t)cap_h, sizeof(uint64_t));
    uint32_t *src = (uint32_t *)malloc((size_t)(2 * m + 1) * sizeof(uint32_t));
    uint32_t *dst = (uint32_t *)malloc((size_t)(2 * m + 1) * sizeof(uint32_t));
    if (!set || !src || !dst) {
        free(set); free(src); free(dst); free(A.prob); free(A.alias);
        return OR_ERR_NOMEM;
    }
    uint64_t have = 0;
    for (uint64_t t = 0; have < m; ++t) {
        uint32_t a = alias_draw(&A, sm64(es + 2 * t));
        uint32_t b = alias_draw(&A, sm64(es + 2 * t + 1));
        if (a == b) continue;
        if (a > b) { uint32_t x = a; a = b; b = x; }
        uint64_t key = ((uint64_t)a << 32) | b;
        uint64_t hsh = sm64(key) & (cap_h - 1);
        while (set[hsh] && set[hsh] != key) hsh = (hsh + 1) & (cap_h - 1);
        if (set[hsh]) continue;
        set[hsh] = key;
        src[2 * have] = a; dst[2 * have] = b;
        src[2 * have + 1] = b; dst[2 * have + 1] = a;
        ++have;
    }
    free(set); free(A.prob); free(A.alias);
    rc = or_graph_from_arcs(n, 2 * m, src, dst, g);
    free(src); free(dst);
    return rc;
}

int or_relabel_by_degree(const or_graph *g, or_graph *out, uint32_t *orig) {
    memset(out, 0, sizeof(*out));
    const uint32_t n = g->n;
    const int sym = or_is_symmetric(g);
    uint64_t *key = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    uint32_t *rank = (uint32_t *)malloc(((size_t)n + 1) * sizeof(uint32_t));
    uint32_t *src = (uint32_t *)malloc((size_t)(g->arcs + 1) * sizeof(uint32_t));
    uint32_t *dst = (uint32_t *)malloc((size_t)(g->arcs + 1) * sizeof(uint32_t));
    if (!key || !rank || !src || !dst) { free(key); free(rank); free(src); free(dst); return OR_ERR_NOMEM; }
    for (uint32_t v = 0; v < n; ++v) {
        uint64_t d = g->out_off[v + 1] - g->out_off[v];
        if (!sym) d += g->in_off[v + 1] - g->in_off[v];
        key[v] = (d << 32) | v;
    }
    qsort(key, n, sizeof(uint64_t), cmp_u64);
    for (uint32_t r = 0; r < n; ++r) {
        uint32_t v = (uint32_t)(key[r] & 0xffffffffu);
        rank[v] = r;
        if (orig) orig[r] = v;
    }
    uint64_t a = 0;
    for (uint32_t v = 0; v < n; ++v)
        for (uint64_t i = g->out_off[v]; i < g->out_off[v + 1]; ++i) {
            src[a] = rank[v];
            dst[a] = rank[g->out_adj[i]];
            ++a;
        }
    int rc = or_graph_from_arcs(n, a, src, dst, out);
    free(key); free(rank); free(src); free(dst);
    return rc;
}
