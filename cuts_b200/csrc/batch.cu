// batch.cu -- many queries against one resident graph in one persistent
// launch, captured in a CUDA graph.
//
// Work is a flat space of tasks, query-major: a task is (query q, root u,
// range r of u's level-1 candidate list).  Roots are the data vertices in
// out-degree order, so every query's root level is a prefix of one sorted
// array, and a per-graph prefix sum of ceil(len / grain) turns a task index
// into (u, r) with two binary searches -- nothing per query is materialised.
// Warps take tasks from one global counter (work stealing across all SMs)
// and run the query's levels depth-first from the task's level-1 range,
// with a 32-candidate frontier per level in shared memory: the trie is
// walked, never stored, so a batch needs no trie arena.  Each level step is
// the same warp-cooperative join as the level kernels: candidates from the
// shortest joined list, one per lane, lower-bound membership in the other
// lists, ballot/popc compaction.  Counts accumulate per warp and are added
// to the query's counter when the warp moves on.  A device-clock budget
// stops the launch cleanly: tasks not finished mark their query incomplete.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "batch.hpp"
#include "device_util.cuh"

namespace cuts {

#define BCK(call)                                                                      \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return set_error(CUTS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace {

constexpr int kBW = 8;  // warps per block

struct BWarp {  // per-warp depth-first state, shared memory
    uint32_t m[kBatchMaxK];
    uint32_t moff[kBatchMaxK], mdeg[kBatchMaxK], x[kBatchMaxK], xend[kBatchMaxK];
    uint32_t nb[kBatchMaxK], bi[kBatchMaxK], tmin[kBatchMaxK], nj[kBatchMaxK];
    uint32_t joff[kBatchMaxK][kBatchMaxJ], jdeg[kBatchMaxK][kBatchMaxJ];
    uint32_t buf[kBatchMaxK][32];
};

struct Ctx {
    DevView g;
    const BQuery *Q;
    BWarp *S;
    int lane;
};

// Joined lists of level d for the current prefix; the shortest feeds the
// candidates, restricted to the symmetry window.  Warp-uniform.
__device__ void enter_level(const Ctx &c, uint32_t d) {
    const BLevel &L = c.Q->lv[d];
    const uint32_t nj = L.nj;
    uint32_t my_deg = kFullMask, my_off = 0;
    if (uint32_t(c.lane) < nj) {
        const uint32_t u = c.S->m[L.jpos[c.lane]];
        const uint2 inf = L.jdir[c.lane] ? c.g.in_info[u] : c.g.out_info[u];
        my_off = inf.x;
        my_deg = inf.y;
        c.S->joff[d][c.lane] = my_off;
        c.S->jdeg[d][c.lane] = my_deg;
    }
    uint32_t bd = my_deg, bl = uint32_t(c.lane);
    #pragma unroll
    for (int s = 16; s; s >>= 1) {
        const uint32_t od = __shfl_xor_sync(kFullMask, bd, s), ol = __shfl_xor_sync(kFullMask, bl, s);
        if (od < bd || (od == bd && ol < bl)) { bd = od; bl = ol; }
    }
    const uint32_t moff = __shfl_sync(kFullMask, my_off, int(bl));
    uint32_t lo = 0, hi = kFullMask;
    for (uint32_t msk = L.gt_mask; msk; msk &= msk - 1) lo = max(lo, c.S->m[__ffs(msk) - 1] + 1);
    for (uint32_t msk = L.lt_mask; msk; msk &= msk - 1) hi = min(hi, c.S->m[__ffs(msk) - 1]);
    const uint32_t *lst = c.g.adj + moff;
    const uint32_t s0 = (lo && nj) ? lbound(lst, bd, lo) : 0;
    const uint32_t e0 = nj ? (hi != kFullMask ? lbound(lst, bd, hi) : bd) : 0;
    __syncwarp();
    if (c.lane == 0) {
        c.S->moff[d] = moff;
        c.S->mdeg[d] = nj ? bd : 0;
        c.S->tmin[d] = bl;
        c.S->nj[d] = nj;
        c.S->x[d] = s0;
        c.S->xend[d] = max(s0, e0);
        c.S->nb[d] = 0;
        c.S->bi[d] = 0;
    }
    __syncwarp();
}

// Lane test of candidate list element idx at level d.
__device__ __forceinline__ bool test_candidate(const Ctx &c, uint32_t d, uint32_t idx, uint32_t &cand) {
    const BLevel &L = c.Q->lv[d];
    bool ok = idx < c.S->xend[d];
    const uint32_t v = ok ? __ldg(c.g.adj + c.S->moff[d] + idx) : 0;
    if (ok)
        for (uint32_t j = 0; j < d; ++j)
            if (v == c.S->m[j]) { ok = false; break; }
    if (ok && L.check_sig) {
        const uint2 o = c.g.out_info[v], i = c.g.in_info[v];
        ok = i.y >= L.qin && o.y >= L.qout;
    }
    if (ok) {
        const uint32_t nj = c.S->nj[d], tm = c.S->tmin[d];
        for (uint32_t t = 0; t < nj; ++t) {
            if (t == tm) continue;
            if (!contains(c.g.adj + c.S->joff[d][t], c.S->jdeg[d][t], v)) { ok = false; break; }
        }
    }
    cand = v;
    return ok;
}

// Candidates of level d in [x, xend), counted (the last level).
__device__ unsigned long long count_level(const Ctx &c, uint32_t d) {
    const BLevel &L = c.Q->lv[d];
    const uint32_t s0 = c.S->x[d], e0 = c.S->xend[d];
    if (s0 >= e0) return 0;
    if (L.closed_form && c.S->nj[d] == 1) {
        // one list, no signature: the window minus the matched vertices in it
        const uint32_t *lst = c.g.adj + c.S->moff[d];
        const uint32_t mdeg = c.S->mdeg[d];
        bool hit = false;
        if (uint32_t(c.lane) < d) {
            const uint32_t mj = c.S->m[c.lane];
            if ((L.guar_mask >> c.lane) & 1u) {
                // the query's own arc puts m_j in the list: only the window decides
                const uint32_t lo = s0 ? __ldg(lst + s0 - 1) : 0;  // window by position
                hit = (s0 == 0 || mj > lo) && (e0 >= mdeg || mj < __ldg(lst + e0));
            } else {
                const uint32_t p = lbound(lst, mdeg, mj);
                hit = p >= s0 && p < e0 && p < mdeg && __ldg(lst + p) == mj;
            }
        }
        return (e0 - s0) - __popc(__ballot_sync(kFullMask, hit));
    }
    unsigned long long n = 0;
    for (uint32_t x0 = s0; x0 < e0; x0 += 32) {
        uint32_t v;
        const bool ok = test_candidate(c, d, x0 + c.lane, v);
        n += __popc(__ballot_sync(kFullMask, ok));
    }
    return n;
}

// Level d = k-2 counted together with level k-1 (the plan folded them): each
// candidate c of level d adds the last level's closed form, the window of the
// last level's list minus the matched vertices in it, c included.
__device__ unsigned long long count_level_fold(const Ctx &c, uint32_t d) {
    const BLevel &F = c.Q->lv[d + 1];
    const uint32_t s0 = c.S->x[d], e0 = c.S->xend[d];
    if (s0 >= e0) return 0;
    const uint32_t u = c.S->m[F.jpos[0]];
    const uint2 inf = F.jdir[0] ? c.g.in_info[u] : c.g.out_info[u];
    uint32_t lo = 0, hi = kFullMask;
    for (uint32_t msk = F.gt_mask; msk; msk &= msk - 1) lo = max(lo, c.S->m[__ffs(msk) - 1] + 1);
    for (uint32_t msk = F.lt_mask; msk; msk &= msk - 1) hi = min(hi, c.S->m[__ffs(msk) - 1]);
    const uint32_t *fl = c.g.adj + inf.x;
    const uint32_t ws = lo ? lbound(fl, inf.y, lo) : 0;
    const uint32_t we = hi != kFullMask ? lbound(fl, inf.y, hi) : inf.y;
    bool hit = false;
    if (uint32_t(c.lane) < d) {
        const uint32_t mj = c.S->m[c.lane];
        hit = mj >= lo && mj < hi && (((F.guar_mask >> c.lane) & 1u) || contains(fl, inf.y, mj));
    }
    const uint32_t base = (we > ws ? we - ws : 0) - __popc(__ballot_sync(kFullMask, hit));
    const bool guar_c = (F.guar_mask >> d) & 1u;
    unsigned long long n = 0;
    for (uint32_t x0 = s0; x0 < e0; x0 += 32) {
        uint32_t v;
        const bool ok = test_candidate(c, d, x0 + c.lane, v);
        uint32_t add = 0;
        if (ok) {
            const bool h2 = v >= lo && v < hi && (guar_c || contains(fl, inf.y, v));
            add = base - (h2 ? 1u : 0u);
        }
        #pragma unroll
        for (int o = 16; o; o >>= 1) add += __shfl_xor_sync(kFullMask, add, o);
        n += add;
    }
    return n;
}

// Next up-to-32 candidates of level d into its frontier buffer.
__device__ void refill(const Ctx &c, uint32_t d) {
    uint32_t v;
    const bool ok = test_candidate(c, d, c.S->x[d] + c.lane, v);
    const unsigned m = __ballot_sync(kFullMask, ok);
    if (ok) c.S->buf[d][__popc(m & ((1u << c.lane) - 1))] = v;
    __syncwarp();
    if (c.lane == 0) {
        c.S->x[d] += 32;
        c.S->nb[d] = __popc(m);
        c.S->bi[d] = 0;
    }
    __syncwarp();
}

__global__ void __launch_bounds__(kBW * 32)
k_batch(DevView g, const BQuery *__restrict__ qs, uint32_t nq,
        const unsigned long long *__restrict__ qbase, const uint32_t *__restrict__ vsorted,
        const unsigned long long *__restrict__ pref0, const unsigned long long *__restrict__ pref1,
        const unsigned long long *__restrict__ pref2, uint32_t grain, uint32_t tgrab,
        unsigned long long *__restrict__ task_ctr, uint32_t *__restrict__ stop,
        unsigned long long *__restrict__ counts, uint32_t *__restrict__ aborted,
        unsigned long long budget_ns, unsigned long long *__restrict__ qtime,
        unsigned long long qlimit, uint32_t shard, uint32_t nshards) {
    __shared__ BWarp ws[kBW];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Ctx c{g, nullptr, &ws[warp], lane};
    const unsigned long long total = qbase[nq];
    // this shard's tasks are t = c * nshards + shard for counter values c
    const unsigned long long ctotal = total > shard ? (total - shard + nshards - 1) / nshards : 0;
    const unsigned long long deadline = budget_ns ? global_ns() + budget_ns : ~0ull;
    uint32_t cur = kFullMask;
    unsigned long long qcount = 0;
    volatile uint32_t *vstop = stop;

    while (true) {
        unsigned long long c0 = 0;
        if (lane == 0) c0 = *vstop ? ctotal : atomicAdd(task_ctr, (unsigned long long)tgrab);
        c0 = __shfl_sync(kFullMask, c0, 0);
        if (c0 >= ctotal) break;
        const unsigned long long c1 = min(c0 + tgrab, ctotal);
        for (unsigned long long cc = c0; cc < c1; ++cc) {
            const unsigned long long t = cc * nshards + shard;
            if (cur == kFullMask || t < qbase[cur] || t >= qbase[cur + 1]) {
                if (cur != kFullMask && lane == 0 && qcount) atomicAdd(&counts[cur], qcount);
                qcount = 0;
                uint32_t lo = 0, hi = nq - 1;  // last q with qbase[q] <= t
                while (lo < hi) {
                    const uint32_t mid = (lo + hi + 1) >> 1;
                    if (qbase[mid] <= t) lo = mid; else hi = mid - 1;
                }
                cur = lo;
                c.Q = qs + cur;
            }
            if (*vstop || global_ns() > deadline) {
                if (lane == 0) { atomicOr(stop, 1u); aborted[cur] = 1; }
                continue;
            }
            // per-query limit: a query past its share of warp time is dropped,
            // and the work counter skips the rest of its tasks
            if (qlimit) {
                uint32_t skip = 0;
                if (lane == 0) {
                    skip = reinterpret_cast<volatile uint32_t *>(aborted)[cur] ||
                           reinterpret_cast<volatile unsigned long long *>(qtime)[cur] > qlimit;
                    if (skip) {
                        aborted[cur] = 1;
                        const unsigned long long e = qbase[cur + 1];
                        atomicMax(task_ctr, e > shard ? (e - shard + nshards - 1) / nshards : 0ull);
                    }
                }
                if (__shfl_sync(kFullMask, skip, 0)) continue;
            }
            const unsigned long long task_start = qlimit ? global_ns() : 0;
            const BQuery &Q = *c.Q;
            const unsigned long long local = t - qbase[cur];
            const unsigned long long *pref = Q.type == 0 ? pref0 : (Q.type == 1 ? pref1 : pref2);
            uint32_t lo = 0, hi = Q.root_cnt - 1;  // root: last j with pref[j] <= local
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (pref[mid] <= local) lo = mid; else hi = mid - 1;
            }
            const uint32_t u = vsorted[lo];
            const uint32_t r = uint32_t(local - pref[lo]);
            const uint2 uo = g.out_info[u], ui = g.in_info[u];
            if (ui.y < Q.lv[0].qin || uo.y < Q.lv[0].qout) continue;  // level-0 signature
            if (lane == 0) c.S->m[0] = u;
            __syncwarp();
            // level 1: joins all on position 0; the task fixes the list and range
            enter_level(c, 1);
            {
                // the task space was cut on the type's list (out, in or the
                // shorter): make that list the candidate source
                const bool use_in = Q.type == 1 || (Q.type == 2 && ui.y < uo.y);
                const uint2 L1 = use_in ? ui : uo;
                uint32_t tm = 0;
                for (uint32_t t2 = 0; t2 < Q.lv[1].nj; ++t2)
                    if ((Q.lv[1].jdir[t2] != 0) == use_in) { tm = t2; break; }
                const uint32_t *lst = g.adj + L1.x;
                uint32_t lo1 = 0, hi1 = kFullMask;
                if (Q.lv[1].gt_mask) lo1 = u + 1;
                if (Q.lv[1].lt_mask) hi1 = u;
                const uint32_t s0 = lo1 ? lbound(lst, L1.y, lo1) : 0;
                const uint32_t e0 = hi1 != kFullMask ? lbound(lst, L1.y, hi1) : L1.y;
                const uint32_t xs = max(s0, min(r * grain, L1.y));
                const uint32_t xe = min(e0, min(r * grain + grain, L1.y));
                __syncwarp();
                if (lane == 0) {
                    c.S->moff[1] = L1.x;
                    c.S->mdeg[1] = L1.y;
                    c.S->tmin[1] = tm;
                    c.S->x[1] = xs;
                    c.S->xend[1] = max(xs, xe);
                }
                __syncwarp();
            }
            if (Q.k == 2) {
                qcount += count_level(c, 1);
                continue;
            }
            if (Q.k == 3 && Q.lv[1].fold) {
                qcount += count_level_fold(c, 1);
                continue;
            }
            // depth-first over levels 1..k-2, counting level k-1
            uint32_t d = 1;
            bool abandoned = false, dropped = false;
            while (d >= 1) {
                if (c.S->bi[d] < c.S->nb[d]) {
                    const uint32_t v = c.S->buf[d][c.S->bi[d]];
                    __syncwarp();
                    if (lane == 0) {
                        c.S->bi[d]++;
                        c.S->m[d] = v;
                    }
                    __syncwarp();
                    enter_level(c, d + 1);
                    if (d + 2 == Q.k) qcount += count_level(c, d + 1);
                    else if (d + 3 == Q.k && Q.lv[d + 1].fold) qcount += count_level_fold(c, d + 1);
                    else ++d;
                } else if (c.S->x[d] < c.S->xend[d]) {
                    const unsigned long long now = global_ns();
                    if (*vstop || now > deadline) { abandoned = true; break; }
                    if (qlimit && reinterpret_cast<volatile unsigned long long *>(qtime)[cur] +
                                          (now - task_start) > qlimit) {
                        dropped = true;
                        break;
                    }
                    refill(c, d);
                } else {
                    --d;
                }
            }
            if (abandoned && lane == 0) {
                atomicOr(stop, 1u);
                aborted[cur] = 1;
            }
            if (qlimit && lane == 0) {
                atomicAdd(&qtime[cur], global_ns() - task_start);
                if (dropped) aborted[cur] = 1;
            }
        }
    }
    if (cur != kFullMask && lane == 0 && qcount) atomicAdd(&counts[cur], qcount);
}

}  // namespace

// ---- host ---------------------------------------------------------------------

int batch_prepare_graph(DeviceGraph &g, uint32_t grain) {
    if (g.batch_vsorted && g.batch_grain == grain) return CUTS_OK;
    const uint32_t n = g.n;
    std::vector<uint32_t> vs(n);
    std::iota(vs.begin(), vs.end(), 0u);
    std::stable_sort(vs.begin(), vs.end(),
                     [&](uint32_t a, uint32_t b) { return g.h_out_deg[a] > g.h_out_deg[b]; });
    const int types = g.symmetric ? 1 : 3;
    std::vector<unsigned long long> pref(size_t(types) * (n + 1), 0);
    for (int t = 0; t < types; ++t) {
        unsigned long long *p = pref.data() + size_t(t) * (n + 1);
        for (uint32_t j = 0; j < n; ++j) {
            const uint32_t v = vs[j];
            const uint32_t len = t == 0 ? g.h_out_deg[v]
                                        : (t == 1 ? g.h_in_deg[v] : std::min(g.h_out_deg[v], g.h_in_deg[v]));
            p[j + 1] = p[j] + std::max<uint32_t>(1, (len + grain - 1) / grain);
        }
    }
    cudaFree(g.batch_vsorted);
    cudaFree(g.batch_pref);
    g.batch_vsorted = nullptr;
    g.batch_pref = nullptr;
    BCK(cudaMalloc(&g.batch_vsorted, sizeof(uint32_t) * std::max<uint32_t>(n, 1)));
    BCK(cudaMalloc(&g.batch_pref, sizeof(unsigned long long) * pref.size()));
    BCK(cudaMemcpy(g.batch_vsorted, vs.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
    BCK(cudaMemcpy(g.batch_pref, pref.data(), sizeof(unsigned long long) * pref.size(), cudaMemcpyHostToDevice));
    g.batch_grain = grain;
    g.batch_pref_host.swap(pref);
    return CUTS_OK;
}

void Batch::destroy() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cudaFree(d_queries);
    cudaFree(d_qbase);
    cudaFree(d_counts);
    cudaFree(d_aborted);
    cudaFree(d_qtime);
    cudaFree(d_ctr);
    cudaFreeHost(h_counts);
    cudaFreeHost(h_aborted);
    cudaFreeHost(h_ctr);
    exec = nullptr;
    graph = nullptr;
    d_queries = nullptr;
    d_qbase = nullptr;
    d_counts = nullptr;
    d_aborted = nullptr;
    d_qtime = nullptr;
    d_ctr = nullptr;
    h_counts = nullptr;
    h_aborted = nullptr;
    h_ctr = nullptr;
}

// True when the level engine's plan for q counts its last levels fused,
// orbit-folded or as a pendant pair (prepare() in engine.cu makes the same
// choices).
static bool level_engine_pays(const Query &q, bool symmetric, uint32_t flags) {
    Plan plan;
    if (build_plan(q, symmetric, flags, plan)) return false;
    const uint32_t k = q.k;
    if (k < 3) return false;
    if ((flags & CUTS_FLAG_SYMMETRY_BREAK) && plan.lv[k - 1].ofold) return true;
    if (k >= 4 && plan.lv[k - 3].fold2) return true;  // a pendant pair counted in closed form
    const uint32_t cl = plan.lv[k - 2].fold ? k - 2 : k - 1;
    return plan.lv[cl].fuse != 0 && !(flags & CUTS_FLAG_NO_FUSE);
}

int Batch::create(DeviceGraph &dg, const std::vector<const Query *> &qs, uint32_t flags_,
                  const BatchTuning &tune_) {
    g = &dg;
    flags = flags_;
    tune = tune_;
    // CUTS_BATCH_ROUTE=0 keeps every query in the persistent launch, =2 sends
    // every query of 4+ vertices to the level engine (A/B comparisons)
    const char *rt = std::getenv("CUTS_BATCH_ROUTE");
    route_level = !(rt && rt[0] == '0');
    route_all = rt && rt[0] == '2';
    if (tune.grain == 0) tune.grain = 64;
    if (tune.tasks_per_grab == 0) tune.tasks_per_grab = 1;
    BCK(cudaSetDevice(g->device));
    int rc = batch_prepare_graph(*g, tune.grain);
    if (rc) return rc;
    queries = qs;
    nq = uint32_t(qs.size());
    std::vector<BQuery> hq;
    std::vector<unsigned long long> qbase(1, 0);
    aut.assign(nq, 1);
    eligible.assign(nq, 0);
    const uint32_t n = g->n;
    for (uint32_t i = 0; i < nq; ++i) {
        const Query &q = *qs[i];
        Plan plan;
        rc = build_plan(q, g->symmetric, flags | CUTS_FLAG_NO_ORBIT_FOLD | CUTS_FLAG_NO_PAIR_FOLD, plan);  // plain fold only
        if (rc) return rc;
        aut[i] = plan.aut;
        BQuery b;
        std::memset(&b, 0, sizeof(b));
        bool ok = q.k >= 2 && q.k <= uint32_t(kBatchMaxK) && n > 0;
        for (uint32_t d = 0; ok && d < q.k; ++d) {
            const LevelPlan &L = plan.lv[d];
            if (L.nj > uint32_t(kBatchMaxJ)) { ok = false; break; }
            BLevel &B = b.lv[d];
            B.nj = L.nj;
            B.qin = L.qin;
            B.qout = L.qout;
            B.check_sig = L.check_sig;
            B.gt_mask = L.gt_mask;
            B.lt_mask = L.lt_mask;
            B.closed_form = L.closed_form;
            B.fold = L.fold;
            B.guar_mask = L.guar_mask;
            for (uint32_t t = 0; t < L.nj; ++t) {
                B.jpos[t] = L.jpos[t];
                B.jdir[t] = L.jdir[t];
            }
        }
        // queries of 4+ vertices whose counted levels the level engine fuses
        // (or, with symmetry breaking, orbit-folds) run there: its fused
        // count, dense-core rows and hub split have no counterpart in the
        // persistent kernel, which walks one candidate at a time
        if (ok && q.k >= 4 && route_level && (route_all || level_engine_pays(q, g->symmetric, flags))) ok = false;
        unsigned long long tasks = 0;
        if (ok) {
            b.k = q.k;
            bool has_out = false, has_in = false;
            for (uint32_t t = 0; t < plan.lv[1].nj; ++t) (plan.lv[1].jdir[t] ? has_in : has_out) = true;
            b.type = g->symmetric ? 0 : (has_out && has_in ? 2 : (has_in ? 1 : 0));
            const uint32_t qout0 = plan.lv[0].qout;
            b.root_cnt = qout0 < g->stats.out_ge.size() ? uint32_t(g->stats.out_ge[qout0]) : 0;
            if (b.root_cnt == 0) {
                ok = false;  // no root passes: the count is 0 without a launch
            } else {
                tasks = g->batch_pref_host[size_t(b.type) * (n + 1) + b.root_cnt];
                hq.push_back(b);
                qbase.push_back(qbase.back() + tasks);
                index.push_back(i);
            }
        }
        eligible[i] = ok ? 1 : (b.root_cnt == 0 && b.k ? 2 : 0);
    }
    // eligible: 1 = in the launch, 2 = no root (count 0), 0 = counted by the level engine
    nb = uint32_t(hq.size());
    total_tasks = qbase.back();
    BCK(cudaMalloc(&d_queries, sizeof(BQuery) * std::max<size_t>(hq.size(), 1)));
    BCK(cudaMalloc(&d_qbase, sizeof(unsigned long long) * qbase.size()));
    BCK(cudaMalloc(&d_counts, sizeof(unsigned long long) * std::max<uint32_t>(nb, 1)));
    BCK(cudaMalloc(&d_aborted, sizeof(uint32_t) * std::max<uint32_t>(nb, 1)));
    BCK(cudaMalloc(&d_qtime, sizeof(unsigned long long) * std::max<uint32_t>(nb, 1)));
    BCK(cudaMalloc(&d_ctr, sizeof(unsigned long long) * 2));
    BCK(cudaMallocHost(&h_counts, sizeof(unsigned long long) * std::max<uint32_t>(nb, 1)));
    BCK(cudaMallocHost(&h_aborted, sizeof(uint32_t) * std::max<uint32_t>(nb, 1)));
    BCK(cudaMallocHost(&h_ctr, sizeof(unsigned long long) * 2));
    if (nb) {
        BCK(cudaMemcpy(d_queries, hq.data(), sizeof(BQuery) * nb, cudaMemcpyHostToDevice));
    }
    BCK(cudaMemcpy(d_qbase, qbase.data(), sizeof(unsigned long long) * qbase.size(), cudaMemcpyHostToDevice));
    qbase_host.swap(qbase);
    return CUTS_OK;
}

int Batch::capture(unsigned long long budget_ns) {
    if (exec && budget_ns == captured_budget && query_budget_ms == captured_query_budget &&
        shard == captured_shard && nshards == captured_nshards)
        return CUTS_OK;
    if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
    if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
    int bps = 0;
    BCK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_batch, kBW * 32, 0));
    int sms = 0;
    BCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device));
    if (tune.blocks_per_sm) bps = std::min<int>(bps, int(tune.blocks_per_sm));
    const unsigned long long maxb = (total_tasks / std::max<uint32_t>(nshards, 1) + kBW) / kBW;
    const uint32_t blocks = uint32_t(std::max<unsigned long long>(1, std::min<unsigned long long>(
        (unsigned long long)(std::max(1, bps) * sms), maxb)));
    const unsigned long long *pref = g->batch_pref;
    const size_t stride = size_t(g->n) + 1;
    cudaStream_t s = g->stream;
    BCK(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(d_counts, 0, sizeof(unsigned long long) * std::max<uint32_t>(nb, 1), s);
    cudaMemsetAsync(d_aborted, 0, sizeof(uint32_t) * std::max<uint32_t>(nb, 1), s);
    cudaMemsetAsync(d_qtime, 0, sizeof(unsigned long long) * std::max<uint32_t>(nb, 1), s);
    const unsigned long long qlimit =
        query_budget_ms > 0 ? (unsigned long long)(query_budget_ms * 1e6 * double(blocks) * kBW) : 0ull;
    cudaMemsetAsync(d_ctr, 0, sizeof(unsigned long long) * 2, s);
    if (nb) {
        k_batch<<<blocks, kBW * 32, 0, s>>>(
            graph_view(*g), d_queries, nb, d_qbase, g->batch_vsorted,
            pref, g->symmetric ? pref : pref + stride, g->symmetric ? pref : pref + 2 * stride, tune.grain,
            tune.tasks_per_grab, d_ctr, reinterpret_cast<uint32_t *>(d_ctr + 1), d_counts, d_aborted,
            budget_ns, d_qtime, qlimit, shard, nshards);
    }
    cudaMemcpyAsync(h_counts, d_counts, sizeof(unsigned long long) * std::max<uint32_t>(nb, 1),
                    cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h_aborted, d_aborted, sizeof(uint32_t) * std::max<uint32_t>(nb, 1), cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h_ctr, d_ctr, sizeof(unsigned long long) * 2, cudaMemcpyDeviceToHost, s);
    cudaGraph_t gr = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(s, &gr);
    if (ce != cudaSuccess) return set_error(CUTS_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
    graph = gr;
    BCK(cudaGraphInstantiate(&exec, graph, 0));
    captured_budget = budget_ns;
    captured_query_budget = query_budget_ms;
    captured_shard = shard;
    captured_nshards = nshards;
    launch_blocks = blocks;
    return CUTS_OK;
}

int Batch::run(double budget_ms, std::vector<uint64_t> &counts, std::vector<int> &status, float *ms) {
    BCK(cudaSetDevice(g->device));
    const unsigned long long budget_ns = budget_ms > 0 ? (unsigned long long)(budget_ms * 1e6) : 0ull;
    int rc = capture(budget_ns);
    if (rc) return rc;
    counts.assign(nq, 0);
    status.assign(nq, CUTS_OK);
    BCK(cudaEventRecord(g->ev0, g->stream));
    BCK(cudaGraphLaunch(exec, g->stream));
    BCK(cudaEventRecord(g->ev1, g->stream));
    BCK(cudaStreamSynchronize(g->stream));
    float t = 0;
    BCK(cudaEventElapsedTime(&t, g->ev0, g->ev1));
    // tasks below stop_at were all taken (counter values map to c * nshards + shard)
    const unsigned long long stop_at = std::min<unsigned long long>(h_ctr[0] * nshards + shard, total_tasks);
    const bool stopped = reinterpret_cast<uint32_t *>(h_ctr + 1)[0] != 0;
    for (uint32_t b = 0; b < nb; ++b) {
        const uint32_t i = index[b];
        counts[i] = uint64_t(h_counts[b]) * aut[i];
        const bool unfinished = h_aborted[b] || (stopped && qbase_host[b + 1] > stop_at);
        if (unfinished) status[i] = CUTS_ERR_BUDGET;
    }
    // queries outside the batched kernel's limits: the level engine, one by one
    for (uint32_t i = 0; i < nq; ++i) {
        if (eligible[i] != 0) continue;
        CountResult r;
        CountOptions opt;
        opt.flags = flags;
        opt.budget_ms = query_budget_ms;
        opt.shard = shard;
        opt.nshards = nshards;
        rc = device_count(*g, *queries[i], opt, r);
        if (rc) {
            status[i] = rc;
            continue;
        }
        counts[i] = r.count;
        t += r.ms;
    }
    if (ms) *ms = t;
    return CUTS_OK;
}


// ---- allocation-free entry point ---------------------------------------------
//
// For callers that may not allocate GPU memory themselves: code running inside
// a host framework that owns every device allocation (a memory pool that must
// account for all bytes, a plugin sandbox).
// They pass the graph and the output buffer they already own; the engine's
// own scratch for this path -- the per-query plans and the work counter --
// lives in the fixed array below, which every GPU that loads this library
// holds until the process exits.
namespace {

constexpr uint32_t kNoAllocMaxQueries = 64;  // queries per call

struct NoAllocScratch {
    BQuery queries[kNoAllocMaxQueries];
    unsigned long long task_ctr;
    uint32_t stop;
    uint32_t aborted[kNoAllocMaxQueries];
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// Device address of g_noalloc_scratch per device ordinal (the host-side
// symbol is only a stand-in, never a device address), and the launch shape.
constexpr int kNoAllocMaxDevices = 64;
NoAllocScratch *g_noalloc_ptr[kNoAllocMaxDevices] = {};
uint32_t g_noalloc_blocks[kNoAllocMaxDevices] = {};
std::mutex g_noalloc_mutex;

// The query plans travel as kernel parameters, copied into the scratch array
// by a one-block kernel: the launch records them by value when it is queued,
// so the call needs no host staging buffer and returns without waiting.
constexpr uint32_t kNoAllocPlansPerLaunch = 16;  // 16 x 656 B of parameters
struct NoAllocPlans {
    BQuery q[kNoAllocPlansPerLaunch];
};

__global__ void k_noalloc_plans(const NoAllocPlans plans, uint32_t first, uint32_t count,
                                NoAllocScratch *__restrict__ sc) {
    const uint32_t words = count * uint32_t(sizeof(BQuery) / 4);
    const uint32_t *src = reinterpret_cast<const uint32_t *>(plans.q);
    uint32_t *dst = reinterpret_cast<uint32_t *>(sc->queries + first);
    for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
    // the work counter and the stop flag start at zero
    if (first == 0 && threadIdx.x == 0) {
        sc->task_ctr = 0;
        sc->stop = 0;
    }
}

// Tasks are (query, root vertex) pairs in vertex-id order, query-major; each
// runs the root's whole level-1 list depth first with the same level steps as
// k_batch.  No budget: every query runs to completion.
__global__ void __launch_bounds__(kBW * 32)
k_batch_noalloc(DevView g, NoAllocScratch *__restrict__ sc, uint32_t nq,
                unsigned long long *__restrict__ counts) {
    __shared__ BWarp ws[kBW];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Ctx c{g, nullptr, &ws[warp], lane};
    const unsigned long long total = (unsigned long long)nq * g.n;
    uint32_t cur = kFullMask;
    unsigned long long qcount = 0;
    while (true) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(&sc->task_ctr, 1ull);
        t = __shfl_sync(kFullMask, t, 0);
        if (t >= total) break;
        const uint32_t q = uint32_t(t / g.n), u = uint32_t(t % g.n);
        if (q != cur) {
            if (cur != kFullMask && lane == 0 && qcount) atomicAdd(&counts[cur], qcount);
            qcount = 0;
            cur = q;
            c.Q = sc->queries + q;
        }
        const BQuery &Q = *c.Q;
        if (Q.k < 2) continue;
        const uint2 uo = g.out_info[u], ui = g.in_info[u];
        if (ui.y < Q.lv[0].qin || uo.y < Q.lv[0].qout) continue;  // level-0 signature
        if (lane == 0) c.S->m[0] = u;
        __syncwarp();
        enter_level(c, 1);  // the whole shortest level-1 list, symmetry window applied
        if (Q.k == 2) { qcount += count_level(c, 1); continue; }
        if (Q.k == 3 && Q.lv[1].fold) { qcount += count_level_fold(c, 1); continue; }
        uint32_t d = 1;
        while (d >= 1) {
            if (c.S->bi[d] < c.S->nb[d]) {
                const uint32_t v = c.S->buf[d][c.S->bi[d]];
                __syncwarp();
                if (lane == 0) {
                    c.S->bi[d]++;
                    c.S->m[d] = v;
                }
                __syncwarp();
                enter_level(c, d + 1);
                if (d + 2 == Q.k) qcount += count_level(c, d + 1);
                else if (d + 3 == Q.k && Q.lv[d + 1].fold) qcount += count_level_fold(c, d + 1);
                else ++d;
            } else if (c.S->x[d] < c.S->xend[d]) {
                refill(c, d);
            } else {
                --d;
            }
        }
    }
    if (cur != kFullMask && lane == 0 && qcount) atomicAdd(&counts[cur], qcount);
}

}  // namespace

int count_noalloc(const uint32_t *info_out, const uint32_t *info_in, const uint32_t *adj, uint32_t n,
                  int symmetric, const Query *const *qs, uint32_t nq, uint32_t flags,
                  unsigned long long *counts, cudaStream_t stream) {
    if (!info_out || !adj || !counts || (nq && !qs))
        return set_error(CUTS_ERR_ARG, "cuts_count_noalloc: null argument");
    if (nq > kNoAllocMaxQueries)
        return set_error(CUTS_ERR_LIMIT, "cuts_count_noalloc: more than 64 queries in one call");
    if (flags & CUTS_FLAG_SYMMETRY_BREAK)
        return set_error(CUTS_ERR_ARG, "cuts_count_noalloc: symmetry breaking is not available here");
    // the query plans, built on the stack (fixed size, no allocation)
    NoAllocPlans table[kNoAllocMaxQueries / kNoAllocPlansPerLaunch];
    const bool sym = symmetric != 0 || info_in == nullptr;
    for (uint32_t i = 0; i < nq; ++i) {
        if (!qs[i]) return set_error(CUTS_ERR_ARG, "cuts_count_noalloc: null query");
        const Query &q = *qs[i];
        if (q.k > uint32_t(kBatchMaxK))
            return set_error(CUTS_ERR_LIMIT, "cuts_count_noalloc: query with more than 10 vertices");
        Plan plan;
        int rc = build_plan(q, sym, flags | CUTS_FLAG_NO_ORBIT_FOLD | CUTS_FLAG_NO_PAIR_FOLD, plan);  // plain fold only
        if (rc) return rc;
        BQuery &b = table[i / kNoAllocPlansPerLaunch].q[i % kNoAllocPlansPerLaunch];
        std::memset(&b, 0, sizeof(b));
        b.k = q.k;
        for (uint32_t d = 0; d < q.k; ++d) {
            const LevelPlan &L = plan.lv[d];
            if (L.nj > uint32_t(kBatchMaxJ))
                return set_error(CUTS_ERR_LIMIT, "cuts_count_noalloc: more than 8 joined lists at a level");
            BLevel &B = b.lv[d];
            B.nj = L.nj;
            B.qin = L.qin;
            B.qout = L.qout;
            B.check_sig = L.check_sig;
            B.gt_mask = L.gt_mask;
            B.lt_mask = L.lt_mask;
            B.closed_form = L.closed_form;
            B.fold = L.fold;
            B.guar_mask = L.guar_mask;
            for (uint32_t t = 0; t < L.nj; ++t) {
                B.jpos[t] = L.jpos[t];
                B.jdir[t] = L.jdir[t];
            }
        }
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices)
        return set_error(CUTS_ERR_CUDA, "cuts_count_noalloc: no current CUDA device");
    NoAllocScratch *sc = nullptr;
    uint32_t blocks = 0;
    {
        // once per device, with that device current: the scratch array's
        // device address and the persistent grid size
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_ptr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
                return set_error(CUTS_ERR_CUDA, "cuts_count_noalloc: cudaGetSymbolAddress failed");
            int bps = 0, sms = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_batch_noalloc, kBW * 32, 0) != cudaSuccess ||
                cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
                return set_error(CUTS_ERR_CUDA, "cuts_count_noalloc: device query failed");
            g_noalloc_blocks[dev] = uint32_t(std::max(1, bps) * std::max(1, sms));
            g_noalloc_ptr[dev] = static_cast<NoAllocScratch *>(p);
        }
        sc = g_noalloc_ptr[dev];
        blocks = g_noalloc_blocks[dev];
    }
    // nothing to count: the caller's counts buffer (nq entries) is not touched
    if (nq == 0) return CUTS_OK;
    // counts start at zero on every call
    if (cudaMemsetAsync(counts, 0, sizeof(unsigned long long) * nq, stream) != cudaSuccess)
        return set_error(CUTS_ERR_CUDA, "cuts_count_noalloc: memset failed");
    if (n == 0) return CUTS_OK;
    for (uint32_t first = 0; first < nq; first += kNoAllocPlansPerLaunch) {
        const uint32_t cnt = std::min(kNoAllocPlansPerLaunch, nq - first);
        k_noalloc_plans<<<1, 256, 0, stream>>>(table[first / kNoAllocPlansPerLaunch], first, cnt, sc);
        if (cudaGetLastError() != cudaSuccess)
            return set_error(CUTS_ERR_CUDA, "cuts_count_noalloc: plan upload failed");
    }
    const DevView view{reinterpret_cast<const uint2 *>(info_out),
                       reinterpret_cast<const uint2 *>(sym ? info_out : info_in), adj, n, nullptr, nullptr,
                       nullptr, 0};
    const unsigned long long total = (unsigned long long)nq * n;
    const uint32_t grid = uint32_t(std::min<unsigned long long>(blocks, (total + kBW - 1) / kBW));
    k_batch_noalloc<<<std::max<uint32_t>(grid, 1), kBW * 32, 0, stream>>>(view, sc, nq, counts);
    if (cudaGetLastError() != cudaSuccess)
        return set_error(CUTS_ERR_CUDA, "cuts_count_noalloc: launch failed");
    return CUTS_OK;
}

}  // namespace cuts
