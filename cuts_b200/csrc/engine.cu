// engine.cu -- device layout, level kernels and the chunked level driver.
//
// Method (the reference's, device_funcs.cu:267-405 and host_funcs.cu:
// 39-171): a vertex-at-a-time join along the matching order.  Level L_0
// holds the root candidates; level L_i holds (vertex, parent index) trie
// entries, each extending one entry of L_{i-1} by a data vertex that lies
// in every joined adjacency list, is not matched yet and passes the degree
// signature.  The last level is counted, not stored.
//
// B200 layout of the work:
//   * one warp per parent entry, parents handed out by a global work cursor
//     in grains (work stealing across all SMs of a persistent grid);
//   * the smallest joined list supplies the candidates (32 per step, one
//     per lane); membership in the other lists is a lower-bound search;
//   * survivors are placed with a warp ballot/popc into a per-warp shared
//     staging buffer and flushed with one global atomic per buffer, so the
//     next level is written in coalesced runs;
//   * each stored entry carries an upper bound on its own child count (the
//     shortest list it will join at the next level); a tile-sum + scan
//     planner cuts every level into chunks whose bound fits the level's
//     capacity, and the driver expands chunk by chunk depth-first, so the
//     trie never exceeds the arena whatever the graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cerrno>
#include <charconv>
#include <chrono>
#include <climits>
#include <cstdlib>
#include <cstdio>
#include <memory>
#include <cstring>
#include <string>
#include <vector>

#include <omp.h>

#include "device_util.cuh"
#include "engine.hpp"

namespace cuts {

#define CK(call)                                                                       \
    do {                                                                               \
        cudaError_t e_ = (call);                                                       \
        if (e_ != cudaSuccess)                                                         \
            return set_error(CUTS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace {

constexpr uint32_t kFull = 0xffffffffu;
constexpr int kWarps = 8;       // warps per block in the level kernels
constexpr int kOutBuf = 128;    // per-warp staged output entries
constexpr uint32_t kTile = 256; // planner tile (parents)

// Plan + level pointers, resident in device memory for the run.
struct RunParams {
    Plan plan;
    uint32_t stored;   // levels kept in HBM: k-1 when counting, k when dumping
    // level whose entries keep, in their ub slot, the adj offset their vertex
    // was drawn from (the last stored level before a fused count: its child
    // bound is never read); kFull = none
    uint32_t pos_lvl;
    uint32_t fuse_stride;  // words per warp row of the fused kernel's scratch
    uint32_t *fuse_scratch;
    uint32_t *fuse_big;    // the fused kernel's deferred parents (counters, arrays, pool)
    uint32_t fuse_big_cap;
    uint32_t fuse_pool_words;
    uint32_t *vert[kMaxK];
    uint32_t *par[kMaxK];
    uint32_t *ub[kMaxK];
    // device-time budget: kernels take no more work once budget_ns has
    // passed since *stamp (written by k_roots) and raise *over instead
    unsigned long long budget_ns;
    unsigned long long *stamp;
    uint32_t *over;
};

// Absolute device-clock deadline of a budgeted run (0 = none).
__device__ __forceinline__ unsigned long long run_deadline(const RunParams *rp) {
    const unsigned long long b = rp->budget_ns;
    return b ? *rp->stamp + b : 0ull;
}

// True (and the run flagged) once the deadline has passed; lane 0 calls it.
__device__ __forceinline__ bool past_deadline(const RunParams *rp, unsigned long long deadline) {
    if (!deadline || global_ns() <= deadline) return false;
    atomicOr(rp->over, 1u);
    return true;
}

// Orbit fold (a pendant's closed form summed over its attachment orbit O):
// the part of the weight fixed by positions below `upto`,
//   sum_{x in O, x < upto} ( |L(m_x)| - #{j < upto : m_j in L(m_x)} ),
// where m(j) gives the matched vertex of position j.
template <class M>
__device__ __forceinline__ uint32_t orbit_base(const DevView &g, const LevelPlan &F, uint32_t upto, M m) {
    uint32_t base = 0;
    for (uint32_t xm = F.ofold & ((1u << upto) - 1); xm; xm &= xm - 1) {
        const uint32_t x = __ffs(xm) - 1;
        const uint2 inf = F.jdir[0] ? g.in_info[m(x)] : g.out_info[m(x)];
        const uint32_t *l = g.adj + inf.x;
        uint32_t sub = 0;
        for (uint32_t j = 0; j < upto; ++j)
            if (((F.oguar[x] >> j) & 1u) || contains(l, inf.y, m(j))) ++sub;
        base += inf.y - sub;
    }
    return base;
}

// The weight of candidate t at position c given the base of positions below
// c: each earlier orbit list holds t (implied by the query's arcs, checked at
// plan time), and when c is in the orbit, t's own list holds every m_j, j < c.
__device__ __forceinline__ uint32_t orbit_weight(const DevView &g, const LevelPlan &F, uint32_t c,
                                                 uint32_t base, uint32_t t, bool loops) {
    uint32_t w = base - __popc(F.ofold & ((1u << c) - 1));
    if ((F.ofold >> c) & 1u) {
        const uint2 ti = F.jdir[0] ? g.in_info[t] : g.out_info[t];
        w += ti.y - c;
        if (loops && contains(g.adj + ti.x, ti.y, t)) --w;
    }
    return w;
}

// Pendant pair (plan fold2 at level k-3; A = level k-2's plan, B = level
// k-1's, both joining the same list): with m(j) the matched vertex of
// position j <= k-3, the number of (t1, t2) with t1 in A's window of the
// list, t2 in B's, both unmatched, t1 != t2, and -- kind 2 -- t2 above
// (below) t1 on the same window.  O(log degree) per candidate.  Adds |A'|
// (the level k-2 size) to lvl2.
template <class M>
__device__ uint64_t pendant_pairs(const DevView &g, const LevelPlan &A, const LevelPlan &B, uint32_t kind,
                                  uint32_t lvl, bool loops, M m, unsigned long long &lvl2) {
    const uint32_t pen = 1u << (lvl + 1);
    uint32_t lo[2], hi[2], s0[2], e0[2], off[2], len[2], cnt[2], u[2];
    for (int r = 0; r < 2; ++r) {
        const LevelPlan &L = r ? B : A;
        u[r] = m(L.jpos[0]);
        const uint2 inf = L.jdir[0] ? g.in_info[u[r]] : g.out_info[u[r]];
        off[r] = inf.x;
        len[r] = inf.y;
        lo[r] = 0;
        hi[r] = kFullMask;
        for (uint32_t msk = L.gt_mask & ~pen; msk; msk &= msk - 1) lo[r] = max(lo[r], m(__ffs(msk) - 1) + 1);
        for (uint32_t msk = L.lt_mask & ~pen; msk; msk &= msk - 1) hi[r] = min(hi[r], m(__ffs(msk) - 1));
        const uint32_t *l = g.adj + off[r];
        const bool dir = L.jdir[0] != 0;
        s0[r] = lo[r] ? lbound_own(g, dir, u[r], l, len[r], lo[r], loops) : 0;
        e0[r] = hi[r] != kFullMask ? lbound_own(g, dir, u[r], l, len[r], hi[r], loops) : len[r];
        if (e0[r] < s0[r]) e0[r] = s0[r];
        const uint32_t guar = r ? B.guar_mask : A.guar1;
        uint32_t sub = 0;
        for (uint32_t j = 0; j <= lvl; ++j) {
            const uint32_t mj = m(j);
            if (mj >= lo[r] && mj < hi[r] && (((guar >> j) & 1u) || contains(l, len[r], mj))) ++sub;
        }
        cnt[r] = e0[r] - s0[r] - sub;
    }
    lvl2 += cnt[0];
    if (kind == 2) return uint64_t(cnt[0]) * (cnt[0] - (cnt[0] ? 1 : 0)) / 2;
    // |A'| |B'| - |A' n B'|
    uint64_t both = 0;
    const uint32_t wlo = max(lo[0], lo[1]), whi = min(hi[0], hi[1]);
    if (wlo < whi) {
        // one list: its entries in both windows form the window [wlo, whi)
        const uint32_t a = max(s0[0], s0[1]), b = min(e0[0], e0[1]);
        both = b > a ? b - a : 0;
        // matched vertices lying in both windows and lists
        for (uint32_t j = 0; j <= lvl; ++j) {
            const uint32_t mj = m(j);
            if (mj < wlo || mj >= whi) continue;
            const bool in0 = ((A.guar1 >> j) & 1u) || contains(g.adj + off[0], len[0], mj);
            const bool in1 = ((B.guar_mask >> j) & 1u) || contains(g.adj + off[1], len[1], mj);
            if (in0 && in1) --both;
        }
    }
    return uint64_t(cnt[0]) * cnt[1] - both;
}

enum Mode { kExpand = 0, kCountMode = 1, kBytesMode = 2 };

// ---- level 0: signature scan (device_funcs.cu:267-279) ---------------
__global__ void k_roots(DevView g, const RunParams *__restrict__ rp, uint32_t shard, uint32_t nshards,
                        uint32_t *__restrict__ n0) {
    const Plan &P = rp->plan;
    const uint32_t qin = P.lv[0].qin, qout = P.lv[0].qout;
    // L_0 entries carry the child bound for level 1, whose joins all use
    // position 0 (only needed when level 1 is stored)
    const bool need_ub = rp->stored >= 2;
    bool use_out = false, use_in = false;
    if (P.k >= 2)
        for (uint32_t t = 0; t < P.lv[1].nj; ++t) (P.lv[1].jdir[t] ? use_in : use_out) = true;
    uint32_t *vert0 = rp->vert[0], *ub0 = rp->ub[0];
    const int lane = threadIdx.x & 31;
    if (blockIdx.x == 0 && threadIdx.x == 0 && rp->budget_ns) *rp->stamp = global_ns();
    for (uint32_t base = blockIdx.x * blockDim.x; base < g.n; base += gridDim.x * blockDim.x) {
        const uint32_t u = base + threadIdx.x;
        bool ok = false;
        uint32_t ub = UINT_MAX;
        if (u < g.n && u % nshards == shard) {  // rank striding, device_funcs.cu:273
            const uint2 o = g.out_info[u], i = g.in_info[u];
            ok = o.y >= qout && i.y >= qin;
            if (use_out) ub = min(ub, o.y);
            if (use_in) ub = min(ub, i.y);
        }
        const unsigned m = __ballot_sync(kFull, ok);
        if (m) {
            uint32_t pos = 0;
            if (lane == 0) pos = atomicAdd(n0, uint32_t(__popc(m)));
            pos = __shfl_sync(kFull, pos, 0) + __popc(m & ((1u << lane) - 1));
            if (ok) {
                vert0[pos] = u;
                if (need_ub) ub0[pos] = ub;
            }
        }
    }
}

// ---- levels 1..k-1 -----------------------------------------------------
// MODE kExpand: write L_lvl from parents [pa, pb) of L_{lvl-1}.
// MODE kCountMode: last level, accumulate the count.
// MODE kBytesMode: accumulate the algorithmic bytes of the last level.
template <int MODE>
__global__ void __launch_bounds__(kWarps * 32)
k_level(DevView g, const RunParams *__restrict__ rp, uint32_t lvl, uint32_t pa, uint32_t pb,
        uint32_t grain, uint32_t *__restrict__ cursor, uint32_t *__restrict__ out_n,
        uint32_t out_cap, uint32_t *__restrict__ err, unsigned long long *__restrict__ acc) {
    __shared__ LevelPlan sL, sN;
    __shared__ uint32_t *s_vert[kMaxK];
    __shared__ uint32_t *s_par[kMaxK];
    __shared__ uint32_t s_k, s_sym, s_stored;
    __shared__ uint32_t wm[kWarps][kMaxK];
    __shared__ uint32_t joff[kWarps][kMaxJ], jdeg[kWarps][kMaxJ];
    __shared__ uint32_t ob_v[MODE == kExpand ? kWarps : 1][kOutBuf];
    __shared__ uint32_t ob_p[MODE == kExpand ? kWarps : 1][kOutBuf];
    __shared__ uint32_t ob_u[MODE == kExpand ? kWarps : 1][kOutBuf];

    {
        const uint32_t words = sizeof(LevelPlan) / 4;
        const uint32_t *srcL = reinterpret_cast<const uint32_t *>(&rp->plan.lv[lvl]);
        uint32_t *dL = reinterpret_cast<uint32_t *>(&sL);
        for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dL[i] = srcL[i];
        const uint32_t nl = lvl + 1 < rp->plan.k ? lvl + 1 : lvl;
        const uint32_t *srcN = reinterpret_cast<const uint32_t *>(&rp->plan.lv[nl]);
        uint32_t *dN = reinterpret_cast<uint32_t *>(&sN);
        for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dN[i] = srcN[i];
        if (threadIdx.x < kMaxK) {
            s_vert[threadIdx.x] = rp->vert[threadIdx.x];
            s_par[threadIdx.x] = rp->par[threadIdx.x];
        }
        if (threadIdx.x == 0) { s_k = rp->plan.k; s_sym = rp->plan.symmetric; s_stored = rp->stored; }
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t lanemask_lt = (1u << lane) - 1;
    uint32_t *my_m = wm[warp];
    const uint32_t k = s_k;
    const bool sym = s_sym != 0;
    // entries of L_lvl need a child bound when level lvl+1 is stored too; at
    // the position level the slot keeps where the vertex sits in its list
    const bool store_pos = MODE == kExpand && lvl == rp->pos_lvl;
    const bool need_ub = (MODE == kExpand && lvl + 1 < s_stored) || store_pos;
    uint32_t *out_v = MODE == kExpand ? rp->vert[lvl] : nullptr;
    uint32_t *out_p = MODE == kExpand ? rp->par[lvl] : nullptr;
    uint32_t *out_u = MODE == kExpand ? rp->ub[lvl] : nullptr;
    // next-level joins on the child itself (position lvl) bound its children
    bool ub_out = false, ub_in = false;
    if (need_ub && !store_pos)
        for (uint32_t t = 0; t < sN.nj; ++t)
            if (sN.jpos[t] == lvl) (sN.jdir[t] ? ub_in : ub_out) = true;
    const uint32_t nj = sL.nj;
    const bool check_sig = sL.check_sig != 0;
    const bool load_info = check_sig || ub_out || ub_in;

    uint32_t cached_q = kFull;  // lane 0: L_{lvl-2} index whose path is in my_m[0..lvl-2]
    uint32_t obn = 0;           // staged outputs (warp-uniform)
    unsigned long long local = 0;
    const uint32_t total = pb - pa;
    const unsigned long long deadline = run_deadline(rp);

    auto flush = [&]() {
        if constexpr (MODE != kExpand) return;
        __syncwarp();
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(out_n, obn);
        base = __shfl_sync(kFull, base, 0);
        if (base + obn <= out_cap && base + obn >= base) {
            for (uint32_t i = lane; i < obn; i += 32) {
                out_v[base + i] = ob_v[warp][i];
                out_p[base + i] = ob_p[warp][i];
                if (need_ub) out_u[base + i] = ob_u[warp][i];
            }
        } else if (lane == 0) {
            atomicOr(err, 1u);
        }
        obn = 0;
        __syncwarp();
    };

    while (true) {
        uint32_t start = 0;
        if (lane == 0) start = past_deadline(rp, deadline) ? total : atomicAdd(cursor, grain);
        start = __shfl_sync(kFull, start, 0);
        if (start >= total) break;
        const uint32_t end = min(start + grain, total);
        for (uint32_t pi = start; pi < end; ++pi) {
            const uint32_t p = pa + pi;
            // rebuild the parent's partial match (device_funcs.cu:39-55),
            // reusing the ancestors shared with the previous parent
            if (lane == 0) {
                my_m[lvl - 1] = s_vert[lvl - 1][p];
                if (lvl >= 2) {
                    uint32_t q = s_par[lvl - 1][p];
                    if (q != cached_q) {
                        cached_q = q;
                        for (int j = int(lvl) - 2; j >= 0; --j) {
                            my_m[j] = s_vert[j][q];
                            if (j > 0) q = s_par[j][q];
                        }
                    }
                }
            }
            __syncwarp();

            // joined lists; the shortest supplies the candidates
            uint32_t my_deg = kFull, my_off = 0;
            if (uint32_t(lane) < nj) {
                const uint32_t u = my_m[sL.jpos[lane]];
                const uint2 inf = sL.jdir[lane] ? g.in_info[u] : g.out_info[u];
                my_off = inf.x;
                my_deg = inf.y;
                joff[warp][lane] = my_off;
                jdeg[warp][lane] = my_deg;
            }
            uint32_t bd = my_deg, bl = uint32_t(lane);
            #pragma unroll
            for (int s = 16; s; s >>= 1) {
                const uint32_t od = __shfl_xor_sync(kFull, bd, s), ol = __shfl_xor_sync(kFull, bl, s);
                if (od < bd || (od == bd && ol < bl)) { bd = od; bl = ol; }
            }
            if (nj == 0) { __syncwarp(); continue; }  // unreachable for validated orders
            const uint32_t tmin = bl, mdeg = bd;
            const uint32_t moff = __shfl_sync(kFull, my_off, int(tmin));
            __syncwarp();

            if constexpr (MODE == kBytesMode) {
                if (lane == 0) {
                    unsigned long long b = 8;
                    for (uint32_t t = 0; t < nj; ++t) b += 4ull * jdeg[warp][t] + 8;
                    local += b;
                }
                __syncwarp();
                continue;
            }

            // symmetry-breaking window [lo, hi) on the candidate value
            uint32_t lo = 0, hi = kFull;
            for (uint32_t msk = sL.gt_mask; msk; msk &= msk - 1) lo = max(lo, my_m[__ffs(msk) - 1] + 1);
            for (uint32_t msk = sL.lt_mask; msk; msk &= msk - 1) hi = min(hi, my_m[__ffs(msk) - 1]);
            const uint32_t *mlist = g.adj + moff;
            const uint32_t s0 = lo ? lbound(mlist, mdeg, lo) : 0;
            const uint32_t e0 = hi != kFull ? lbound(mlist, mdeg, hi) : mdeg;

            if (MODE == kCountMode && sL.closed_form) {  // uniform branch
                // one joined list, no signature: every list element in the
                // window except the already-matched vertices extends
                if (s0 < e0) {
                    bool hit = false;
                    if (uint32_t(lane) < lvl) {
                        const uint32_t mj = my_m[lane];
                        hit = mj >= lo && mj < hi && contains(mlist, mdeg, mj);
                    }
                    const uint32_t sub = __popc(__ballot_sync(kFull, hit));
                    if (lane == 0) local += (e0 - s0) - sub;
                }
                __syncwarp();
                continue;
            }

            uint32_t ubp = kFull;
            if (need_ub) {
                uint32_t d = kFull;
                if (uint32_t(lane) < sN.nj && sN.jpos[lane] < lvl) {
                    const uint32_t u = my_m[sN.jpos[lane]];
                    d = (sN.jdir[lane] ? g.in_info[u] : g.out_info[u]).y;
                }
                ubp = warp_min(d);
            }

            for (uint32_t x0 = s0; x0 < e0; x0 += 32) {
                const uint32_t x = x0 + lane;
                bool ok = x < e0;
                const uint32_t c = ok ? __ldg(mlist + x) : 0;
                if (ok)
                    for (uint32_t j = 0; j < lvl; ++j)
                        if (c == my_m[j]) { ok = false; break; }
                uint2 co = make_uint2(0, 0), ci = make_uint2(0, 0);
                if (ok && load_info) {
                    co = g.out_info[c];
                    ci = sym ? co : g.in_info[c];
                }
                if (ok && check_sig) ok = ci.y >= sL.qin && co.y >= sL.qout;
                if (ok)
                    for (uint32_t t = 0; t < nj; ++t) {
                        if (t == tmin) continue;
                        if (!contains(g.adj + joff[warp][t], jdeg[warp][t], c)) { ok = false; break; }
                    }
                if constexpr (MODE == kCountMode) {
                    local += ok;
                } else {
                    uint32_t ub = ubp;
                    if (ub_out) ub = min(ub, co.y);
                    if (ub_in) ub = min(ub, ci.y);
                    if (store_pos) ub = moff + x;
                    const unsigned m = __ballot_sync(kFull, ok);
                    const uint32_t nn = __popc(m);
                    if (obn + nn > uint32_t(kOutBuf)) flush();
                    if (ok) {
                        const uint32_t r = obn + __popc(m & lanemask_lt);
                        ob_v[warp][r] = c;
                        ob_p[warp][r] = p;
                        ob_u[warp][r] = ub;
                    }
                    obn += nn;
                }
            }
            __syncwarp();
        }
    }
    if constexpr (MODE == kExpand) {
        if (obn) flush();
    } else {
        #pragma unroll
        for (int s = 16; s; s >>= 1) local += __shfl_xor_sync(kFull, local, s);
        if (lane == 0 && local) atomicAdd(acc, local);
    }
}

// ---- levels 1..k-1, flattened form ------------------------------------
// A warp takes 32 consecutive parents, one per lane.  Each lane rebuilds its
// parent's partial match (32 pointer chases in flight at once), gathers its
// joined lists and picks the shortest.  The candidate lists of the 32
// parents are then treated as one concatenated sequence: an inclusive warp
// scan of their lengths gives every lane, at every step, the parent that
// owns candidate f = step*32 + lane (a 5-step binary search over the scan
// with shuffles), so all 32 lanes stay busy whether the lists hold 2 or
// 20,000 entries.  Per-parent state lives in the owner lane's registers
// (read with shuffles) and in shared memory laid out [join][lane], so lanes
// reading different owners hit different banks.  Last-level parents with a
// single joined list and no signature are counted by the closed form, one
// parent per lane.
constexpr int kFW = 4;    // warps per block
constexpr int kFJ = 8;    // joined lists per level in this form (more: warp-per-parent kernel)

template <int MODE>
__global__ void __launch_bounds__(kFW * 32)
k_level_flat(DevView g, const RunParams *__restrict__ rp, uint32_t lvl, uint32_t pa, uint32_t pb,
             uint32_t *__restrict__ cursor, uint32_t *__restrict__ out_n, uint32_t out_cap,
             uint32_t *__restrict__ err, unsigned long long *__restrict__ acc,
             unsigned long long *__restrict__ acc2, unsigned long long *__restrict__ acc3) {
    __shared__ LevelPlan sL, sN, sN2;
    __shared__ uint32_t *s_vert[kMaxK];
    __shared__ uint32_t *s_par[kMaxK];
    __shared__ uint32_t s_k, s_sym, s_stored;
    __shared__ uint32_t sm_m[kFW][kMaxK][33];   // [position][lane]
    __shared__ uint32_t sm_off[kFW][kFJ][32], sm_deg[kFW][kFJ][32];
    __shared__ uint32_t ob_v[MODE == kExpand ? kFW : 1][kOutBuf];
    __shared__ uint32_t ob_p[MODE == kExpand ? kFW : 1][kOutBuf];
    __shared__ uint32_t ob_u[MODE == kExpand ? kFW : 1][kOutBuf];
    {
        const uint32_t words = sizeof(LevelPlan) / 4;
        const uint32_t *srcL = reinterpret_cast<const uint32_t *>(&rp->plan.lv[lvl]);
        uint32_t *dL = reinterpret_cast<uint32_t *>(&sL);
        for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dL[i] = srcL[i];
        const uint32_t nl = lvl + 1 < rp->plan.k ? lvl + 1 : lvl;
        const uint32_t *srcN = reinterpret_cast<const uint32_t *>(&rp->plan.lv[nl]);
        uint32_t *dN = reinterpret_cast<uint32_t *>(&sN);
        for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dN[i] = srcN[i];
        const uint32_t nl2 = lvl + 2 < rp->plan.k ? lvl + 2 : nl;
        const uint32_t *srcN2 = reinterpret_cast<const uint32_t *>(&rp->plan.lv[nl2]);
        uint32_t *dN2 = reinterpret_cast<uint32_t *>(&sN2);
        for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dN2[i] = srcN2[i];
        if (threadIdx.x < kMaxK) {
            s_vert[threadIdx.x] = rp->vert[threadIdx.x];
            s_par[threadIdx.x] = rp->par[threadIdx.x];
        }
        if (threadIdx.x == 0) { s_k = rp->plan.k; s_sym = rp->plan.symmetric; s_stored = rp->stored; }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t lanemask_lt = (1u << lane) - 1;
    const bool sym = s_sym != 0;
    // pendant pair: this level (k-3) also counts levels k-2 and k-1
    const uint32_t fold2 = MODE != kExpand ? sL.fold2 : 0u;
    unsigned long long local3 = 0;
    const bool store_pos = MODE == kExpand && lvl == rp->pos_lvl;
    const bool need_ub = (MODE == kExpand && lvl + 1 < s_stored) || store_pos;
    uint32_t *out_v = MODE == kExpand ? rp->vert[lvl] : nullptr;
    uint32_t *out_p = MODE == kExpand ? rp->par[lvl] : nullptr;
    uint32_t *out_u = MODE == kExpand ? rp->ub[lvl] : nullptr;
    bool ub_out = false, ub_in = false;
    if (need_ub && !store_pos)
        for (uint32_t t = 0; t < sN.nj; ++t)
            if (sN.jpos[t] == lvl) (sN.jdir[t] ? ub_in : ub_out) = true;
    const uint32_t nj = sL.nj;
    const bool check_sig = sL.check_sig != 0;
    const bool load_info = check_sig || ub_out || ub_in;
    const bool closed = MODE == kCountMode && sL.closed_form;
    // level k-2 counting level k-1 too: each candidate c adds the last
    // level's closed form, |window of L| - matched vertices in it, where L
    // is an earlier vertex's list and c itself is one of the matched
    const bool fold = MODE != kExpand && sL.fold;
    const bool fold_guar_c = fold && ((sN.guar_mask >> lvl) & 1u);
    const bool loops = rp->plan.data_loops != 0;
    const uint32_t total = pb - pa;
    const unsigned long long deadline = run_deadline(rp);
    unsigned long long local = 0, local2 = 0;
    uint32_t obn = 0;

    auto flush = [&]() {
        if constexpr (MODE != kExpand) return;
        __syncwarp();
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(out_n, obn);
        base = __shfl_sync(kFullMask, base, 0);
        if (base + obn <= out_cap && base + obn >= base) {
            for (uint32_t i = lane; i < obn; i += 32) {
                out_v[base + i] = ob_v[warp][i];
                out_p[base + i] = ob_p[warp][i];
                if (need_ub) out_u[base + i] = ob_u[warp][i];
            }
        } else if (lane == 0) {
            atomicOr(err, 1u);
        }
        obn = 0;
        __syncwarp();
    };

    while (true) {
        uint32_t start = 0;
        if (lane == 0) start = past_deadline(rp, deadline) ? total : atomicAdd(cursor, 32u);
        start = __shfl_sync(kFullMask, start, 0);
        if (start >= total) break;
        const uint32_t p = pa + start + lane;
        const bool have = start + lane < total;
        // this lane's parent: partial match into column `lane`
        if (have) {
            uint32_t e = p;
            for (int j = int(lvl) - 1; j >= 0; --j) {
                sm_m[warp][j][lane] = s_vert[j][e];
                if (j > 0) e = s_par[j][e];
            }
        }
        // joined lists, shortest first
        uint32_t moff = 0, mdeg = 0, tmin = 0, s0 = 0, e0 = 0, ubp = kFullMask;
        uint32_t f_off = 0, f_deg = 0, f_lo = 0, f_hi = kFullMask, fbase = 0;
        unsigned long long bytes = 0;
        if (have) {
            mdeg = kFullMask;
            for (uint32_t t = 0; t < nj; ++t) {
                const uint32_t u = sm_m[warp][sL.jpos[t]][lane];
                const uint2 inf = sL.jdir[t] ? g.in_info[u] : g.out_info[u];
                sm_off[warp][t][lane] = inf.x;
                sm_deg[warp][t][lane] = inf.y;
                if (MODE == kBytesMode) bytes += 4ull * inf.y + 8;
                if (inf.y < mdeg) { mdeg = inf.y; moff = inf.x; tmin = t; }
            }
            if (nj == 0) mdeg = 0;
            uint32_t lo = 0, hi = kFullMask;
            for (uint32_t msk = sL.gt_mask; msk; msk &= msk - 1) lo = max(lo, sm_m[warp][__ffs(msk) - 1][lane] + 1);
            for (uint32_t msk = sL.lt_mask; msk; msk &= msk - 1) hi = min(hi, sm_m[warp][__ffs(msk) - 1][lane]);
            const uint32_t *lst = g.adj + moff;
            const uint32_t mu = nj ? sm_m[warp][sL.jpos[tmin]][lane] : 0;
            const bool mdir = nj && sL.jdir[tmin];
            s0 = lo ? lbound_own(g, mdir, mu, lst, mdeg, lo, loops) : 0;
            e0 = hi != kFullMask ? lbound_own(g, mdir, mu, lst, mdeg, hi, loops) : mdeg;
            if (e0 < s0) e0 = s0;
            if (need_ub)
                for (uint32_t t = 0; t < sN.nj; ++t)
                    if (sN.jpos[t] < lvl) {
                        const uint32_t u = sm_m[warp][sN.jpos[t]][lane];
                        ubp = min(ubp, (sN.jdir[t] ? g.in_info[u] : g.out_info[u]).y);
                    }
            if (fold && sN.ofold) {
                fbase = orbit_base(g, sN, lvl, [&](uint32_t j) { return sm_m[warp][j][lane]; });
            } else if (fold) {
                const uint32_t u = sm_m[warp][sN.jpos[0]][lane];
                const uint2 inf = sN.jdir[0] ? g.in_info[u] : g.out_info[u];
                f_off = inf.x;
                f_deg = inf.y;
                for (uint32_t msk = sN.gt_mask; msk; msk &= msk - 1) f_lo = max(f_lo, sm_m[warp][__ffs(msk) - 1][lane] + 1);
                for (uint32_t msk = sN.lt_mask; msk; msk &= msk - 1) f_hi = min(f_hi, sm_m[warp][__ffs(msk) - 1][lane]);
                const uint32_t *fl = g.adj + f_off;
                const uint32_t ws = f_lo ? lbound(fl, f_deg, f_lo) : 0;
                const uint32_t we = f_hi != kFullMask ? lbound(fl, f_deg, f_hi) : f_deg;
                uint32_t sub = 0;
                for (uint32_t j = 0; j < lvl; ++j) {
                    const uint32_t mj = sm_m[warp][j][lane];
                    if (mj >= f_lo && mj < f_hi && (((sN.guar_mask >> j) & 1u) || contains(fl, f_deg, mj))) ++sub;
                }
                fbase = (we > ws ? we - ws : 0) - sub;
            }
            if (MODE == kBytesMode) {
                // what this kernel's algorithm reads for the parent: its own
                // and its ancestors' (vertex, parent) entries, the joined
                // vertices' info, then either the closed form's probes or the
                // streamed candidate window plus, per candidate, the signature
                // gather and one lower-bound probe sequence per other list
                (void)bytes;
                auto probes = [](uint32_t len) { return 32u - __clz(len | 1u); };
                unsigned long long b = 8ull * lvl + 8ull * nj;
                const uint32_t len = e0 - s0;
                if (sL.closed_form) {  // the count kernel's closed form
                    b += 4ull * lvl * probes(mdeg);
                } else {
                    uint32_t per = check_sig ? 8 : 0;
                    for (uint32_t t = 0; t < nj; ++t)
                        if (t != tmin) per += 4 * probes(sm_deg[warp][t][lane]);
                    if (fold) {
                        b += 8 + 4ull * lvl * probes(f_deg);
                        if (!fold_guar_c) per += 4 * probes(f_deg);
                    }
                    b += 4ull * len + uint64_t(len) * per;
                }
                local += b;
            }
            if (closed && MODE == kCountMode) {
                // one list, no signature: the window minus the matched vertices in it
                uint32_t sub = 0;
                for (uint32_t j = 0; j < lvl; ++j) {
                    const uint32_t mj = sm_m[warp][j][lane];
                    if (mj >= lo && mj < hi && (((sL.guar_mask >> j) & 1u) || contains(lst, mdeg, mj))) ++sub;
                }
                local += (e0 - s0) - sub;
            }
        }
        if (MODE == kBytesMode || closed) continue;
        __syncwarp();
        // concatenated candidate sequence of the 32 parents
        const uint32_t len = e0 - s0;
        uint32_t incl = len;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFullMask, incl, o);
            if (lane >= o) incl += y;
        }
        const uint32_t ftotal = __shfl_sync(kFullMask, incl, 31);
        uint32_t gal_owner = kFullMask, gal_pos0 = 0, gal_pos1 = 0;
        for (uint32_t fstep = 0; fstep < ftotal; fstep += 32) {
            const uint32_t f = fstep + lane;
            // owner = number of lanes whose inclusive end is <= f
            uint32_t owner = 0;
            #pragma unroll
            for (int step = 16; step; step >>= 1) {
                const uint32_t probe = __shfl_sync(kFullMask, incl, int(owner + step - 1));
                if (probe <= f) owner += step;
            }
            owner = min(owner, 31u);
            const uint32_t o_incl = __shfl_sync(kFullMask, incl, int(owner));
            const uint32_t o_len = __shfl_sync(kFullMask, len, int(owner));
            const uint32_t o_s0 = __shfl_sync(kFullMask, s0, int(owner));
            const uint32_t o_moff = __shfl_sync(kFullMask, moff, int(owner));
            const uint32_t o_tmin = __shfl_sync(kFullMask, tmin, int(owner));
            const uint32_t o_ubp = __shfl_sync(kFullMask, ubp, int(owner));
            bool ok = f < ftotal;
            const uint32_t idx = o_s0 + (f - (o_incl - o_len));
            const uint32_t c = ok ? __ldg(g.adj + o_moff + idx) : 0;
            if (ok)
                for (uint32_t j = 0; j < lvl; ++j)
                    if (c == sm_m[warp][j][owner]) { ok = false; break; }
            uint2 co = make_uint2(0, 0), ci = make_uint2(0, 0);
            if (ok && load_info) {
                co = g.out_info[c];
                ci = sym ? co : g.in_info[c];
            }
            if (ok && check_sig) ok = ci.y >= sL.qin && co.y >= sL.qout;
            if (owner != gal_owner) {  // new parent for this lane: restart the searches
                gal_owner = owner;
                gal_pos0 = gal_pos1 = 0;
            }
            if (ok) {
                uint32_t r = 0;
                for (uint32_t t = 0; t < nj; ++t) {
                    if (t == o_tmin) continue;
                    const uint32_t *lst = g.adj + sm_off[warp][t][owner];
                    const uint32_t len2 = sm_deg[warp][t][owner];
                    // this lane's candidates for one parent rise, so its lower
                    // bounds in each other list rise too: gallop from the last
                    const uint32_t from = r == 0 ? gal_pos0 : (r == 1 ? gal_pos1 : 0);
                    const uint32_t pos = lbound_from(lst, len2, from, c);
                    if (r == 0) gal_pos0 = pos;
                    else if (r == 1) gal_pos1 = pos;
                    ++r;
                    if (pos >= len2 || __ldg(lst + pos) != c) { ok = false; break; }
                }
            }
            if constexpr (MODE == kCountMode) {
                if (fold2) {
                    if (ok) {
                        const uint64_t p2 = pendant_pairs(g, sN, sN2, fold2, lvl, loops,
                            [&](uint32_t j) { return j == lvl ? c : sm_m[warp][j][owner]; }, local3);
                        local += p2;
                        ++local2;
                    }
                } else if (fold) {
                    const uint32_t o_fbase = __shfl_sync(kFullMask, fbase, int(owner));
                    const uint32_t o_foff = __shfl_sync(kFullMask, f_off, int(owner));
                    const uint32_t o_fdeg = __shfl_sync(kFullMask, f_deg, int(owner));
                    const uint32_t o_flo = __shfl_sync(kFullMask, f_lo, int(owner));
                    const uint32_t o_fhi = __shfl_sync(kFullMask, f_hi, int(owner));
                    if (ok && sN.ofold) {
                        local += orbit_weight(g, sN, lvl, o_fbase, c, loops);
                        ++local2;
                    } else if (ok) {
                        const bool hit = c >= o_flo && c < o_fhi &&
                                         (fold_guar_c || contains(g.adj + o_foff, o_fdeg, c));
                        local += o_fbase - (hit ? 1u : 0u);
                        ++local2;
                    }
                } else {
                    local += ok;
                }
            } else {
                uint32_t ub = o_ubp;
                if (ub_out) ub = min(ub, co.y);
                if (ub_in) ub = min(ub, ci.y);
                if (store_pos) ub = o_moff + idx;  // where c sits in the list it came from
                const unsigned m = __ballot_sync(kFullMask, ok);
                const uint32_t nn = __popc(m);
                if (obn + nn > uint32_t(kOutBuf)) flush();
                if (ok) {
                    const uint32_t r = obn + __popc(m & lanemask_lt);
                    ob_v[warp][r] = c;
                    ob_p[warp][r] = pa + start + owner;
                    ob_u[warp][r] = ub;
                }
                obn += nn;
            }
        }
        __syncwarp();
    }
    if constexpr (MODE == kExpand) {
        if (obn) flush();
    } else {
        #pragma unroll
        for (int s = 16; s; s >>= 1) {
            local += __shfl_xor_sync(kFullMask, local, s);
            local2 += __shfl_xor_sync(kFullMask, local2, s);
            local3 += __shfl_xor_sync(kFullMask, local3, s);
        }
        if (lane == 0 && local) atomicAdd(acc, local);
        if (lane == 0 && local2 && acc2) atomicAdd(acc2, local2);
        if (lane == 0 && local3 && acc3) atomicAdd(acc3, local3);
    }
}

// ---- fused count of levels p and c = p + 1 ---------------------------
// When the plan fuses the counted level c with p = c - 1, c's candidates for
// a vertex s chosen at p are the members t of p's candidate set S (same
// parent) that lie in s's list.  One warp per parent at level p - 1: build S
// once (the usual scan of the shortest joined list, membership in the
// others, ballot compaction) into the warp's scratch row, then intersect S
// with the list of every s in S, 32 vertices s at a time (one per lane), and
// count (or, for a folded c, add the last level's closed form per t).
// Level p is never written to the trie.
//
// The work of one parent grows like |S|^2, so a hub parent would keep one
// warp busy long after the others finish.  Phase 1 therefore defers every
// parent with |S| > kBigS: it copies S into a pool and records the parent;
// phase 2 (a second launch, after a one-block scan of the deferred parents'
// group counts) hands out their groups of 32 vertices s to all warps.
constexpr int kZW = 4;          // warps per block
constexpr uint32_t kBigS = 256;  // default |S| above which a parent is split

// Parents deferred by phase 1 and their saved candidate sets.
struct FusedBig {
    unsigned long long *n;  // [0] entries appended, [1] pool words taken
    uint32_t *gi;           // parent index (in L_{p-1}) of each entry
    uint32_t *soff;         // offset of its S in the pool
    uint32_t *ns;           // |S|
    uint32_t *pref;         // inclusive prefix sum of groups of 32 (phase 2)
    uint32_t *pool;
    uint32_t cap;
    unsigned long long pool_words;
};

// Phase 1 keeps a parent's candidate set S in shared memory when it holds at
// most kTS vertices; every pair (s, t) of S is then tested by a lane-balanced
// walk (see pair_walk below).
constexpr uint32_t kTS = 256;
constexpr uint32_t kHS = 512;  // hash slots of the admissible t, buckets of 4 (load at most 1/2)

// WALK instances (phase 1 of plans the pair walk covers): 8 resident blocks
// (32 warps) per SM at up to 64 registers -- the walk keeps its row state
// in registers and ~25 KB of tables in shared memory.  The others: 12
// resident blocks (48 warps) at 40 registers -- they wait on dependent L2
// loads, and the extra warps outweigh the spills that cap costs.
template <int MODE, bool WALK, bool TALLY = false>
__global__ void __launch_bounds__(kZW * 32, WALK ? 8 : 12)
k_fused(DevView g, const RunParams *__restrict__ rp, uint32_t p, uint32_t pa, uint32_t pb, uint32_t phase,
        uint32_t split, uint32_t *__restrict__ cursor, uint32_t *__restrict__ scratch, uint32_t stride, FusedBig big,
        unsigned long long *__restrict__ acc, unsigned long long *__restrict__ acc_c,
        unsigned long long *__restrict__ acc_p, unsigned long long *__restrict__ acc_bytes) {
    constexpr bool walk_ok = WALK && MODE == kCountMode;
    // TALLY: also add the bytes this count reads from global memory to
    // *acc_bytes (the last level's algorithmic traffic; counts go to scratch)
    constexpr bool tally = TALLY && MODE == kCountMode;
    unsigned long long tb = 0;
    __shared__ LevelPlan sP, sC, sF;
    __shared__ uint32_t *s_vert[kMaxK];
    __shared__ uint32_t *s_par[kMaxK];
    __shared__ uint32_t wm[kZW][kMaxK];
    __shared__ uint32_t joff[kZW][kMaxJ], jdeg[kZW][kMaxJ], jver[kZW][kMaxJ];
    __shared__ uint32_t xoff[kZW][kMaxJ], xdeg[kZW][kMaxJ];
    // the pair walk's per-parent tables: S, and a hash table of the vertices
    // admissible as t (keys in buckets of 4, their index in S and term B)
    __shared__ uint32_t tS[walk_ok ? kZW : 1][kTS];
    __shared__ uint4 tHK[walk_ok ? kZW : 1][kHS / 4];
    // dense core: the admissible t of S as bits of the core (per warp)
    __shared__ uint32_t tSV[walk_ok ? kZW : 1][kCore / 32];
    __shared__ uint8_t tHI[walk_ok ? kZW : 1][kHS];
    __shared__ int32_t tHB[walk_ok ? kZW : 1][kHS];
    {
        const uint32_t words = sizeof(LevelPlan) / 4;
        const uint32_t c = p + 1;
        const uint32_t f = c + 1 < rp->plan.k ? c + 1 : c;
        const uint32_t *a = reinterpret_cast<const uint32_t *>(&rp->plan.lv[p]);
        const uint32_t *b = reinterpret_cast<const uint32_t *>(&rp->plan.lv[c]);
        const uint32_t *d = reinterpret_cast<const uint32_t *>(&rp->plan.lv[f]);
        for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) {
            reinterpret_cast<uint32_t *>(&sP)[i] = a[i];
            reinterpret_cast<uint32_t *>(&sC)[i] = b[i];
            reinterpret_cast<uint32_t *>(&sF)[i] = d[i];
        }
        if (threadIdx.x < kMaxK) {
            s_vert[threadIdx.x] = rp->vert[threadIdx.x];
            s_par[threadIdx.x] = rp->par[threadIdx.x];
        }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t lanemask_lt = (1u << lane) - 1;
    uint32_t *my_m = wm[warp];
    uint32_t *const row = scratch + size_t(blockIdx.x * kZW + warp) * stride;

    const uint32_t c = p + 1;
    // the counted level c is folded when level c carries the fold flag
    const bool cfold = sC.fold != 0;
    const uint32_t tp = sC.fuse_tp;
    const uint32_t extra = sC.fuse_extra;
    const bool sig_c = sC.check_sig && (sC.qin > sP.qin || sC.qout > sP.qout);
    const uint32_t below = (1u << p) - 1;
    const bool c_gt_s = (sC.gt_mask >> p) & 1u, c_lt_s = (sC.lt_mask >> p) & 1u;
    const bool fguar_t = cfold && ((sF.guar_mask >> c) & 1u);
    const bool loops = rp->plan.data_loops != 0;
    // an extra list of c on position p itself changes with s: per-s loop
    bool extra_on_p = false;
    for (uint32_t t = 0; t < sC.nj; ++t)
        if (((extra >> t) & 1u) && sC.jpos[t] == p) extra_on_p = true;
    unsigned long long local = 0, local_c = 0, local_p = 0;
    uint32_t cached_q = kFullMask;
    const bool phase2 = phase == 2;
    uint32_t nbig = 0, total = pb - pa;
    if (phase2) {
        const unsigned long long n0 = big.n[0];
        nbig = n0 < big.cap ? uint32_t(n0) : big.cap;
        total = nbig ? big.pref[nbig - 1] : 0;
    }
    const unsigned long long deadline = run_deadline(rp);
    auto probes = [](uint32_t len) { return 32u - __clz(len | 1u); };

    // level c for the vertices s = S[i0 .. i0+32) of one parent
    auto group = [&](const uint32_t *S, uint32_t ns, uint32_t i0, uint32_t lo_c, uint32_t hi_c) {
        if (!extra_on_p) {
            // one s per lane; the 32 (s, t) sequences are concatenated and
            // spread over all lanes, as in k_level_flat
            const uint32_t i = i0 + lane;
            // the iterated range starts at itb (in S when iters, else in the
            // adjacency array); the probed one is [ostart, oend) of S or of
            // the list at ooff
            uint32_t sv = kFullMask, itb = 0, ooff = 0, ostart = 0, oend = 0, nit = 0, iters = 1;
            uint32_t fbase = 0, foff = 0, fdeg = 0, flo = 0, fhi = kFullMask;
            if (i < ns) {
                sv = S[i];
                const uint2 is = sC.jdir[tp] ? g.in_info[sv] : g.out_info[sv];
                const uint32_t lsoff = is.x, ds = is.y;
                uint32_t lo_t = lo_c, hi_t = hi_c;
                if (c_gt_s) lo_t = max(lo_t, sv + 1);
                if (c_lt_s) hi_t = min(hi_t, sv);
                const uint32_t ts = lo_t ? lbound(S, ns, lo_t) : 0;
                const uint32_t te = hi_t != kFullMask ? lbound(S, ns, hi_t) : ns;
                const uint32_t *Ls = g.adj + lsoff;
                const bool sdir = sC.jdir[tp] != 0;
                const uint32_t ls0 = lo_t ? lbound_own(g, sdir, sv, Ls, ds, lo_t, loops) : 0;
                const uint32_t ls1 = hi_t != kFullMask ? lbound_own(g, sdir, sv, Ls, ds, hi_t, loops) : ds;
                const uint32_t nS = te > ts ? te - ts : 0, nL = ls1 > ls0 ? ls1 - ls0 : 0;
                iters = nS <= nL ? 1u : 0u;  // iterate the shorter side
                nit = iters ? nS : nL;
                itb = iters ? ts : lsoff + ls0;
                ooff = iters ? lsoff : 0;
                ostart = iters ? ls0 : ts;
                oend = iters ? ls1 : te;
                if (cfold && sF.ofold) {
                    fbase = orbit_base(g, sF, p + 1, [&](uint32_t j) { return j == p ? sv : my_m[j]; });
                } else if (cfold) {
                    // folded last level: f_base(s) = |window of L_F| - matched in it
                    const uint32_t jf = sF.jpos[0];
                    const uint32_t u = jf == p ? sv : my_m[jf];
                    const uint2 inf = sF.jdir[0] ? g.in_info[u] : g.out_info[u];
                    foff = inf.x;
                    fdeg = inf.y;
                    for (uint32_t msk = sF.gt_mask; msk; msk &= msk - 1) {
                        const uint32_t j = __ffs(msk) - 1;
                        flo = max(flo, (j == p ? sv : my_m[j]) + 1);
                    }
                    for (uint32_t msk = sF.lt_mask; msk; msk &= msk - 1) {
                        const uint32_t j = __ffs(msk) - 1;
                        fhi = min(fhi, j == p ? sv : my_m[j]);
                    }
                    const uint32_t *fl = g.adj + foff;
                    const uint32_t ws = flo ? lbound(fl, fdeg, flo) : 0;
                    const uint32_t we = fhi != kFullMask ? lbound(fl, fdeg, fhi) : fdeg;
                    uint32_t sub = 0;
                    for (uint32_t j = 0; j <= p; ++j) {
                        const uint32_t mj = j == p ? sv : my_m[j];
                        if (mj >= flo && mj < fhi && (((sF.guar_mask >> j) & 1u) || contains(fl, fdeg, mj))) ++sub;
                    }
                    fbase = (we > ws ? we - ws : 0) - sub;
                }
                if (MODE == kBytesMode || tally) {
                    const unsigned long long by = 12 + 4ull * nit + uint64_t(nit) * 4 * probes(iters ? ds : nS) +
                                                  (sig_c ? 8ull * nit : 0) +
                                                  (cfold ? 8 + 4ull * (p + 1) * probes(fdeg) : 0);
                    if (MODE == kBytesMode) local += by;
                    else tb += by;
                }
            }
            if (MODE == kBytesMode) return;
            uint32_t incl = nit;
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(kFullMask, incl, o);
                if (lane >= o) incl += y;
            }
            const uint32_t ftotal = __shfl_sync(kFullMask, incl, 31);
            const uint32_t excl = incl - nit;
            uint32_t gal_owner = kFullMask, gal = 0;
            for (uint32_t fstep = 0; fstep < ftotal; fstep += 32) {
                const uint32_t f = fstep + lane;
                uint32_t owner = 0;
                #pragma unroll
                for (int step = 16; step; step >>= 1) {
                    const uint32_t probe = __shfl_sync(kFullMask, incl, int(owner + step - 1));
                    if (probe <= f) owner += step;
                }
                owner = min(owner, 31u);
                const int ow = int(owner);
                const uint32_t o_excl = __shfl_sync(kFullMask, excl, ow);
                const uint32_t o_sv = __shfl_sync(kFullMask, sv, ow);
                const uint32_t o_itb = __shfl_sync(kFullMask, itb, ow);
                const uint32_t o_ooff = __shfl_sync(kFullMask, ooff, ow);
                const uint32_t o_ostart = __shfl_sync(kFullMask, ostart, ow);
                const uint32_t o_oend = __shfl_sync(kFullMask, oend, ow);
                const uint32_t o_iters = __shfl_sync(kFullMask, iters, ow);
                uint32_t o_fbase = 0, o_foff = 0, o_fdeg = 0, o_flo = 0, o_fhi = 0;
                if (cfold) o_fbase = __shfl_sync(kFullMask, fbase, ow);
                if (cfold && !sF.ofold) {  // the plain fold's list and window
                    o_foff = __shfl_sync(kFullMask, foff, ow);
                    o_fdeg = __shfl_sync(kFullMask, fdeg, ow);
                    o_flo = __shfl_sync(kFullMask, flo, ow);
                    o_fhi = __shfl_sync(kFullMask, fhi, ow);
                }
                bool ok = f < ftotal;
                if (owner != gal_owner) {
                    gal_owner = owner;
                    gal = o_ostart;
                }
                uint32_t t = 0;
                if (ok) {
                    const uint32_t y = f - o_excl;
                    if (o_iters) {
                        t = S[o_itb + y];
                        const uint32_t *Lo = g.adj + o_ooff;
                        const uint32_t pos = lbound_from(Lo, o_oend, gal, t);
                        gal = pos;
                        ok = pos < o_oend && __ldg(Lo + pos) == t;
                    } else {
                        t = __ldg(g.adj + o_itb + y);
                        const uint32_t pos = lbound_from(S, o_oend, gal, t);
                        gal = pos;
                        ok = pos < o_oend && S[pos] == t;
                    }
                }
                if (ok && t == o_sv) ok = false;
                if (ok && extra)
                    for (uint32_t tt = 0; tt < sC.nj; ++tt)
                        if ((extra >> tt) & 1u)
                            if (!contains(g.adj + xoff[warp][tt], xdeg[warp][tt], t)) { ok = false; break; }
                if (ok && sig_c) {
                    const uint2 o = g.out_info[t], i2 = g.in_info[t];
                    ok = i2.y >= sC.qin && o.y >= sC.qout;
                }
                if (ok) {
                    ++local_c;
                    if (cfold && sF.ofold) {
                        local += orbit_weight(g, sF, c, o_fbase, t, loops);
                    } else if (cfold) {
                        const bool h = t >= o_flo && t < o_fhi && (fguar_t || contains(g.adj + o_foff, o_fdeg, t));
                        local += o_fbase - (h ? 1u : 0u);
                    } else {
                        ++local;
                    }
                }
            }
            __syncwarp();
            return;
        }
        // a list of c on p itself: one s at a time, lane-parallel over t
        const uint32_t iend = min(i0 + 32, ns);
        for (uint32_t i = i0; i < iend; ++i) {
            const uint32_t sv = S[i];
            const uint2 is = sC.jdir[tp] ? g.in_info[sv] : g.out_info[sv];
            const uint32_t *Ls = g.adj + is.x;
            const uint32_t ds = is.y;
            uint32_t lo_t = lo_c, hi_t = hi_c;
            if (c_gt_s) lo_t = max(lo_t, sv + 1);
            if (c_lt_s) hi_t = min(hi_t, sv);
            const uint32_t ts = lo_t ? lbound(S, ns, lo_t) : 0;
            const uint32_t te = hi_t != kFullMask ? lbound(S, ns, hi_t) : ns;
            if (ts >= te) continue;
            __syncwarp();
            if (uint32_t(lane) < sC.nj && ((extra >> lane) & 1u) && sC.jpos[lane] == p) {
                const uint2 inf = sC.jdir[lane] ? g.in_info[sv] : g.out_info[sv];
                xoff[warp][lane] = inf.x;
                xdeg[warp][lane] = inf.y;
            }
            uint32_t fbase = 0, fdeg = 0, flo = 0, fhi = kFullMask;
            const uint32_t *fl = nullptr;
            if (cfold && sF.ofold) {
                fbase = orbit_base(g, sF, p + 1, [&](uint32_t j) { return j == p ? sv : my_m[j]; });
            } else if (cfold) {
                const uint32_t jf = sF.jpos[0];
                const uint32_t u = jf == p ? sv : my_m[jf];
                const uint2 inf = sF.jdir[0] ? g.in_info[u] : g.out_info[u];
                fl = g.adj + inf.x;
                fdeg = inf.y;
                for (uint32_t msk = sF.gt_mask; msk; msk &= msk - 1) {
                    const uint32_t j = __ffs(msk) - 1;
                    flo = max(flo, (j == p ? sv : my_m[j]) + 1);
                }
                for (uint32_t msk = sF.lt_mask; msk; msk &= msk - 1) {
                    const uint32_t j = __ffs(msk) - 1;
                    fhi = min(fhi, j == p ? sv : my_m[j]);
                }
                const uint32_t ws = flo ? lbound(fl, fdeg, flo) : 0;
                const uint32_t we = fhi != kFullMask ? lbound(fl, fdeg, fhi) : fdeg;
                bool hit = false;
                if (uint32_t(lane) <= p) {
                    const uint32_t mj = uint32_t(lane) == p ? sv : my_m[lane];
                    hit = mj >= flo && mj < fhi && (((sF.guar_mask >> lane) & 1u) || contains(fl, fdeg, mj));
                }
                fbase = (we > ws ? we - ws : 0) - __popc(__ballot_sync(kFullMask, hit));
            }
            __syncwarp();
            const uint32_t ls0 = lo_t ? lbound(Ls, ds, lo_t) : 0;
            const uint32_t ls1 = hi_t != kFullMask ? lbound(Ls, ds, hi_t) : ds;
            const uint32_t nS = te - ts, nL = ls1 > ls0 ? ls1 - ls0 : 0;
            const bool iterS = nS <= nL;
            const uint32_t nit = iterS ? nS : nL;
            if (MODE == kBytesMode || tally) {
                const unsigned long long by = 12 + 4ull * nit + uint64_t(nit) * 4 * probes(iterS ? ds : nS) +
                                              (sig_c ? 8ull * nit : 0) + (cfold ? 8 + 4ull * (p + 1) * probes(fdeg) : 0);
                if (lane == 0) {
                    if (MODE == kBytesMode) local += by;
                    else tb += by;
                }
                if (MODE == kBytesMode) continue;
            }
            uint32_t gal = iterS ? ls0 : ts;
            for (uint32_t y0 = 0; y0 < nit; y0 += 32) {
                const uint32_t y = y0 + lane;
                bool ok = y < nit;
                uint32_t t = 0;
                if (ok) {
                    if (iterS) {
                        t = S[ts + y];
                        const uint32_t pos = lbound_from(Ls, ls1, gal, t);
                        gal = pos;
                        ok = pos < ls1 && __ldg(Ls + pos) == t;
                    } else {
                        t = __ldg(Ls + ls0 + y);
                        const uint32_t pos = lbound_from(S, te, gal, t);
                        gal = pos;
                        ok = pos < te && S[pos] == t;
                    }
                }
                if (ok && t == sv) ok = false;
                if (ok && extra)
                    for (uint32_t tt = 0; tt < sC.nj; ++tt)
                        if ((extra >> tt) & 1u)
                            if (!contains(g.adj + xoff[warp][tt], xdeg[warp][tt], t)) { ok = false; break; }
                if (ok && sig_c) {
                    const uint2 o = g.out_info[t], i2 = g.in_info[t];
                    ok = i2.y >= sC.qin && o.y >= sC.qout;
                }
                if (ok) {
                    ++local_c;
                    if (cfold && sF.ofold) {
                        local += orbit_weight(g, sF, c, fbase, t, loops);
                    } else if (cfold) {
                        const bool h = t >= flo && t < fhi && (fguar_t || contains(fl, fdeg, t));
                        local += fbase - (h ? 1u : 0u);
                    } else {
                        ++local;
                    }
                }
            }
        }
        __syncwarp();
    };

    // Level c over all pairs of a parent whose S fits tS (phase 1).  A pair
    // (s, t) of S counts when t lies in s's list, inside s's window (t > s
    // or t < s when the plan orders them; t != s otherwise), and passes the
    // tests that depend on t alone (window of the positions below p, the
    // extra lists, the signature); its weight splits as A(s) + B(t):
    //   no fold:     1 + 0;
    //   orbit fold:  (orbit base with s at p) - #orbit positions below c,
    //                plus, when c is in the orbit, |L(t)| - c - [t loops];
    //   plain fold:  f_base(s) - [t in the fold's window and list], the fold's
    //                list and window fixed by the positions below p
    //                (walk_ok is set only then).
    // The admissible t go into a hash table in shared memory (buckets of
    // four keys read with one 128-bit load; each slot keeps B(t) and t's
    // index in S).  Each s's list window is then streamed with 128-bit
    // loads: the windows of 32 vertices s (one per lane, each lane also
    // holding its A(s)) form one sequence of 16-byte quads spread over the
    // lanes, two quads per lane per step (owner found by a binary search
    // over the lanes' inclusive scan), and each of the four list entries of
    // a quad is looked up in the table -- coalesced global reads and
    // shared-memory probes instead of a search in a list and a gather of
    // the pendant's weight per pair.
    auto pair_walk = [&](uint32_t ns, uint32_t lo_c, uint32_t hi_c) {
        uint32_t *const S = tS[warp];
        const long long akc = (cfold && sF.ofold) ? __popc(sF.ofold & ((1u << c) - 1)) : 0;
        const bool c_in_orbit = cfold && sF.ofold && ((sF.ofold >> c) & 1u);
        const bool p_in_orbit = cfold && sF.ofold && ((sF.ofold >> p) & 1u);
        // plain fold: the fold's list and window, fixed for this parent
        uint32_t f_off = 0, f_deg = 0, f_lo = 0, f_hi = kFullMask, f_ws = 0, f_we = 0, f_sub = 0;
        if (cfold && !sF.ofold) {
            const uint32_t u = my_m[sF.jpos[0]];
            const uint2 inf = sF.jdir[0] ? g.in_info[u] : g.out_info[u];
            f_off = inf.x;
            f_deg = inf.y;
            for (uint32_t msk = sF.gt_mask & below; msk; msk &= msk - 1) f_lo = max(f_lo, my_m[__ffs(msk) - 1] + 1);
            for (uint32_t msk = sF.lt_mask & below; msk; msk &= msk - 1) f_hi = min(f_hi, my_m[__ffs(msk) - 1]);
            const uint32_t *fl = g.adj + f_off;
            f_ws = f_lo ? lbound(fl, f_deg, f_lo) : 0;
            f_we = f_hi != kFullMask ? lbound(fl, f_deg, f_hi) : f_deg;
            for (uint32_t j = 0; j < p; ++j) {
                const uint32_t mj = my_m[j];
                if (mj >= f_lo && mj < f_hi && (((sF.guar_mask >> j) & 1u) || contains(fl, f_deg, mj))) ++f_sub;
            }
        }
        // orbit fold: the part of the orbit base fixed by the positions below
        // p (the lists of the orbit positions x < p, minus the members the
        // positions below p put there)
        uint32_t ob_par = 0;
        const uint32_t ob_low = (cfold && sF.ofold) ? (sF.ofold & below) : 0;
        for (uint32_t xm = ob_low; xm; xm &= xm - 1) {
            const uint32_t x = __ffs(xm) - 1;
            const uint2 inf = sF.jdir[0] ? g.in_info[my_m[x]] : g.out_info[my_m[x]];
            uint32_t sub = 0;
            for (uint32_t j = 0; j < p; ++j)
                if (((sF.oguar[x] >> j) & 1u) || contains(g.adj + inf.x, inf.y, my_m[j])) ++sub;
            ob_par += inf.y - sub;
        }
        // the table: buckets of 4 slots (one 128-bit shared load), a power of
        // two of at least one bucket per two vertices of S, 8..kHS/4; a full
        // bucket continues in the next one
        uint32_t lg = 3;
        while ((1u << lg) * 2 < ns && (1u << lg) < kHS / 4) ++lg;
        const uint32_t bmask = (1u << lg) - 1;
        const uint32_t hshift = 32 - lg;
        uint4 *const HK4 = tHK[warp];
        uint32_t *const HK = reinterpret_cast<uint32_t *>(tHK[warp]);
        uint8_t *const HI = tHI[warp];
        int32_t *const HB = tHB[warp];
        const bool need_idx = !c_gt_s && !c_lt_s && loops;
        // dense core path for rows s in the core: every t > s is then in the
        // core too, and s's pairs are popcounts of its bitmap row against
        // the admissible t (needs t > s, no extra lists, and B(t) from t's
        // degree alone)
        const bool core_rows = g.core_bits && c_gt_s && !extra && (!cfold || (sF.ofold && !loops));
        // the table serves rows below the core only
        const bool table = !core_rows || S[0] < g.core0;
        uint32_t *const SV = tSV[warp];
        if (core_rows) SV[lane] = 0;
        if (table)
            for (uint32_t x = lane; x <= bmask; x += 32) HK4[x] = make_uint4(kFullMask, kFullMask, kFullMask, kFullMask);
        __syncwarp();
        // the admissible t, with B(t), into the table
        uint32_t nv = 0;
        for (uint32_t i0 = 0; i0 < ns; i0 += 32) {
            const uint32_t i = i0 + lane;
            bool ok = i < ns;
            const uint32_t v = ok ? S[i] : 0;
            if (ok) {
                ok = v >= lo_c && v < hi_c;
                if (ok && extra)
                    for (uint32_t tt = 0; tt < sC.nj; ++tt)
                        if ((extra >> tt) & 1u)
                            if (!contains(g.adj + xoff[warp][tt], xdeg[warp][tt], v)) { ok = false; break; }
                if (ok && sig_c) {
                    const uint2 o = g.out_info[v], i2 = g.in_info[v];
                    ok = i2.y >= sC.qin && o.y >= sC.qout;
                }
            }
            if (ok && core_rows && v >= g.core0) {
                const uint32_t u = v - g.core0;
                atomicOr(&SV[u >> 5], 1u << (u & 31));
            }
            if (ok && table) {
                int32_t b = 0;
                if (c_in_orbit) {
                    if (tally) tb += 8;
                    const uint2 vi = sF.jdir[0] ? g.in_info[v] : g.out_info[v];
                    b = int32_t(vi.y) - int32_t(c) - ((loops && contains(g.adj + vi.x, vi.y, v)) ? 1 : 0);
                } else if (cfold && !sF.ofold) {
                    const bool h = v >= f_lo && v < f_hi && (fguar_t || contains(g.adj + f_off, f_deg, v));
                    b = h ? -1 : 0;
                }
                uint32_t bk = (v * 2654435769u) >> hshift;
                while (true) {
                    uint32_t slot = kFullMask;
                    #pragma unroll
                    for (uint32_t q = 0; q < 4; ++q)
                        if (slot == kFullMask && atomicCAS(&HK[bk * 4 + q], kFullMask, v) == kFullMask) slot = bk * 4 + q;
                    if (slot != kFullMask) {
                        HI[slot] = uint8_t(i);
                        HB[slot] = b;
                        break;
                    }
                    bk = (bk + 1) & bmask;
                }
            }
            nv += __popc(__ballot_sync(kFullMask, ok));
        }
        if (nv == 0) return;
        __syncwarp();
        long long sum = 0;
        unsigned long long hits = 0;
        const uint4 *const adj4 = reinterpret_cast<const uint4 *>(g.adj);
        for (uint32_t r0 = 0; r0 < ns; r0 += 32) {
            // this lane's row: s = S[r0 + lane], its list window as quads and
            // its term A(s)
            const uint32_t i = r0 + lane;
            uint32_t ea = 0, eb = 0, nq = 0, arow = 1;
            if (i < ns) {
                const uint32_t sv = S[i];
                {
                    // A(s): the orbit base with s at p (orbit_base's sum, the
                    // parent's part computed once), or the plain fold's base
                    if (cfold && sF.ofold) {
                        arow = ob_par;
                        for (uint32_t xm = ob_low; xm; xm &= xm - 1) {
                            const uint32_t x = __ffs(xm) - 1;
                            if ((sF.oguar[x] >> p) & 1u) {
                                --arow;
                            } else {
                                const uint2 xi = sF.jdir[0] ? g.in_info[my_m[x]] : g.out_info[my_m[x]];
                                if (contains(g.adj + xi.x, xi.y, sv)) --arow;
                            }
                        }
                        if (p_in_orbit) {
                            const uint2 vi = sF.jdir[0] ? g.in_info[sv] : g.out_info[sv];
                            uint32_t sub = (((sF.oguar[p] >> p) & 1u) || (loops && contains(g.adj + vi.x, vi.y, sv)))
                                               ? 1u : 0u;
                            for (uint32_t j = 0; j < p; ++j)
                                if (((sF.oguar[p] >> j) & 1u) || contains(g.adj + vi.x, vi.y, my_m[j])) ++sub;
                            arow += vi.y - sub;
                        }
                    } else if (cfold) {
                        const bool in = sv >= f_lo && sv < f_hi &&
                                        (((sF.guar_mask >> p) & 1u) || contains(g.adj + f_off, f_deg, sv));
                        arow = (f_we > f_ws ? f_we - f_ws : 0) - f_sub - (in ? 1u : 0u);
                    }
                }
                if (core_rows && sv >= g.core0) {
                    // a core row: t ranges over the admissible core bits
                    // above s in s's bitmap row
                    const uint32_t si = sv - g.core0;
                    const uint4 *rowp = reinterpret_cast<const uint4 *>(g.core_bits + size_t(si) * (kCore / 32));
                    const uint32_t w0 = si >> 5;
                    uint32_t cnt = 0;
                    long long dsum = 0;
                    for (uint32_t q = w0 >> 2; q < kCore / 128; ++q) {
                        const uint4 r4 = __ldg(rowp + q);
                        const uint32_t rw[4] = {r4.x, r4.y, r4.z, r4.w};
                        #pragma unroll
                        for (uint32_t k = 0; k < 4; ++k) {
                            const uint32_t j = 4 * q + k;
                            if (j < w0) continue;
                            uint32_t w = rw[k] & SV[j];
                            if (j == w0) w &= ~((2u << (si & 31)) - 1u);
                            cnt += __popc(w);
                            if (c_in_orbit)
                                for (; w; w &= w - 1) dsum += g.out_info[g.core0 + 32 * j + __ffs(w) - 1].y;
                        }
                    }
                    // the row's bitmap words from s's own word on, and t's
                    // degree per hit (orbit fold)
                    if (tally) tb += 8 + 16ull * (kCore / 128 - (w0 >> 2)) + (c_in_orbit ? 8ull * cnt : 0);
                    if (cnt) {
                        hits += cnt;
                        // B(t) = |L(t)| - c for the orbit fold's pendant (no self-loops here)
                        sum += (long long)cnt * ((long long)arow - akc) + (c_in_orbit ? dsum - (long long)cnt * c : 0);
                    }
                } else {
                    const uint2 is = sC.jdir[tp] ? g.in_info[sv] : g.out_info[sv];
                    const uint32_t *Ls = g.adj + is.x;
                    uint32_t lo_v = lo_c, hi_v = hi_c;
                    if (c_gt_s) lo_v = max(lo_v, sv + 1);
                    if (c_lt_s) hi_v = min(hi_v, sv);
                    const bool sdir = sC.jdir[tp] != 0;
                    const uint32_t p0 = lo_v ? lbound_own(g, sdir, sv, Ls, is.y, lo_v, loops) : 0;
                    const uint32_t p1 = hi_v != kFullMask ? lbound_own(g, sdir, sv, Ls, is.y, hi_v, loops) : is.y;
                    if (p1 > p0) {
                        ea = is.x + p0;
                        eb = is.x + p1;
                        nq = ((eb + 3) >> 2) - (ea >> 2);
                    }
                    // s's info, its window bound, the window's quads
                    if (tally) tb += 12 + 16ull * nq;
                }
            }
            uint32_t incl = nq;
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(kFullMask, incl, o);
                if (lane >= o) incl += y;
            }
            const uint32_t qtotal = __shfl_sync(kFullMask, incl, 31);
            const uint32_t excl = incl - nq;
            // two quads per lane per step (more loads in flight)
            for (uint32_t fstep = 0; fstep < qtotal; fstep += 64) {
                uint32_t quad[2], qea[2], qeb[2], qoi[2], qa[2];
                bool have[2];
                #pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t f = fstep + 32 * h + lane;
                    uint32_t owner = 0;
                    #pragma unroll
                    for (int step = 16; step; step >>= 1) {
                        const uint32_t probe = __shfl_sync(kFullMask, incl, int(owner + step - 1));
                        if (probe <= f) owner += step;
                    }
                    owner = min(owner, 31u);
                    const int ow = int(owner);
                    const uint32_t o_excl = __shfl_sync(kFullMask, excl, ow);
                    qea[h] = __shfl_sync(kFullMask, ea, ow);
                    qeb[h] = __shfl_sync(kFullMask, eb, ow);
                    qa[h] = __shfl_sync(kFullMask, arow, ow);
                    have[h] = f < qtotal;
                    qoi[h] = r0 + owner;
                    quad[h] = (qea[h] >> 2) + (f - o_excl);
                }
                uint4 xq[2];
                #pragma unroll
                for (int h = 0; h < 2; ++h) xq[h] = have[h] ? __ldg(adj4 + quad[h]) : make_uint4(0, 0, 0, 0);
                #pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if (!have[h]) continue;
                    const uint32_t e0 = quad[h] << 2;
                    const uint32_t vals[4] = {xq[h].x, xq[h].y, xq[h].z, xq[h].w};
                    uint32_t cnt = 0;
                    long long bs = 0;
                    #pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const uint32_t e = e0 + uint32_t(k);
                        if (e < qea[h] || e >= qeb[h]) continue;
                        const uint32_t v = vals[k];
                        uint32_t bk = (v * 2654435769u) >> hshift;
                        while (true) {
                            const uint4 kk = HK4[bk];
                            const uint32_t eq = (kk.x == v ? 1u : 0u) | (kk.y == v ? 2u : 0u) |
                                                (kk.z == v ? 4u : 0u) | (kk.w == v ? 8u : 0u);
                            if (eq) {
                                const uint32_t slot = bk * 4 + __ffs(eq) - 1;
                                // t == s only when s lists itself (a data self-loop)
                                if (!need_idx || HI[slot] != qoi[h]) {
                                    ++cnt;
                                    bs += HB[slot];
                                }
                                break;
                            }
                            if (kk.w == kFullMask) break;  // slots fill in order: an empty slot ends the chain
                            bk = (bk + 1) & bmask;
                        }
                    }
                    if (cnt) {
                        hits += cnt;
                        sum += (long long)cnt * ((long long)qa[h] - akc) + bs;
                    }
                }
            }
        }
        local += (unsigned long long)sum;
        local_c += hits;
    };

    while (true) {
        uint32_t gi = 0;
        if (lane == 0) gi = past_deadline(rp, deadline) ? total : atomicAdd(cursor, 1u);
        gi = __shfl_sync(kFullMask, gi, 0);
        if (gi >= total) break;
        // phase 2: work item gi is group grp of deferred parent b
        uint32_t q0, b = 0, grp = 0;
        if (!phase2) {
            q0 = pa + gi;
        } else {
            uint32_t lo = 0, hi = nbig - 1;  // first b with pref[b] > gi
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (big.pref[mid] > gi) hi = mid; else lo = mid + 1;
            }
            b = lo;
            grp = gi - (b ? big.pref[b - 1] : 0);
            q0 = big.gi[b];
        }
        if (lane == 0) {  // matched vertices of the parent at level p-1
            my_m[p - 1] = s_vert[p - 1][q0];
            if (p >= 2) {
                uint32_t q = s_par[p - 1][q0];
                if (q != cached_q) {
                    cached_q = q;
                    for (int j = int(p) - 2; j >= 0; --j) {
                        my_m[j] = s_vert[j][q];
                        if (j > 0) q = s_par[j][q];
                    }
                }
            }
        }
        __syncwarp();
        const uint32_t *S = row;
        uint32_t ns = 0;
        if (!phase2) {
            // level p: joined lists, the shortest supplies S
            const uint32_t njp = sP.nj;
            uint32_t md = kFullMask, mo = 0;
            if (uint32_t(lane) < njp) {
                const uint32_t u = my_m[sP.jpos[lane]];
                const uint2 inf = sP.jdir[lane] ? g.in_info[u] : g.out_info[u];
                mo = inf.x;
                md = inf.y;
                joff[warp][lane] = mo;
                jdeg[warp][lane] = md;
                jver[warp][lane] = u;
            }
            uint32_t bd = md, bl = uint32_t(lane);
            #pragma unroll
            for (int o = 16; o; o >>= 1) {
                const uint32_t od = __shfl_xor_sync(kFullMask, bd, o), ol = __shfl_xor_sync(kFullMask, bl, o);
                if (od < bd || (od == bd && ol < bl)) { bd = od; bl = ol; }
            }
            const uint32_t moff = __shfl_sync(kFullMask, mo, int(bl)), mdeg = njp ? bd : 0, tmin = bl;
            __syncwarp();
            uint32_t lo = 0, hi = kFullMask;
            for (uint32_t msk = sP.gt_mask; msk; msk &= msk - 1) lo = max(lo, my_m[__ffs(msk) - 1] + 1);
            for (uint32_t msk = sP.lt_mask; msk; msk &= msk - 1) hi = min(hi, my_m[__ffs(msk) - 1]);
            const uint32_t *mlist = g.adj + moff;
            const uint32_t mu = njp ? my_m[sP.jpos[tmin]] : 0;  // the vertex whose list supplies S
            const bool mdir = njp && sP.jdir[tmin];
            uint32_t s0 = kFullMask;
            if (lo && p >= 2 && rp->pos_lvl == p - 1 && lo == my_m[p - 1] + 1) {
                // the window starts right after the parent's own vertex: when
                // that vertex was drawn from this very list, its offset is known
                const uint32_t apos = rp->ub[p - 1][q0];
                if (apos >= moff && apos - moff < mdeg) s0 = apos - moff + 1;
            }
            if (s0 == kFullMask) s0 = lo ? lbound_own(g, mdir, mu, mlist, mdeg, lo, loops) : 0;
            const uint32_t e0 = hi != kFullMask ? lbound_own(g, mdir, mu, mlist, mdeg, hi, loops) : mdeg;
            // this lane's candidates rise, so its lower bounds in the first
            // two other lists rise too: gallop from the last
            uint32_t gp0 = 0, gp1 = 0;
            // S goes to shared memory when the pair walk will read it (the
            // other paths search S with global-memory loads)
            uint32_t *const small = walk_ok ? tS[warp] : row;
            for (uint32_t x0 = s0; x0 < e0; x0 += 32) {
                const uint32_t x = x0 + lane;
                bool ok = x < e0;
                const uint32_t v = ok ? __ldg(mlist + x) : 0;
                if (ok)
                    for (uint32_t j = 0; j < p; ++j)
                        if (v == my_m[j]) { ok = false; break; }
                if (ok) {
                    const uint2 o = g.out_info[v], i = g.in_info[v];
                    ok = i.y >= sP.qin && o.y >= sP.qout;
                }
                if (ok) {
                    uint32_t r = 0;
                    for (uint32_t t = 0; t < njp; ++t) {
                        if (t == tmin) continue;
                        const uint32_t *lst = g.adj + joff[warp][t];
                        const uint32_t len2 = jdeg[warp][t];
                        const uint32_t ut = jver[warp][t];
                        if (g.core_bits && ut >= g.core0 && v >= g.core0) {
                            // both in the dense core: one bit of ut's row
                            const uint32_t bi = v - g.core0;
                            const uint32_t w = __ldg(g.core_bits + size_t(ut - g.core0) * (kCore / 32) + (bi >> 5));
                            if (!((w >> (bi & 31)) & 1u)) { ok = false; break; }
                            continue;
                        }
                        if (r < 2) {
                            const uint32_t pos = lbound_from(lst, len2, r == 0 ? gp0 : gp1, v);
                            if (r == 0) gp0 = pos; else gp1 = pos;
                            if (pos >= len2 || __ldg(lst + pos) != v) { ok = false; break; }
                        } else if (!contains(lst, len2, v)) {
                            ok = false;
                            break;
                        }
                        ++r;
                    }
                }
                const unsigned m = __ballot_sync(kFullMask, ok);
                if (ok) {
                    const uint32_t idx = ns + __popc(m & lanemask_lt);
                    if (idx < kTS) small[idx] = v;
                    else row[idx] = v;
                }
                ns += __popc(m);
                if ((MODE == kBytesMode || tally) && lane == 0) {
                    uint32_t per = 8;
                    for (uint32_t t = 0; t < njp; ++t)
                        if (t != tmin) per += 4 * probes(jdeg[warp][t]);
                    const unsigned long long by = 4ull * min(32u, e0 - x0) + uint64_t(min(32u, e0 - x0)) * per;
                    if (MODE == kBytesMode) local += by;
                    else tb += by;
                }
            }
            __syncwarp();
            if (tally && lane == 0) tb += 8ull * p + 8ull * njp + 4ull * ns;
            if (MODE == kCountMode && ns > split) {
                // defer: save S in the pool for phase 2 (or keep it here when full)
                unsigned long long off = 0;
                uint32_t e = kFullMask;
                if (lane == 0 && big.n[1] < big.pool_words) {
                    off = atomicAdd(&big.n[1], (unsigned long long)ns);
                    if (off + ns <= big.pool_words) {
                        const unsigned long long e64 = atomicAdd(&big.n[0], 1ull);
                        if (e64 < big.cap) e = uint32_t(e64);
                    }
                }
                e = __shfl_sync(kFullMask, e, 0);
                off = __shfl_sync(kFullMask, off, 0);
                if (e != kFullMask) {
                    for (uint32_t i = lane; i < ns; i += 32) big.pool[off + i] = i < kTS ? small[i] : row[i];
                    if (lane == 0) {
                        big.gi[e] = q0;
                        big.soff[e] = uint32_t(off);
                        big.ns[e] = ns;
                    }
                    __syncwarp();
                    continue;
                }
            }
            if (lane == 0) {
                local_p += ns;
                if (MODE == kBytesMode) local += 8ull * p + 8ull * njp + 4ull * ns;
            }
            if (walk_ok && ns > kTS) {
                // the first kTS entries join the rest in the scratch row
                for (uint32_t i = lane; i < kTS; i += 32) row[i] = small[i];
                __syncwarp();
            }
        } else {
            S = big.pool + big.soff[b];
            ns = big.ns[b];
            if (lane == 0 && grp == 0) local_p += ns;
        }
        // extra lists of level c on positions below p: fixed for this parent
        if (uint32_t(lane) < sC.nj && ((extra >> lane) & 1u) && sC.jpos[lane] < p) {
            const uint32_t u = my_m[sC.jpos[lane]];
            const uint2 inf = sC.jdir[lane] ? g.in_info[u] : g.out_info[u];
            xoff[warp][lane] = inf.x;
            xdeg[warp][lane] = inf.y;
        }
        __syncwarp();
        // level c over the vertices s of S
        uint32_t lo_c = 0, hi_c = kFullMask;
        for (uint32_t msk = sC.gt_mask & below; msk; msk &= msk - 1) lo_c = max(lo_c, my_m[__ffs(msk) - 1] + 1);
        for (uint32_t msk = sC.lt_mask & below; msk; msk &= msk - 1) hi_c = min(hi_c, my_m[__ffs(msk) - 1]);
        if (!phase2) {
            if (walk_ok && ns <= kTS) {
                if constexpr (walk_ok) pair_walk(ns, lo_c, hi_c);
                __syncwarp();
            } else
                for (uint32_t i0 = 0; i0 < ns; i0 += 32) group(S, ns, i0, lo_c, hi_c);
        } else {
            group(S, ns, grp * 32, lo_c, hi_c);
        }
    }
    #pragma unroll
    for (int o = 16; o; o >>= 1) {
        local += __shfl_xor_sync(kFullMask, local, o);
        local_c += __shfl_xor_sync(kFullMask, local_c, o);
    }
    if (lane == 0) {
        if (local) atomicAdd(acc, local);
        if (MODE == kCountMode) {
            if (local_c) atomicAdd(acc_c, local_c);
            if (local_p) atomicAdd(acc_p, local_p);
        }
    }
    if (tally) {
        #pragma unroll
        for (int o = 16; o; o >>= 1) tb += __shfl_xor_sync(kFullMask, tb, o);
        if (lane == 0 && tb) atomicAdd(acc_bytes, tb);
    }
}

// Inclusive prefix sum of the deferred parents' group counts (one block).
__global__ void __launch_bounds__(1024) k_fused_scan(FusedBig big) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    const unsigned long long n0 = big.n[0];
    const uint32_t n = n0 < big.cap ? uint32_t(n0) : big.cap;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (uint32_t base = 0; base < n; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        uint32_t v = i < n ? (big.ns[i] + 31) / 32 : 0, x = v;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(kFullMask, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t s = lane < int(blockDim.x / 32) ? wsum[lane] : 0;
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(kFullMask, s, o);
                if (lane >= o) s += y;
            }
            wsum[lane] = s;
        }
        __syncthreads();
        const uint32_t pre = carry + (w ? wsum[w - 1] : 0) + x;
        if (i < n) big.pref[i] = pre;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = pre;
        __syncthreads();
    }
}

// ---- chunk planner ------------------------------------------------------
// Tile sums of the child bounds of parents [pa, pb).
__global__ void k_tile_sums(const uint32_t *__restrict__ ub, uint32_t pa, uint32_t pb,
                            uint32_t tile, uint64_t *__restrict__ tsum,
                            unsigned long long *__restrict__ tmax) {
    __shared__ unsigned long long red[32];
    const uint32_t ntiles = (pb - pa + tile - 1) / tile;
    for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const uint32_t b = pa + t * tile, e = min(b + tile, pb);
        unsigned long long s = 0;
        for (uint32_t i = b + threadIdx.x; i < e; i += blockDim.x) s += ub[i];
        #pragma unroll
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x < 32) {
            s = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0;
            #pragma unroll
            for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
            if (threadIdx.x == 0) {
                tsum[t] = s;
                atomicMax(tmax, s);
            }
        }
        __syncthreads();
    }
}

// Chunk boundaries (tile indices): tile t opens a chunk when
// floor(prefix(t) / cap_eff) differs from tile t-1's; with cap_eff = cap -
// (max tile sum) every chunk's bound sum stays within cap.  One block.
__global__ void __launch_bounds__(1024)
k_plan(const uint64_t *__restrict__ tsum, uint32_t ntiles, unsigned long long cap_eff,
       uint32_t *__restrict__ bounds, uint32_t *__restrict__ nb_out) {
    __shared__ unsigned long long ws[32];
    __shared__ uint32_t wf[32];
    __shared__ unsigned long long carry;
    __shared__ uint32_t nb;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) { carry = 0; nb = 0; }
    __syncthreads();
    for (uint32_t base = 0; base < ntiles; base += blockDim.x) {
        const uint32_t t = base + threadIdx.x;
        const unsigned long long v = t < ntiles ? tsum[t] : 0;
        // inclusive block scan of v
        unsigned long long x = v;
        #pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) ws[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned long long w = lane < int(blockDim.x / 32) ? ws[lane] : 0;
            #pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(kFull, w, o);
                if (lane >= o) w += y;
            }
            ws[lane] = w;
        }
        __syncthreads();
        const unsigned long long incl = x + (warp ? ws[warp - 1] : 0) + carry;
        const unsigned long long excl = incl - v;
        bool flag = false;
        if (t < ntiles) {
            if (t == 0) flag = true;
            else {
                const unsigned long long prev_excl = excl - tsum[t - 1];
                flag = (excl / cap_eff) != (prev_excl / cap_eff);
            }
        }
        // ordered compaction of the flags
        const unsigned m = __ballot_sync(kFull, flag);
        if (lane == 0) wf[warp] = __popc(m);
        __syncthreads();
        uint32_t before = 0, tot = 0;
        for (int w = 0; w < int(blockDim.x / 32); ++w) {
            if (w < warp) before += wf[w];
            tot += wf[w];
        }
        if (flag) bounds[nb + before + __popc(m & ((1u << lane) - 1))] = t;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        if (threadIdx.x == 0) nb += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        bounds[nb] = ntiles;
        *nb_out = nb;
    }
}

int g_num_sms = 0;
int g_level_blocks[3] = {0, 0, 0};
int g_flat_blocks[3] = {0, 0, 0};
int g_fused_blocks[3] = {0, 0, 0};
int g_fused_walk_blocks = 0;
// CUTS_LEVEL_KERNEL=warp selects the warp-per-parent form (A/B comparisons)
bool g_use_flat = true;

int launch_geometry() {
    if (g_num_sms) return CUTS_OK;
    int dev = 0;
    CK(cudaGetDevice(&dev));
    CK(cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, dev));
    int b = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_level<kExpand>, kWarps * 32, 0));
    g_level_blocks[kExpand] = std::max(1, b) * g_num_sms;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_level<kCountMode>, kWarps * 32, 0));
    g_level_blocks[kCountMode] = std::max(1, b) * g_num_sms;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_level<kBytesMode>, kWarps * 32, 0));
    g_level_blocks[kBytesMode] = std::max(1, b) * g_num_sms;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_level_flat<kExpand>, kFW * 32, 0));
    g_flat_blocks[kExpand] = std::max(1, b) * g_num_sms;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_level_flat<kCountMode>, kFW * 32, 0));
    g_flat_blocks[kCountMode] = std::max(1, b) * g_num_sms;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_level_flat<kBytesMode>, kFW * 32, 0));
    g_flat_blocks[kBytesMode] = std::max(1, b) * g_num_sms;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_fused<kCountMode, false>, kZW * 32, 0));
    g_fused_blocks[kCountMode] = std::max(1, b) * g_num_sms;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_fused<kBytesMode, false>, kZW * 32, 0));
    g_fused_blocks[kBytesMode] = std::max(1, b) * g_num_sms;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_fused<kCountMode, true>, kZW * 32, 0));
    g_fused_walk_blocks = std::max(1, b) * g_num_sms;
    const char *kv = std::getenv("CUTS_LEVEL_KERNEL");
    g_use_flat = !(kv && std::strcmp(kv, "warp") == 0);
    return CUTS_OK;
}

// u32 scratch slots
enum : int { kSlotN0 = 0, kSlotErr = 1, kSlotNb = 2, kSlotOver = 3, kSlotOut = 8, kSlotCursor = 32, kSlots = 64 };
constexpr int kU64Stamp = 5;  // d_u64 slot: device clock at the start of a budgeted run
constexpr int kU64Scratch = 8;  // d_u64 slots 8..10: counts of the bytes pass (discarded)
constexpr int kU64Pair = 6;     // d_u64 slot: level k-2 size of a pendant-pair count
constexpr int kU64Slots = 16;

}  // namespace

// ---- upload -------------------------------------------------------------

// Allocates a DeviceGraph, builds its layout on the device from CSR arrays
// in host memory (layout.cu) and the engine's scratch.
static int device_graph_build(uint32_t n, const uint64_t *out_off, const uint32_t *out_adj,
                              const uint64_t *in_off, const uint32_t *in_adj, int sym_hint, bool validate,
                              int device, DeviceGraph **out) {
    *out = nullptr;
    CK(cudaSetDevice(device));
    auto *g = new DeviceGraph();
    g->device = device;
    auto fail = [&](cudaError_t e, const char *what) {
        device_graph_free(g);
        return set_error(CUTS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking))) return fail(e, "stream");
    {
        // the trie arena and the layout's scratch come from the device's
        // default pool; keep up to 32 GB of freed blocks there, so a graph
        // built after another one reuses its memory instead of mapping anew
        cudaMemPool_t pool = nullptr;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t keep = 32ull << 30;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    int rc = device_layout(n, out_off, out_adj, in_off, in_adj, sym_hint, validate, *g);
    if (rc) {
        device_graph_free(g);
        return rc;
    }
    if ((e = cudaMalloc(&g->d_u32, sizeof(uint32_t) * kSlots))) return fail(e, "scratch");
    if ((e = cudaMalloc(&g->d_u64, sizeof(unsigned long long) * kU64Slots))) return fail(e, "scratch");
    if ((e = cudaMalloc(&g->d_plan, sizeof(RunParams)))) return fail(e, "scratch");
    if ((e = cudaMallocHost(&g->h_u32, sizeof(uint32_t) * kSlots))) return fail(e, "pinned");
    if ((e = cudaMallocHost(&g->h_u64, sizeof(unsigned long long) * kU64Slots))) return fail(e, "pinned");
    if ((e = cudaMallocHost(&g->h_plan, sizeof(RunParams)))) return fail(e, "pinned");
    if ((e = cudaEventCreate(&g->ev0)) || (e = cudaEventCreate(&g->ev1))) return fail(e, "event");
    if ((e = cudaStreamSynchronize(g->stream))) return fail(e, "upload sync");
    // default arena: proportional to the graph, within [256 MB, 64 GB] and
    // at most 60% of the free memory
    size_t freeb = 0, totb = 0;
    cudaMemGetInfo(&freeb, &totb);
    double want = 384.0 * double(g->arcs) + 64.0 * n;
    want = std::max(want, 256.0 * (1 << 20));
    want = std::min(want, 64.0 * (1ull << 30));
    want = std::min(want, 0.6 * double(freeb));
    g->arena_bytes = size_t(want);
    g->arena_default = g->arena_bytes;
    *out = g;
    return CUTS_OK;
}

int device_graph_upload(const HostGraph &hg, int device, DeviceGraph **out) {
    return device_graph_build(hg.n, hg.out_off.data(), hg.out_adj.data(),
                              hg.symmetric ? nullptr : hg.in_off.data(), hg.symmetric ? nullptr : hg.in_adj.data(),
                              hg.symmetric ? 1 : 0, false, device, out);
}

int device_graph_from_csr(uint32_t n, const uint64_t *out_off, const uint32_t *out_adj, const uint64_t *in_off,
                          const uint32_t *in_adj, int device, DeviceGraph **out) {
    return device_graph_build(n, out_off, out_adj, in_off, in_adj, -1, true, device, out);
}

void device_graph_free(DeviceGraph *g) {
    if (!g) return;
    cudaSetDevice(g->device);
    if (g->stream) {
        // the arena and the layout's arrays go back to the device's pool,
        // after the work queued on the graph's stream
        if (g->in_info && g->in_info != g->out_info) cudaFreeAsync(g->in_info, g->stream);
        for (void *p : {static_cast<void *>(g->arena), static_cast<void *>(g->out_info),
                        static_cast<void *>(g->adj), static_cast<void *>(g->bwd_out),
                        static_cast<void *>(g->core_bits)})
            if (p) cudaFreeAsync(p, g->stream);
        cudaStreamSynchronize(g->stream);
    }
    cudaFree(g->d_u32);
    cudaFree(g->d_u64);
    cudaFree(g->d_plan);
    cudaFree(g->d_tiles);
    cudaFree(g->d_bounds);
    cudaFree(g->batch_vsorted);
    cudaFree(g->batch_pref);
    cudaFreeHost(g->h_u32);
    cudaFreeHost(g->h_u64);
    cudaFreeHost(g->h_plan);
    cudaFreeHost(g->h_bounds);
    if (g->ev0) cudaEventDestroy(g->ev0);
    if (g->ev1) cudaEventDestroy(g->ev1);
    if (g->stream) cudaStreamDestroy(g->stream);
    delete g;
}

// ---- driver -----------------------------------------------------------------

namespace {

struct Run {
    DeviceGraph &g;
    DevView view;
    RunParams *hp;        // pinned host copy
    RunParams *dp;        // device copy
    uint32_t k;
    uint64_t cap;         // entries per stored level >= 1
    uint32_t grain;
    bool bytes_mode;
    CountResult &res;
    bool dump = false;
    bool profile = false;
    double budget_ms = 0;
    std::chrono::steady_clock::time_point t_start = std::chrono::steady_clock::now();
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
    FILE *dump_file = nullptr;
    const Query *query = nullptr;
    uint64_t dumped = 0;

    int sync() {
        CK(cudaStreamSynchronize(g.stream));
        return CUTS_OK;
    }

    int ensure_tiles(size_t ntiles) {
        if (ntiles + 1 <= g.tiles_cap) return CUTS_OK;
        size_t nc = std::max(ntiles + 1, g.tiles_cap * 2);
        cudaFree(g.d_tiles);
        cudaFree(g.d_bounds);
        cudaFreeHost(g.h_bounds);
        g.d_tiles = nullptr; g.d_bounds = nullptr; g.h_bounds = nullptr; g.tiles_cap = 0;
        CK(cudaMalloc(&g.d_tiles, sizeof(uint64_t) * nc));
        CK(cudaMalloc(&g.d_bounds, sizeof(uint32_t) * nc));
        CK(cudaMallocHost(&g.h_bounds, sizeof(uint32_t) * nc));
        g.tiles_cap = nc;
        return CUTS_OK;
    }

    // Splits parents [pa, pb) of L_{lvl-1} into chunks whose child bounds fit cap.
    int plan_chunks(uint32_t lvl, uint32_t pa, uint32_t pb, std::vector<uint32_t> &cuts) {
        cuts.clear();
        if (uint64_t(pb - pa) * g.max_deg <= cap) { cuts = {pa, pb}; return CUTS_OK; }
        uint64_t tile = std::min<uint64_t>(kTile, cap / (2ull * std::max<uint32_t>(g.max_deg, 1)));
        if (tile == 0)
            return set_error(CUTS_ERR_CAPACITY, "level capacity below twice the maximum degree");
        const uint32_t ntiles = uint32_t((uint64_t(pb - pa) + tile - 1) / tile);
        int rc = ensure_tiles(ntiles);
        if (rc) return rc;
        CK(cudaMemsetAsync(g.d_u64 + 1, 0, sizeof(unsigned long long), g.stream));
        const uint32_t blocks = std::min<uint32_t>(ntiles, uint32_t(g_num_sms) * 16);
        k_tile_sums<<<blocks, 256, 0, g.stream>>>(hp->ub[lvl - 1], pa, pb, uint32_t(tile), g.d_tiles,
                                                 g.d_u64 + 1);
        CK(cudaMemcpyAsync(g.h_u64 + 1, g.d_u64 + 1, sizeof(unsigned long long), cudaMemcpyDeviceToHost, g.stream));
        res.launches++;
        int r2 = sync();
        if (r2) return r2;
        const unsigned long long tmax = g.h_u64[1];
        const unsigned long long cap_eff = cap - tmax;
        k_plan<<<1, 1024, 0, g.stream>>>(g.d_tiles, ntiles, cap_eff, g.d_bounds, g.d_u32 + kSlotNb);
        res.launches++;
        CK(cudaMemcpyAsync(g.h_u32 + kSlotNb, g.d_u32 + kSlotNb, sizeof(uint32_t), cudaMemcpyDeviceToHost, g.stream));
        r2 = sync();
        if (r2) return r2;
        const uint32_t nb = g.h_u32[kSlotNb];
        CK(cudaMemcpyAsync(g.h_bounds, g.d_bounds, sizeof(uint32_t) * (nb + 1), cudaMemcpyDeviceToHost, g.stream));
        r2 = sync();
        if (r2) return r2;
        for (uint32_t c = 0; c <= nb; ++c)
            cuts.push_back(uint32_t(std::min<uint64_t>(pa + uint64_t(g.h_bounds[c]) * tile, pb)));
        return CUTS_OK;
    }

    int launch_level(int mode, uint32_t lvl, uint32_t pa, uint32_t pb) {
        CK(cudaMemsetAsync(g.d_u32 + kSlotCursor, 0, sizeof(uint32_t), g.stream));
        uint32_t *out_n = g.d_u32 + kSlotOut + lvl;
        if (mode == kExpand) CK(cudaMemsetAsync(out_n, 0, sizeof(uint32_t), g.stream));
        const uint32_t work = pb - pa;
        const bool flat = g_use_flat && hp->plan.lv[lvl].nj <= uint32_t(kFJ);
        const uint32_t per_warp = flat ? 32 : grain;
        const uint32_t wpb = flat ? kFW : kWarps;
        const uint32_t warps_needed = (work + per_warp - 1) / per_warp;
        uint32_t blocks = std::min<uint32_t>(uint32_t(flat ? g_flat_blocks[mode] : g_level_blocks[mode]),
                                             (warps_needed + wpb - 1) / wpb);
        blocks = std::max<uint32_t>(blocks, 1);
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (profile) {
            CK(cudaEventCreate(&e0));
            CK(cudaEventCreate(&e1));
            CK(cudaEventRecord(e0, g.stream));
        }
        if (flat) {
            unsigned long long *acc = mode == kBytesMode ? g.d_u64 + 2 : g.d_u64;
            if (mode == kExpand)
                k_level_flat<kExpand><<<blocks, kFW * 32, 0, g.stream>>>(view, dp, lvl, pa, pb,
                    g.d_u32 + kSlotCursor, out_n, uint32_t(cap), g.d_u32 + kSlotErr, acc, nullptr, nullptr);
            else if (mode == kCountMode)
                k_level_flat<kCountMode><<<blocks, kFW * 32, 0, g.stream>>>(view, dp, lvl, pa, pb,
                    g.d_u32 + kSlotCursor, out_n, 0, g.d_u32 + kSlotErr, acc, g.d_u64 + 3, g.d_u64 + kU64Pair);
            else
                k_level_flat<kBytesMode><<<blocks, kFW * 32, 0, g.stream>>>(view, dp, lvl, pa, pb,
                    g.d_u32 + kSlotCursor, out_n, 0, g.d_u32 + kSlotErr, acc, nullptr, nullptr);
        } else if (mode == kExpand)
            k_level<kExpand><<<blocks, kWarps * 32, 0, g.stream>>>(view, dp, lvl, pa, pb, grain,
                g.d_u32 + kSlotCursor, out_n, uint32_t(cap), g.d_u32 + kSlotErr, g.d_u64);
        else if (mode == kCountMode)
            k_level<kCountMode><<<blocks, kWarps * 32, 0, g.stream>>>(view, dp, lvl, pa, pb, grain,
                g.d_u32 + kSlotCursor, out_n, 0, g.d_u32 + kSlotErr, g.d_u64);
        else
            k_level<kBytesMode><<<blocks, kWarps * 32, 0, g.stream>>>(view, dp, lvl, pa, pb, grain,
                g.d_u32 + kSlotCursor, out_n, 0, g.d_u32 + kSlotErr, g.d_u64 + 2);
        CK(cudaGetLastError());
        if (profile) {
            CK(cudaEventRecord(e1, g.stream));
            marks.push_back({mode, {e0, e1}});
        }
        res.launches++;
        return CUTS_OK;
    }

    // The fused count of levels p and p+1 over parents [pa, pb) of L_{p-1}:
    // phase 1 over the parents, then (counting) a scan of the parents it
    // deferred and phase 2 over their groups.
    int launch_fused(int mode, uint32_t p, uint32_t pa, uint32_t pb) {
        CK(cudaMemsetAsync(g.d_u32 + kSlotCursor, 0, sizeof(uint32_t), g.stream));
        uint32_t blocks = std::max<uint32_t>(1, std::min<uint32_t>(uint32_t(g_fused_blocks[mode]),
                                                                   (pb - pa + kZW - 1) / kZW));
        FusedBig fb;
        fb.n = reinterpret_cast<unsigned long long *>(hp->fuse_big);
        fb.cap = hp->fuse_big_cap;
        fb.gi = hp->fuse_big + 64;
        fb.soff = fb.gi + fb.cap;
        fb.ns = fb.soff + fb.cap;
        fb.pref = fb.ns + fb.cap;
        fb.pool = fb.pref + fb.cap;
        fb.pool_words = hp->fuse_pool_words;
        if (mode == kCountMode) CK(cudaMemsetAsync(fb.n, 0, 2 * sizeof(unsigned long long), g.stream));
        // CUTS_FUSE_SPLIT=<n> sets the deferral threshold (tests use small values)
        uint32_t split = g.fuse_split ? g.fuse_split : kBigS;
        if (const char *e = std::getenv("CUTS_FUSE_SPLIT")) split = uint32_t(std::strtoul(e, nullptr, 10));
        // the phase-1 pair walk covers the fused plans that order the
        // vertices at p and c (symmetry breaking: each pair of S once, and a
        // row's list window starts or ends at s), except an extra list of c
        // on p itself and a plain fold whose list or window moves with the
        // vertex at p; a plan without that order (every ordered pair, so a
        // row's window is s's whole list) keeps the per-pair intersection,
        // which iterates the shorter side.  CUTS_FUSE_WALK=0 turns the walk
        // off (A/B comparisons)
        uint32_t walk_ok = 1;
        {
            const LevelPlan &Lc = hp->plan.lv[p + 1];
            const LevelPlan &Lf = hp->plan.lv[p + 2 < k ? p + 2 : p + 1];
            if (!(((Lc.gt_mask | Lc.lt_mask) >> p) & 1u)) walk_ok = 0;
            for (uint32_t t = 0; t < Lc.nj; ++t)
                if (((Lc.fuse_extra >> t) & 1u) && Lc.jpos[t] == p) walk_ok = 0;
            if (Lc.fold && !Lf.ofold && (Lf.jpos[0] == p || (((Lf.gt_mask | Lf.lt_mask) >> p) & 1u))) walk_ok = 0;
            if (g.max_deg >= (1u << 31)) walk_ok = 0;
            const char *w = std::getenv("CUTS_FUSE_WALK");
            if (w && w[0] == '0') walk_ok = 0;
        }
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (profile) {
            CK(cudaEventCreate(&e0));
            CK(cudaEventCreate(&e1));
            CK(cudaEventRecord(e0, g.stream));
        }
        if (mode == kBytesMode && !walk_ok) {
            k_fused<kBytesMode, false><<<blocks, kZW * 32, 0, g.stream>>>(view, dp, p, pa, pb, 1, split,
                g.d_u32 + kSlotCursor, hp->fuse_scratch, hp->fuse_stride, fb, g.d_u64 + 2, nullptr, nullptr,
                nullptr);
            CK(cudaGetLastError());
            res.launches++;
        } else {
            // counting; the bytes pass of a walk plan runs the same launches
            // with their byte tally on and the counts sent to scratch slots
            const bool tal = mode == kBytesMode;
            unsigned long long *acc = tal ? g.d_u64 + kU64Scratch : g.d_u64;
            unsigned long long *acc_c = tal ? g.d_u64 + kU64Scratch + 1 : g.d_u64 + 3;
            unsigned long long *acc_p = tal ? g.d_u64 + kU64Scratch + 2 : g.d_u64 + 4;
            unsigned long long *acc_b = tal ? g.d_u64 + 2 : nullptr;
            if (tal) CK(cudaMemsetAsync(fb.n, 0, 2 * sizeof(unsigned long long), g.stream));
            const uint32_t wblocks =
                std::max<uint32_t>(1, std::min<uint32_t>(uint32_t(g_fused_walk_blocks), (pb - pa + kZW - 1) / kZW));
            if (walk_ok && tal)
                k_fused<kCountMode, true, true><<<wblocks, kZW * 32, 0, g.stream>>>(view, dp, p, pa, pb, 1, split,
                    g.d_u32 + kSlotCursor, hp->fuse_scratch, hp->fuse_stride, fb, acc, acc_c, acc_p, acc_b);
            else if (walk_ok)
                k_fused<kCountMode, true><<<wblocks, kZW * 32, 0, g.stream>>>(view, dp, p, pa, pb, 1, split,
                    g.d_u32 + kSlotCursor, hp->fuse_scratch, hp->fuse_stride, fb, acc, acc_c, acc_p, acc_b);
            else
                k_fused<kCountMode, false><<<blocks, kZW * 32, 0, g.stream>>>(view, dp, p, pa, pb, 1, split,
                    g.d_u32 + kSlotCursor, hp->fuse_scratch, hp->fuse_stride, fb, acc, acc_c, acc_p, acc_b);
            CK(cudaGetLastError());
            k_fused_scan<<<1, 1024, 0, g.stream>>>(fb);
            CK(cudaGetLastError());
            CK(cudaMemsetAsync(g.d_u32 + kSlotCursor, 0, sizeof(uint32_t), g.stream));
            if (tal)
                k_fused<kCountMode, false, true><<<uint32_t(g_fused_blocks[kCountMode]), kZW * 32, 0, g.stream>>>(
                    view, dp, p, pa, pb, 2, split, g.d_u32 + kSlotCursor, hp->fuse_scratch, hp->fuse_stride, fb, acc,
                    acc_c, acc_p, acc_b);
            else
                k_fused<kCountMode, false><<<uint32_t(g_fused_blocks[kCountMode]), kZW * 32, 0, g.stream>>>(
                    view, dp, p, pa, pb, 2, split, g.d_u32 + kSlotCursor, hp->fuse_scratch, hp->fuse_stride, fb, acc,
                    acc_c, acc_p, acc_b);
            CK(cudaGetLastError());
            res.launches += 3;
        }
        if (profile) {
            CK(cudaEventRecord(e1, g.stream));
            marks.push_back({kCountMode, {e0, e1}});
        }
        return CUTS_OK;
    }

    // Sums the profiled launch times per kernel (after a sync).
    void collect_profile() {
        for (auto &m : marks) {
            float t = 0;
            cudaEventElapsedTime(&t, m.second.first, m.second.second);
            if (m.first == kExpand) { res.expand_ms += t; res.expand_launches++; }
            else { res.last_level_ms += t; res.last_level_launches++; }
            cudaEventDestroy(m.second.first);
            cudaEventDestroy(m.second.second);
        }
        marks.clear();
    }

    // Expands parents [pa, pb) of L_{lvl-1}, depth first by chunks.
    int expand(uint32_t lvl, uint32_t pa, uint32_t pb) {
        if (pb <= pa) return CUTS_OK;
        // the last level is counted; with a folded plan, level k-2 counts both;
        // with a fused plan, the counting kernel runs one level earlier
        const uint32_t count_lvl = (k >= 4 && hp->plan.lv[k - 3].fold2) ? k - 3
                                   : (k >= 3 && hp->plan.lv[k - 2].fold) ? k - 2 : k - 1;
        if (!dump && k >= 3 && hp->plan.lv[count_lvl].fuse && lvl == count_lvl - 1)
            return launch_fused(bytes_mode ? kBytesMode : kCountMode, lvl, pa, pb);
        if (lvl == count_lvl && !dump) {
            int rc = launch_level(bytes_mode ? kBytesMode : kCountMode, lvl, pa, pb);
            return rc;
        }
        std::vector<uint32_t> cuts;
        int rc = plan_chunks(lvl, pa, pb, cuts);
        if (rc) return rc;
        for (size_t c = 0; c + 1 < cuts.size(); ++c) {
            const uint32_t a = cuts[c], b = cuts[c + 1];
            if (b <= a) continue;
            if (budget_ms > 0 &&
                std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count() >
                    budget_ms)
                return set_error(CUTS_ERR_BUDGET, "time budget exhausted");
            rc = launch_level(kExpand, lvl, a, b);
            if (rc) return rc;
            res.chunks++;
            CK(cudaMemcpyAsync(g.h_u32 + kSlotOut + lvl, g.d_u32 + kSlotOut + lvl, sizeof(uint32_t),
                               cudaMemcpyDeviceToHost, g.stream));
            CK(cudaMemcpyAsync(g.h_u32 + kSlotErr, g.d_u32 + kSlotErr, 3 * sizeof(uint32_t),
                               cudaMemcpyDeviceToHost, g.stream));
            rc = sync();
            if (rc) return rc;
            if (g.h_u32[kSlotOver]) return set_error(CUTS_ERR_BUDGET, "time budget exhausted");
            const uint32_t nout = g.h_u32[kSlotOut + lvl];
            if (g.h_u32[kSlotErr] || nout > cap)
                return set_error(CUTS_ERR_CAPACITY, "level " + std::to_string(lvl) + " overflowed its capacity");
            res.level_sizes[lvl] += nout;
            rc = (dump && lvl + 1 == k) ? write_rows(nout) : expand(lvl + 1, 0, nout);
            if (rc) return rc;
        }
        return CUTS_OK;
    }

    // Dump: materialise the nout complete matches of L_{k-1} in pieces and
    // write one ans.txt line per match, pairs in matching order
    // (util.cpp:53-74).
    int write_rows(uint32_t nout);
};

}  // namespace

namespace {

// Rows of complete matches: row r = the path of L_{k-1} entry first + r,
// k words in matching order.
__global__ void k_materialize(const RunParams *__restrict__ rp, uint32_t first, uint32_t nrows,
                              uint32_t *__restrict__ rows) {
    const uint32_t k = rp->plan.k;
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < nrows; r += gridDim.x * blockDim.x) {
        uint32_t e = first + r;
        uint32_t *row = rows + size_t(r) * k;
        for (int lv = int(k) - 1; lv >= 0; --lv) {
            row[lv] = rp->vert[lv][e];
            if (lv > 0) e = rp->par[lv][e];
        }
    }
}

constexpr uint32_t kDumpRows = 1u << 22;  // rows materialised per piece

// Carves the arena for `stored` levels and uploads the run parameters.
int prepare(DeviceGraph &g, const Query &q, uint32_t flags, uint32_t stored, RunParams *&hp,
            RunParams *&dp, uint64_t &cap) {
    const uint32_t k = q.k;
    hp = static_cast<RunParams *>(g.h_plan);
    std::memset(hp, 0, sizeof(RunParams));
    int rc = build_plan(q, g.symmetric, flags, hp->plan);
    if (rc) return rc;
    const bool counting = stored == k - 1;
    const char *nf = std::getenv("CUTS_NO_FUSE");  // 1 = fusion off process-wide (A/B comparisons)
    const bool env_nofuse = nf && nf[0] == '1';
    if (k >= 3 && hp->plan.lv[k - 1].ofold) {
        // the orbit fold needs its weight evaluated by the flattened or the
        // fused counting kernel, in 32 bits; otherwise break Q's symmetry
        const bool fused = hp->plan.lv[k - 2].fuse && !env_nofuse;
        const bool flat = g_use_flat && hp->plan.lv[k - 2].nj <= uint32_t(kFJ);
        const bool fits = uint64_t(__builtin_popcount(hp->plan.lv[k - 1].ofold)) *
                              std::max<uint32_t>(g.max_deg, 1) < (1ull << 32);
        if (!counting || !(fused || flat) || !fits) {
            rc = build_plan(q, g.symmetric, flags | CUTS_FLAG_NO_ORBIT_FOLD, hp->plan);
            if (rc) return rc;
        }
    }
    hp->plan.data_loops = g.loops ? 1u : 0u;
    if (k >= 4 && hp->plan.lv[k - 3].fold2) {
        // the pendant pair is counted by the flattened kernel at level k-3;
        // where that kernel does not run, plan without it
        if (!counting || !g_use_flat || hp->plan.lv[k - 3].nj > uint32_t(kFJ)) {
            rc = build_plan(q, g.symmetric, flags | CUTS_FLAG_NO_PAIR_FOLD |
                                                (hp->plan.lv[k - 1].ofold ? 0u : CUTS_FLAG_NO_ORBIT_FOLD),
                            hp->plan);
            if (rc) return rc;
            hp->plan.data_loops = g.loops ? 1u : 0u;
        } else {
            stored = k - 3;  // levels k-3.. are counted, not stored
        }
    }
    if (k >= 3 && hp->plan.lv[k - 2].fold) {
        // the folded count runs in the flattened or the fused kernel only
        const bool fused_here = hp->plan.lv[k - 2].fuse != 0;
        if (!fused_here && (!g_use_flat || hp->plan.lv[k - 2].nj > uint32_t(kFJ))) hp->plan.lv[k - 2].fold = 0;
        else if (counting) stored = k - 2;  // level k-2 is counted, not stored
    }
    // the counted level and, when fused, the one before it are not stored
    const uint32_t cl = (k >= 3 && hp->plan.lv[k - 2].fold) ? k - 2 : k - 1;
    if (k >= 3 && !hp->plan.lv[k - 2].fold) hp->plan.lv[k - 2].fuse = 0;
    if (!counting || env_nofuse)
        for (uint32_t i = 0; i < k; ++i) hp->plan.lv[i].fuse = 0;
    const bool fuse = counting && k >= 3 && hp->plan.lv[cl].fuse;
    if (fuse) stored = cl - 1;
    hp->stored = stored;
    // before a fused count of levels p = cl - 1 and cl, the entries of
    // level p - 1 record where their vertex sits in its list
    hp->pos_lvl = (fuse && cl >= 3) ? cl - 2 : 0xffffffffu;
    if (!g.arena) {
        cudaError_t e = cudaMallocAsync(&g.arena, g.arena_bytes, g.stream);
        if (e != cudaSuccess) {
            g.arena = nullptr;
            return set_error(CUTS_ERR_NOMEM, "arena allocation failed: " + std::string(cudaGetErrorString(e)));
        }
    }
    // L_0: vert + ub (n entries each); L_1..L_{stored-1}: vert + par + ub
    const uint64_t n = g.n;
    const uint64_t l0_bytes = ((8 * n + 255) / 256) * 256 + 256;
    // fused kernel: one scratch row per resident warp, as long as the longest list
    uint64_t fuse_bytes = 0, big_bytes = 0;
    if (fuse) {
        hp->fuse_stride = ((std::max<uint32_t>(g.max_deg, 1) + 31) / 32) * 32;
        fuse_bytes = uint64_t(g_fused_blocks[kCountMode] > g_fused_blocks[kBytesMode] ? g_fused_blocks[kCountMode]
                                                                                      : g_fused_blocks[kBytesMode]) *
                     kZW * hp->fuse_stride * 4;
        // deferred parents: 256 B of counters, four arrays of cap words and a
        // pool of saved candidate sets (1/32 of the arena, 1M..16M words)
        hp->fuse_big_cap = 1u << 17;
        const uint64_t pool = std::min<uint64_t>(16ull << 20, std::max<uint64_t>(1ull << 20, g.arena_bytes / 128));
        hp->fuse_pool_words = uint32_t(std::max<uint64_t>(pool, 2ull * hp->fuse_stride));
        big_bytes = 256 + 16ull * hp->fuse_big_cap + 4ull * hp->fuse_pool_words;
        big_bytes = (big_bytes + 255) / 256 * 256;
        fuse_bytes += big_bytes;
    }
    cap = 0;
    if (g.arena_bytes < l0_bytes + fuse_bytes)
        return set_error(CUTS_ERR_NOMEM, "arena smaller than the root level and scratch");
    if (fuse) {
        hp->fuse_scratch = reinterpret_cast<uint32_t *>(static_cast<char *>(g.arena) + g.arena_bytes - fuse_bytes);
        hp->fuse_big = reinterpret_cast<uint32_t *>(static_cast<char *>(g.arena) + g.arena_bytes - big_bytes);
    }
    if (stored >= 2) {
        cap = (g.arena_bytes - l0_bytes - fuse_bytes) / (12ull * (stored - 1));
        cap = std::min<uint64_t>(cap, (1ull << 31) - 64);
        if (g.level_cap_req) cap = std::min<uint64_t>(cap, g.level_cap_req);
        cap &= ~uint64_t(63);
        if (cap < 2ull * std::max<uint32_t>(g.max_deg, 1))
            return set_error(CUTS_ERR_CAPACITY, "level capacity below twice the maximum degree");
    }
    char *base = static_cast<char *>(g.arena);
    hp->vert[0] = reinterpret_cast<uint32_t *>(base);
    hp->ub[0] = reinterpret_cast<uint32_t *>(base + ((4 * n + 255) / 256) * 256);
    hp->par[0] = nullptr;
    char *cur = base + l0_bytes;
    for (uint32_t i = 1; i < stored; ++i) {
        hp->vert[i] = reinterpret_cast<uint32_t *>(cur); cur += 4 * cap;
        hp->par[i] = reinterpret_cast<uint32_t *>(cur); cur += 4 * cap;
        hp->ub[i] = reinterpret_cast<uint32_t *>(cur); cur += 4 * cap;
    }
    hp->budget_ns = 0;
    hp->stamp = g.d_u64 + kU64Stamp;
    hp->over = g.d_u32 + kSlotOver;
    dp = static_cast<RunParams *>(g.d_plan);
    CK(cudaMemcpyAsync(dp, hp, sizeof(RunParams), cudaMemcpyHostToDevice, g.stream));
    return CUTS_OK;
}

// Level 0 into L_0; returns |L_0|.
int run_roots(DeviceGraph &g, Run &run, uint32_t shard, uint32_t nshards, uint32_t &n0) {
    CK(cudaMemsetAsync(g.d_u32, 0, sizeof(uint32_t) * kSlots, g.stream));
    CK(cudaMemsetAsync(g.d_u64, 0, sizeof(unsigned long long) * kU64Slots, g.stream));
    n0 = 0;
    if (!g.n) return CUTS_OK;
    const uint32_t threads = 256;
    const uint32_t blocks = std::min<uint32_t>((g.n + threads - 1) / threads, uint32_t(g_num_sms) * 8);
    k_roots<<<blocks, threads, 0, g.stream>>>(run.view, run.dp, shard, nshards, g.d_u32 + kSlotN0);
    CK(cudaGetLastError());
    run.res.launches++;
    CK(cudaMemcpyAsync(g.h_u32 + kSlotN0, g.d_u32 + kSlotN0, sizeof(uint32_t), cudaMemcpyDeviceToHost, g.stream));
    int rc = run.sync();
    if (rc) return rc;
    n0 = g.h_u32[kSlotN0];
    return CUTS_OK;
}

// Root slices, as the reference's trunks (host_funcs.cu:66-72).
int run_slices(Run &run, uint32_t n0, uint32_t chunks) {
    const uint32_t slice = uint32_t((uint64_t(n0) - 1) / chunks + 1);
    for (uint32_t s = 0; s < chunks; ++s) {
        const uint64_t a = uint64_t(s) * slice;
        if (a >= n0) break;
        int rc = run.expand(1, uint32_t(a), uint32_t(std::min<uint64_t>(a + slice, n0)));
        if (rc) return rc;
    }
    return CUTS_OK;
}

}  // namespace

int Run::write_rows(uint32_t nout) {
    const uint32_t k = this->k;
    const std::vector<uint32_t> &order = query->order;
    uint32_t *d_rows = nullptr, *h_rows = nullptr;
    const uint32_t piece = std::min<uint32_t>(nout, kDumpRows);
    CK(cudaMalloc(&d_rows, sizeof(uint32_t) * size_t(piece) * k));
    cudaError_t e = cudaMallocHost(&h_rows, sizeof(uint32_t) * size_t(piece) * k);
    if (e != cudaSuccess) {
        cudaFree(d_rows);
        return set_error(CUTS_ERR_NOMEM, "pinned dump buffer");
    }
    std::vector<char> text;
    int rc = CUTS_OK;
    for (uint32_t first = 0; first < nout && rc == CUTS_OK; first += piece) {
        const uint32_t nr = std::min(piece, nout - first);
        k_materialize<<<std::max<uint32_t>(1, std::min<uint32_t>((nr + 255) / 256, 4096)), 256, 0, g.stream>>>(
            dp, first, nr, d_rows);
        res.launches++;
        if ((e = cudaMemcpyAsync(h_rows, d_rows, sizeof(uint32_t) * size_t(nr) * k, cudaMemcpyDeviceToHost,
                                 g.stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(g.stream)) != cudaSuccess) {
            rc = set_error(CUTS_ERR_CUDA, std::string("dump copy: ") + cudaGetErrorString(e));
            break;
        }
        // text, formatted in parallel: each thread a contiguous block of
        // rows into its own part of the buffer, written in row order
        const size_t per_row = size_t(k) * 24 + 1;
        text.resize(size_t(nr) * per_row + 16);
        const int nth = std::max(1, std::min(omp_get_max_threads(), int((nr + 4095) / 4096)));
        std::vector<size_t> used(size_t(nth), 0);
        #pragma omp parallel for schedule(static, 1) num_threads(nth)
        for (int t = 0; t < nth; ++t) {
            const uint32_t r0 = uint32_t(uint64_t(nr) * t / nth), r1 = uint32_t(uint64_t(nr) * (t + 1) / nth);
            char *const b0 = text.data() + size_t(r0) * per_row;
            char *w = b0, *const end = text.data() + size_t(r1) * per_row;
            for (uint32_t r = r0; r < r1; ++r) {
                const uint32_t *row = h_rows + size_t(r) * k;
                for (uint32_t j = 0; j < k; ++j) {
                    *w++ = '(';
                    w = std::to_chars(w, end, order[j]).ptr;
                    *w++ = ',';
                    w = std::to_chars(w, end, g.orig.empty() ? row[j] : g.orig[row[j]]).ptr;
                    *w++ = ')';
                }
                *w++ = '\n';
            }
            used[size_t(t)] = size_t(w - b0);
        }
        for (int t = 0; t < nth && rc == CUTS_OK; ++t) {
            const char *b0 = text.data() + size_t(uint64_t(nr) * t / nth) * per_row;
            if (std::fwrite(b0, 1, used[size_t(t)], dump_file) != used[size_t(t)])
                rc = set_error(CUTS_ERR_IO, std::string("short write to the dump file: ") + std::strerror(errno));
        }
        dumped += nr;
    }
    cudaFree(d_rows);
    cudaFreeHost(h_rows);
    return rc;
}

int device_count(DeviceGraph &g, const Query &q, const CountOptions &opt, CountResult &res) {
    res = CountResult();
    if (opt.chunks == 0) return set_error(CUTS_ERR_ARG, "chunks must be >= 1");
    if (opt.nshards == 0 || opt.shard >= opt.nshards) return set_error(CUTS_ERR_ARG, "bad shard");
    CK(cudaSetDevice(g.device));
    int rc = launch_geometry();
    if (rc) return rc;
    const uint32_t k = q.k;
    RunParams *hp = nullptr, *dp = nullptr;
    uint64_t cap = 0;
    rc = prepare(g, q, opt.flags, k - 1, hp, dp, cap);
    if (rc) return rc;
    Run run{g, graph_view(g), hp, dp, k, cap, 4, false, res};
    run.profile = opt.profile;
    run.budget_ms = opt.budget_ms;
    if (opt.budget_ms > 0) {  // the kernels' own deadline (device time from k_roots)
        hp->budget_ns = (unsigned long long)(opt.budget_ms * 1e6);
        CK(cudaMemcpyAsync(dp, hp, sizeof(RunParams), cudaMemcpyHostToDevice, g.stream));
    }
    CK(cudaEventRecord(g.ev0, g.stream));
    uint32_t n0 = 0;
    rc = run_roots(g, run, opt.shard, opt.nshards, n0);
    if (rc) return rc;
    res.level_sizes[0] = n0;
    if (k >= 2 && n0 > 0) {
        rc = run_slices(run, n0, opt.chunks);
        if (rc) return rc;
    }
    CK(cudaEventRecord(g.ev1, g.stream));
    CK(cudaMemcpyAsync(g.h_u64, g.d_u64, sizeof(unsigned long long), cudaMemcpyDeviceToHost, g.stream));
    CK(cudaMemcpyAsync(g.h_u32 + kSlotOver, g.d_u32 + kSlotOver, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                       g.stream));
    rc = run.sync();
    if (rc) return rc;
    run.collect_profile();
    CK(cudaEventElapsedTime(&res.ms, g.ev0, g.ev1));
    if (g.h_u32[kSlotOver]) return set_error(CUTS_ERR_BUDGET, "time budget exhausted");
    const uint64_t raw = k >= 2 ? uint64_t(g.h_u64[0]) : 0;
    res.level_sizes[k - 1] = k >= 2 ? raw : n0;
    if (k >= 4 && hp->plan.lv[k - 3].fold2) {  // level k-3 counted both pendant levels
        CK(cudaMemcpy(g.h_u64 + 3, g.d_u64 + 3, sizeof(unsigned long long) * 4, cudaMemcpyDeviceToHost));
        res.level_sizes[k - 3] = g.h_u64[3];
        res.level_sizes[k - 2] = g.h_u64[kU64Pair];
    }
    if (k >= 3 && hp->plan.lv[k - 2].fold) {
        CK(cudaMemcpy(g.h_u64 + 3, g.d_u64 + 3, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        res.level_sizes[k - 2] = g.h_u64[3];
    }
    if (k >= 3) {
        const uint32_t cl = hp->plan.lv[k - 2].fold ? k - 2 : k - 1;
        if (hp->plan.lv[cl].fuse) {  // the fused level before the counted one
            CK(cudaMemcpy(g.h_u64 + 4, g.d_u64 + 4, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
            res.level_sizes[cl - 1] = g.h_u64[4];
        }
    }
    res.count = raw * hp->plan.aut;
    if (opt.want_bytes && k >= 2 && n0 > 0) {
        // untimed second pass: algorithmic bytes of the last-level kernel
        CountResult tmp;
        if (hp->budget_ns) {  // the bytes pass runs to the end
            hp->budget_ns = 0;
            CK(cudaMemcpyAsync(dp, hp, sizeof(RunParams), cudaMemcpyHostToDevice, g.stream));
        }
        Run r2{g, run.view, hp, dp, k, cap, 4, true, tmp};
        CK(cudaMemsetAsync(g.d_u64 + 2, 0, sizeof(unsigned long long), g.stream));
        rc = run_slices(r2, n0, opt.chunks);
        if (rc) return rc;
        CK(cudaMemcpyAsync(g.h_u64 + 2, g.d_u64 + 2, sizeof(unsigned long long), cudaMemcpyDeviceToHost, g.stream));
        rc = r2.sync();
        if (rc) return rc;
        res.last_level_bytes = g.h_u64[2];
    }
    return CUTS_OK;
}

int device_dump(DeviceGraph &g, const Query &q, const char *path, uint64_t *lines, uint32_t shard,
                uint32_t nshards) {
    if (nshards == 0 || shard >= nshards) return set_error(CUTS_ERR_ARG, "bad shard");
    CK(cudaSetDevice(g.device));
    int rc = launch_geometry();
    if (rc) return rc;
    const uint32_t k = q.k;
    FILE *f = std::fopen(path, "wb");
    if (!f) return set_error(CUTS_ERR_IO, std::string("cannot write ") + path);
    std::unique_ptr<FILE, int (*)(FILE *)> hold(f, std::fclose);
    if (lines) *lines = 0;
    if (k < 2) return CUTS_OK;  // the reference dumps nothing for a 1-vertex query
    RunParams *hp = nullptr, *dp = nullptr;
    uint64_t cap = 0;
    rc = prepare(g, q, CUTS_FLAG_NO_CLOSED_FORM, k, hp, dp, cap);
    if (rc) return rc;
    CountResult res;
    Run run{g, graph_view(g), hp, dp, k, cap, 4, false, res};
    run.dump = true;
    run.dump_file = f;
    run.query = &q;
    uint32_t n0 = 0;
    rc = run_roots(g, run, shard, nshards, n0);
    if (rc) return rc;
    if (n0 > 0) {
        rc = run_slices(run, n0, 1);
        if (rc) return rc;
    }
    if (lines) *lines = run.dumped;
    return CUTS_OK;
}

}  // namespace cuts
