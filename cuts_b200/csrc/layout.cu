// layout.cu -- the data graph's device layout, built on the device.
//
// The caller's CSR (host memory, the reference's format after parsing:
// graph.cpp:29-57 builds the same out/in lists) is copied to the device as
// is; validation, the symmetry check, the degree ranking of vertex ids, the
// padded layout and the per-list sort all run there, so a resident graph
// costs one host-to-device copy plus a few milliseconds of kernels instead
// of host passes over every arc.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include "device_util.cuh"
#include "engine.hpp"

namespace cuts {
namespace {

constexpr uint32_t kPad = 0xffffffffu;

__device__ __forceinline__ uint32_t padded(uint32_t len) { return (len + 3u) & ~3u; }

// Offsets monotone and within the arc count; every list strictly increasing
// with ids below n.  flag |= 1 (offsets) or 2 (lists).  One warp per vertex,
// its lanes across the list (coalesced; a hub's list no longer serialises
// one thread).
__global__ void k_validate(uint32_t n, uint64_t m, const uint64_t *__restrict__ off,
                           const uint32_t *__restrict__ adj, uint32_t *__restrict__ flag) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t v = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; v < n; v += warps) {
        const uint64_t a = off[v], b = off[v + 1];
        if (b < a || b > m) {
            if (lane == 0) atomicOr(flag, 1u);
            continue;
        }
        bool bad = false;
        for (uint64_t x = a + lane; x < b; x += 32) {
            const uint32_t id = adj[x];
            if (id >= n || (x > a && id <= adj[x - 1])) bad = true;
        }
        if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(flag, 2u);
    }
}

// flag |= 1 where the two arrays differ.
template <class T>
__global__ void k_differ(uint64_t cnt, const T *__restrict__ a, const T *__restrict__ b,
                         uint32_t *__restrict__ flag) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < cnt; i += uint64_t(gridDim.x) * blockDim.x)
        if (a[i] != b[i]) atomicOr(flag, 1u);
}

// Every arc u -> v has its reverse.  Order the vertices by (degree, id).
// With no repeated arc (the lists were checked strictly increasing),
// reversal maps the arcs that go down in that order one-to-one into the
// arcs that go up, once every down arc's reverse is found; the two sets then
// have equal sizes exactly when every up arc's reverse exists too.  So only
// a down arc u -> v is searched for, as u in v's list -- the shorter of the
// two: a hub's list is never searched -- and the arcs going up and down are
// counted into updown[0] / updown[1] (a self-loop is its own reverse).  One
// warp per vertex u.
__global__ void k_symmetric(uint32_t n, const uint64_t *__restrict__ off, const uint32_t *__restrict__ adj,
                            uint32_t *__restrict__ flag, unsigned long long *__restrict__ updown) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long up = 0, down = 0;
    for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < n; u += warps) {
        const uint64_t a = off[u], b = off[u + 1];
        const uint64_t du = b - a;
        for (uint64_t x = a + lane; x < b; x += 32) {
            const uint32_t v = adj[x];
            if (v == u) continue;
            const uint64_t lo0 = off[v], hi0 = off[v + 1], dv = hi0 - lo0;
            if (!(dv < du || (dv == du && v < u))) {
                ++up;
                continue;
            }
            ++down;
            uint64_t lo = lo0, hi = hi0;
            while (lo < hi) {
                const uint64_t mid = (lo + hi) >> 1;
                if (adj[mid] < u) lo = mid + 1; else hi = mid;
            }
            if (lo == hi0 || adj[lo] != u) atomicOr(flag, 1u);
        }
    }
    for (int sh = 16; sh; sh >>= 1) {
        up += __shfl_xor_sync(0xffffffffu, up, sh);
        down += __shfl_xor_sync(0xffffffffu, down, sh);
    }
    if (lane == 0 && (up | down)) {
        atomicAdd(updown, up);
        atomicAdd(updown + 1, down);
    }
}

// Sort keys (degree << 32 | vertex): ascending degree, then id.
__global__ void k_keys(uint32_t n, const uint64_t *__restrict__ ooff, const uint64_t *__restrict__ ioff,
                       unsigned long long *__restrict__ keys) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        uint64_t d = ooff[v + 1] - ooff[v];
        if (ioff) d += ioff[v + 1] - ioff[v];
        keys[v] = (d << 32) | v;
    }
}

// orig[d] = the vertex of rank d; rank[v] = its rank.
__global__ void k_ranks(uint32_t n, const unsigned long long *__restrict__ sorted, uint32_t *__restrict__ orig,
                        uint32_t *__restrict__ rank) {
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) {
        const uint32_t v = uint32_t(sorted[d] & 0xffffffffull);
        orig[d] = v;
        rank[v] = d;
    }
}

// Padded length of device vertex d's list (entry n = 0, for the scan's total).
__global__ void k_plen(uint32_t n, const uint32_t *__restrict__ orig, const uint64_t *__restrict__ off,
                       unsigned long long *__restrict__ plen) {
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d <= n; d += gridDim.x * blockDim.x) {
        if (d == n) { plen[d] = 0; continue; }
        const uint32_t v = orig ? orig[d] : d;
        plen[d] = padded(uint32_t(off[v + 1] - off[v]));
    }
}

// info[d] = {base + start, length}; segment bounds for the sort.
__global__ void k_info(uint32_t n, const uint32_t *__restrict__ orig, const uint64_t *__restrict__ off,
                       const unsigned long long *__restrict__ start, uint32_t base, uint2 *__restrict__ info,
                       uint32_t *__restrict__ seg_b, uint32_t *__restrict__ seg_e) {
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) {
        const uint32_t v = orig ? orig[d] : d;
        const uint32_t len = uint32_t(off[v + 1] - off[v]);
        const uint32_t s = base + uint32_t(start[d]);
        info[d] = make_uint2(s, len);
        if (seg_b) {
            seg_b[d] = s;
            seg_e[d] = s + len;
        }
    }
}

// One warp per device vertex: its list, ids mapped through rank (when
// given), and the padding.
__global__ void k_fill(uint32_t n, const uint32_t *__restrict__ orig, const uint32_t *__restrict__ rank,
                       const uint64_t *__restrict__ off, const uint32_t *__restrict__ src,
                       const uint2 *__restrict__ info, uint32_t *__restrict__ dst) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t d = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; d < n; d += warps) {
        const uint32_t v = orig ? orig[d] : d;
        const uint64_t a = off[v];
        const uint2 inf = info[d];
        for (uint32_t j = lane; j < padded(inf.y); j += 32) {
            uint32_t x = kPad;
            if (j < inf.y) {
                x = src[a + j];
                if (rank) x = rank[x];
            }
            dst[inf.x + j] = x;
        }
    }
}

// The padding after each sorted list.
__global__ void k_pad(uint32_t n, const uint2 *__restrict__ info, uint32_t *__restrict__ adj) {
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) {
        const uint2 inf = info[d];
        for (uint32_t j = inf.y; j < padded(inf.y); ++j) adj[inf.x + j] = kPad;
    }
}

// flag |= 1 when some vertex lists itself.
__global__ void k_loops(uint32_t n, const uint2 *__restrict__ info, const uint32_t *__restrict__ adj,
                        uint32_t *__restrict__ flag) {
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) {
        const uint2 inf = info[d];
        if (contains(adj + inf.x, inf.y, d)) atomicOr(flag, 1u);
    }
}

// bwd[d] = entries of d's list below d (a lower-bound search per vertex).
__global__ void k_bwd(uint32_t n, const uint2 *__restrict__ info, const uint32_t *__restrict__ adj,
                      uint32_t *__restrict__ bwd) {
    for (uint32_t d = blockIdx.x * blockDim.x + threadIdx.x; d < n; d += gridDim.x * blockDim.x) {
        const uint2 inf = info[d];
        bwd[d] = lbound(adj + inf.x, inf.y, d);
    }
}

// Dense core rows: one warp per core vertex d, its list entries u >= core0
// set bit u - core0 of row d - core0 (rows are zeroed before).
__global__ void k_core_bits(uint32_t n, uint32_t core0, const uint2 *__restrict__ info,
                            const uint32_t *__restrict__ adj, uint32_t *__restrict__ bits) {
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t words = kCore / 32;
    for (uint32_t d = core0 + (blockIdx.x * blockDim.x + threadIdx.x) / 32; d < n;
         d += (gridDim.x * blockDim.x) / 32) {
        const uint2 inf = info[d];
        const uint32_t *l = adj + inf.x;
        for (uint32_t i = lbound(l, inf.y, core0) + lane; i < inf.y; i += 32) {
            const uint32_t u = l[i] - core0;
            atomicOr(bits + size_t(d - core0) * words + (u >> 5), 1u << (u & 31));
        }
    }
}

// Device buffers of one build, stream-ordered from the device's memory pool
// (reused across builds instead of mapped and unmapped each time), released
// on every exit.
struct Scratch {
    cudaStream_t s;
    std::vector<void *> p;
    explicit Scratch(cudaStream_t st) : s(st) {}
    ~Scratch() {
        for (void *x : p) cudaFreeAsync(x, s);
        cudaStreamSynchronize(s);
    }
    template <class T>
    cudaError_t get(T **out, size_t count) {
        *out = nullptr;
        if (!count) count = 1;
        cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(out), sizeof(T) * count, s);
        if (e == cudaSuccess) p.push_back(*out);
        return e;
    }
};

}  // namespace

#define LCK(x)                                                                                   \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess)                                                                   \
            return set_error(CUTS_ERR_CUDA, std::string("graph layout: ") + cudaGetErrorString(e_)); \
    } while (0)

int device_layout(uint32_t n, const uint64_t *out_off, const uint32_t *out_adj, const uint64_t *in_off,
                  const uint32_t *in_adj, int sym_hint, bool validate, DeviceGraph &g) {
    if (!out_off || (n > 0 && !out_adj && out_off[n] > 0)) return set_error(CUTS_ERR_ARG, "null CSR array");
    if (in_adj && !in_off) return set_error(CUTS_ERR_ARG, "in_adj without in_off");
    if (in_off && !in_adj && n > 0 && in_off[n] > 0) return set_error(CUTS_ERR_ARG, "in_off without in_adj");
    if (out_off[0] != 0 || (in_off && in_off[0] != 0)) return set_error(CUTS_ERR_ARG, "CSR offsets must start at 0");
    const uint64_t m = out_off[n];
    if (in_off && in_off[n] != m) return set_error(CUTS_ERR_ARG, "in/out arc counts differ");
    cudaStream_t s = g.stream;
    const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>((n + 255) / 256, 148u * 16));
    Scratch sc(s);
    uint64_t *d_ooff = nullptr, *d_ioff = nullptr;
    uint32_t *d_oadj = nullptr, *d_iadj = nullptr, *d_flag = nullptr;
    LCK(sc.get(&d_ooff, size_t(n) + 1));
    LCK(sc.get(&d_oadj, m));
    LCK(sc.get(&d_flag, 1));
    LCK(cudaMemcpyAsync(d_ooff, out_off, sizeof(uint64_t) * (size_t(n) + 1), cudaMemcpyHostToDevice, s));
    if (m) LCK(cudaMemcpyAsync(d_oadj, out_adj, sizeof(uint32_t) * m, cudaMemcpyHostToDevice, s));
    if (in_off) {
        LCK(sc.get(&d_ioff, size_t(n) + 1));
        LCK(sc.get(&d_iadj, m));
        LCK(cudaMemcpyAsync(d_ioff, in_off, sizeof(uint64_t) * (size_t(n) + 1), cudaMemcpyHostToDevice, s));
        if (m) LCK(cudaMemcpyAsync(d_iadj, in_adj, sizeof(uint32_t) * m, cudaMemcpyHostToDevice, s));
    }
    uint32_t h_flag = 0;
    auto read_flag = [&]() -> int {
        LCK(cudaMemcpyAsync(&h_flag, d_flag, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        LCK(cudaStreamSynchronize(s));
        return CUTS_OK;
    };
    int rc = CUTS_OK;
    if (validate && n) {
        LCK(cudaMemsetAsync(d_flag, 0, sizeof(uint32_t), s));
        const uint32_t vgrid = std::max<uint32_t>(1, std::min<uint32_t>((n + 7) / 8, 148u * 16));
        k_validate<<<vgrid, 256, 0, s>>>(n, m, d_ooff, d_oadj, d_flag);
        if (in_off) k_validate<<<vgrid, 256, 0, s>>>(n, m, d_ioff, d_iadj, d_flag);
        LCK(cudaGetLastError());
        if ((rc = read_flag())) return rc;
        if (h_flag & 1) return set_error(CUTS_ERR_ARG, "CSR offsets not monotone");
        if (h_flag & 2) return set_error(CUTS_ERR_ARG, "CSR list not strictly sorted or out of range");
    }
    // symmetry: given, compared with the in-lists, or checked arc by arc
    bool symmetric = sym_hint == 1;
    unsigned long long *d_updown = nullptr, h_updown[2] = {0, 0};
    if (sym_hint < 0) {
        LCK(cudaMemsetAsync(d_flag, 0, sizeof(uint32_t), s));
        if (in_off) {
            k_differ<uint64_t><<<grid, 256, 0, s>>>(uint64_t(n) + 1, d_ooff, d_ioff, d_flag);
            const uint32_t g2 = uint32_t(std::max<uint64_t>(1, std::min<uint64_t>((m + 255) / 256, 148u * 16)));
            if (m) k_differ<uint32_t><<<g2, 256, 0, s>>>(m, d_oadj, d_iadj, d_flag);
        } else if (n) {
            LCK(sc.get(&d_updown, 2));
            LCK(cudaMemsetAsync(d_updown, 0, 2 * sizeof(unsigned long long), s));
            k_symmetric<<<std::max<uint32_t>(1, std::min<uint32_t>((n + 7) / 8, 148u * 16)), 256, 0, s>>>(
                n, d_ooff, d_oadj, d_flag, d_updown);
            LCK(cudaMemcpyAsync(h_updown, d_updown, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        }
        LCK(cudaGetLastError());
        if ((rc = read_flag())) return rc;
        symmetric = h_flag == 0 && h_updown[0] == h_updown[1];
        if (!in_off && !symmetric)
            return set_error(CUTS_ERR_ARG, "in-lists omitted but the graph is not symmetric");
    }
    if (!symmetric && !in_off) return set_error(CUTS_ERR_ARG, "directed graph without in-lists");
    const uint64_t *ioff_used = symmetric ? nullptr : d_ioff;

    // degree ranks (CUTS_NO_RELABEL=1 keeps host ids); the per-list sort
    // indexes words with int, so a layout of 2^31 words or more keeps them too
    uint64_t pre_words = 0;
    for (int dir = 0; dir < (symmetric ? 1 : 2); ++dir) {
        const uint64_t *off = dir ? in_off : out_off;
        #pragma omp parallel for reduction(+ : pre_words) schedule(static)
        for (int64_t v = 0; v < int64_t(n); ++v) pre_words += (off[v + 1] - off[v] + 3) & ~uint64_t(3);
    }
    const char *nr = std::getenv("CUTS_NO_RELABEL");
    const bool relabel = !(nr && nr[0] == '1') && n > 1 && pre_words < (uint64_t(1) << 31);
    uint32_t *d_orig = nullptr, *d_rank = nullptr;
    if (relabel) {
        unsigned long long *k0 = nullptr, *k1 = nullptr;
        LCK(sc.get(&k0, n));
        LCK(sc.get(&k1, n));
        LCK(sc.get(&d_orig, n));
        LCK(sc.get(&d_rank, n));
        k_keys<<<grid, 256, 0, s>>>(n, d_ooff, ioff_used, k0);
        LCK(cudaGetLastError());
        size_t tb = 0;
        LCK(cub::DeviceRadixSort::SortKeys(nullptr, tb, k0, k1, int(n), 0, 64, s));
        void *tmp = nullptr;
        LCK(sc.get(reinterpret_cast<char **>(&tmp), tb));
        LCK(cub::DeviceRadixSort::SortKeys(tmp, tb, k0, k1, int(n), 0, 64, s));
        k_ranks<<<grid, 256, 0, s>>>(n, k1, d_orig, d_rank);
        LCK(cudaGetLastError());
    }
    // padded offsets: out-lists, then in-lists of a directed graph
    unsigned long long *plen = nullptr, *pstart = nullptr;
    LCK(sc.get(&plen, size_t(n) + 1));
    LCK(sc.get(&pstart, size_t(n) + 1));
    size_t sb = 0;
    LCK(cub::DeviceScan::ExclusiveSum(nullptr, sb, plen, pstart, int(n) + 1, s));
    void *scan_tmp = nullptr;
    LCK(sc.get(reinterpret_cast<char **>(&scan_tmp), sb));
    uint64_t words[2] = {0, 0};
    const int dirs = symmetric ? 1 : 2;
    std::vector<unsigned long long *> starts(dirs);
    for (int dir = 0; dir < dirs; ++dir) {
        const uint64_t *off = dir ? d_ioff : d_ooff;
        k_plen<<<grid, 256, 0, s>>>(n, d_orig, off, plen);
        LCK(cudaGetLastError());
        unsigned long long *st = nullptr;
        LCK(sc.get(&st, size_t(n) + 1));
        LCK(cub::DeviceScan::ExclusiveSum(scan_tmp, sb, plen, st, int(n) + 1, s));
        unsigned long long tot = 0;
        LCK(cudaMemcpyAsync(&tot, st + n, sizeof(tot), cudaMemcpyDeviceToHost, s));
        LCK(cudaStreamSynchronize(s));
        words[dir] = tot;
        starts[dir] = st;
    }
    const uint64_t total = std::max<uint64_t>(words[0] + words[1], 4);
    if (total >= (uint64_t(1) << 32)) return set_error(CUTS_ERR_LIMIT, "padded adjacency exceeds 2^32 words");

    // device-resident arrays of the graph (owned by g from here on)
    // the graph's own arrays come from the device's default pool too (freed
    // with cudaFreeAsync by device_graph_free), so a rebuilt graph reuses them
    LCK(cudaMallocAsync(reinterpret_cast<void **>(&g.out_info), sizeof(uint2) * std::max<uint32_t>(n, 1), s));
    if (symmetric) g.in_info = g.out_info;
    else LCK(cudaMallocAsync(reinterpret_cast<void **>(&g.in_info), sizeof(uint2) * std::max<uint32_t>(n, 1), s));
    LCK(cudaMallocAsync(reinterpret_cast<void **>(&g.adj), sizeof(uint32_t) * total, s));
    LCK(cudaMemsetAsync(g.adj, 0xff, sizeof(uint32_t) * total, s));
    uint32_t *seg_b = nullptr, *seg_e = nullptr, *fill = g.adj;
    if (relabel) {
        LCK(sc.get(&seg_b, size_t(n) * dirs));
        LCK(sc.get(&seg_e, size_t(n) * dirs));
        LCK(sc.get(&fill, total));
    }
    const uint32_t wgrid = std::max<uint32_t>(1, std::min<uint32_t>((n + 7) / 8, 148u * 16));
    for (int dir = 0; dir < dirs; ++dir) {
        const uint64_t *off = dir ? d_ioff : d_ooff;
        const uint32_t *src = dir ? d_iadj : d_oadj;
        uint2 *info = dir ? g.in_info : g.out_info;
        const uint32_t base = dir ? uint32_t(words[0]) : 0u;
        k_info<<<grid, 256, 0, s>>>(n, d_orig, off, starts[dir], base, info,
                                    seg_b ? seg_b + size_t(dir) * n : nullptr,
                                    seg_e ? seg_e + size_t(dir) * n : nullptr);
        if (n) k_fill<<<wgrid, 256, 0, s>>>(n, d_orig, d_rank, off, src, info, fill);
        LCK(cudaGetLastError());
    }
    if (relabel && m) {
        // each list, now in device ids, sorted into the final array
        size_t tb = 0;
        const int segs = int(n) * dirs;
        LCK(cub::DeviceSegmentedSort::SortKeys(nullptr, tb, fill, g.adj, int(total), segs, seg_b, seg_e, s));
        void *tmp = nullptr;
        LCK(sc.get(reinterpret_cast<char **>(&tmp), tb));
        LCK(cub::DeviceSegmentedSort::SortKeys(tmp, tb, fill, g.adj, int(total), segs, seg_b, seg_e, s));
        for (int dir = 0; dir < dirs; ++dir)
            k_pad<<<grid, 256, 0, s>>>(n, dir ? g.in_info : g.out_info, g.adj);
        LCK(cudaGetLastError());
    }
    LCK(cudaMemsetAsync(d_flag, 0, sizeof(uint32_t), s));
    if (n) k_loops<<<grid, 256, 0, s>>>(n, g.out_info, g.adj, d_flag);
    LCK(cudaGetLastError());
    if ((rc = read_flag())) return rc;
    g.loops = h_flag != 0;
    // per-vertex counts of list entries below the vertex (windows that start
    // or end at a list's own vertex need no search)
    LCK(cudaMallocAsync(reinterpret_cast<void **>(&g.bwd_out), sizeof(uint32_t) * std::max<uint32_t>(n, 1) * (symmetric ? 1 : 2), s));
    g.bwd_in = symmetric ? g.bwd_out : g.bwd_out + n;
    if (n) {
        k_bwd<<<grid, 256, 0, s>>>(n, g.out_info, g.adj, g.bwd_out);
        if (!symmetric) k_bwd<<<grid, 256, 0, s>>>(n, g.in_info, g.adj, g.bwd_in);
    }
    LCK(cudaGetLastError());
    if (symmetric && n) {
        // the dense core: the kCore highest ids (the hubs under the degree
        // ranking), as an adjacency bitmap
        g.core0 = n > kCore ? n - kCore : 0;
        const size_t words = size_t(kCore) * (kCore / 32);
        LCK(cudaMallocAsync(reinterpret_cast<void **>(&g.core_bits), words * sizeof(uint32_t), s));
        LCK(cudaMemsetAsync(g.core_bits, 0, words * sizeof(uint32_t), s));
        k_core_bits<<<(kCore * 32 + 255) / 256, 256, 0, s>>>(n, g.core0, g.out_info, g.adj, g.core_bits);
        LCK(cudaGetLastError());
    }
    g.adj_words = total;
    g.symmetric = symmetric;
    g.n = n;
    g.arcs = m;

    // host-side tables: the id map, degrees by device id, degree tails
    std::vector<uint32_t> orig;
    if (relabel) {
        orig.resize(n);
        LCK(cudaMemcpyAsync(orig.data(), d_orig, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
        LCK(cudaStreamSynchronize(s));
    }
    auto odeg = [&](uint32_t v) { return uint32_t(out_off[v + 1] - out_off[v]); };
    auto ideg = [&](uint32_t v) { return symmetric ? odeg(v) : uint32_t(in_off[v + 1] - in_off[v]); };
    uint32_t maxd = 0;
    #pragma omp parallel for reduction(max : maxd) schedule(static)
    for (int64_t v = 0; v < int64_t(n); ++v) maxd = std::max(maxd, std::max(odeg(uint32_t(v)), ideg(uint32_t(v))));
    g.max_deg = maxd;
    g.h_out_deg.resize(n);
    g.h_in_deg.resize(n);
    #pragma omp parallel for schedule(static)
    for (int64_t d = 0; d < int64_t(n); ++d) {
        const uint32_t v = relabel ? orig[size_t(d)] : uint32_t(d);
        g.h_out_deg[size_t(d)] = odeg(v);
        g.h_in_deg[size_t(d)] = ideg(v);
    }
    DegreeStats st;
    st.n = n;
    st.out_ge.assign(size_t(maxd) + 2, 0);
    st.in_ge.assign(size_t(maxd) + 2, 0);
    // per-thread histograms while they are small (two of 8 B x (maxd + 2)
    // per thread: 1 MB at the bound); one pass otherwise
    #pragma omp parallel if (maxd < (1u << 16))
    {
        std::vector<uint64_t> lo(size_t(maxd) + 2, 0), li(size_t(maxd) + 2, 0);
        #pragma omp for schedule(static) nowait
        for (int64_t v = 0; v < int64_t(n); ++v) {
            lo[odeg(uint32_t(v))]++;
            li[ideg(uint32_t(v))]++;
        }
        #pragma omp critical
        for (size_t d = 0; d < lo.size(); ++d) {
            st.out_ge[d] += lo[d];
            st.in_ge[d] += li[d];
        }
    }
    for (int64_t d = int64_t(maxd); d >= 0; --d) {
        st.out_ge[d] += st.out_ge[d + 1];
        st.in_ge[d] += st.in_ge[d + 1];
    }
    g.stats = std::move(st);
    g.orig.swap(orig);
    return CUTS_OK;
}

}  // namespace cuts
