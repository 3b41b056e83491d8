// gen.cpp -- seeded synthetic inputs: Erdos-Renyi and Chung-Lu data graphs,
// random connected queries.  Every draw comes from a counter-based
// splitmix64 stream, so a graph depends only on its parameters and seed, not
// on the thread count.
#include <algorithm>
#include <cmath>
#include <parallel/algorithm>

#include "host.hpp"

namespace cuts {

void gen_erdos_renyi(uint32_t n, double p, uint64_t seed, HostGraph &g) {
    std::vector<uint32_t> src, dst;
    const uint64_t base = splitmix64(seed ^ 0x45524552ull);
    uint64_t ctr = 0;
    if (p > 0 && n > 1) {
        const double lq = std::log1p(-std::min(p, 1.0 - 1e-16));
        // Batagelj & Brandes (2005), algorithm G(n,p) with geometric skips
        int64_t v = 1, w = -1;
        while (v < int64_t(n)) {
            double r = u01(splitmix64(base + ctr++));
            w += 1 + int64_t(std::floor(std::log1p(-r) / lq));
            while (w >= v && v < int64_t(n)) { w -= v; ++v; }
            if (v < int64_t(n)) {
                src.push_back(uint32_t(v)); dst.push_back(uint32_t(w));
                src.push_back(uint32_t(w)); dst.push_back(uint32_t(v));
            }
        }
    }
    graph_from_arcs(n, src, dst, g);
}

namespace {
struct Alias {
    std::vector<float> prob;
    std::vector<uint32_t> alias;
    uint32_t n = 0;
    // Vose's alias method
    void build(const std::vector<double> &w) {
        n = uint32_t(w.size());
        prob.assign(n, 0.f);
        alias.assign(n, 0);
        double sum = 0;
        for (double x : w) sum += x;
        std::vector<double> sc(n);
        std::vector<uint32_t> small, large;
        for (uint32_t i = 0; i < n; ++i) {
            sc[i] = w[i] * n / sum;
            (sc[i] < 1.0 ? small : large).push_back(i);
        }
        while (!small.empty() && !large.empty()) {
            uint32_t s = small.back(), l = large.back();
            small.pop_back();
            prob[s] = float(sc[s]);
            alias[s] = l;
            sc[l] = (sc[l] + sc[s]) - 1.0;
            if (sc[l] < 1.0) { large.pop_back(); small.push_back(l); }
        }
        for (uint32_t i : large) { prob[i] = 1.f; alias[i] = i; }
        for (uint32_t i : small) { prob[i] = 1.f; alias[i] = i; }
    }
    uint32_t draw(uint64_t h) const {
        uint32_t col = uint32_t(((h >> 32) * uint64_t(n)) >> 32);
        float coin = float(uint32_t(h)) * (1.0f / 4294967296.0f);
        return coin < prob[col] ? col : alias[col];
    }
};
struct KeyT {
    uint64_t key;
    uint64_t t;
    bool operator<(const KeyT &o) const { return key < o.key || (key == o.key && t < o.t); }
};
}  // namespace

int gen_chung_lu(uint32_t n, uint64_t m, double gamma, double wmin, double cap, uint64_t seed,
                 HostGraph &g) {
    if (n < 2 || gamma <= 1.0 || wmin <= 0)
        return set_error(CUTS_ERR_ARG, "chung-lu: need n >= 2, gamma > 1, wmin > 0");
    if (m > uint64_t(n) * (n - 1) / 2) return set_error(CUTS_ERR_ARG, "chung-lu: m too large");
    const uint64_t ws = splitmix64(seed ^ 0x574549474854ull), es = splitmix64(seed ^ 0x45444745ull);
    std::vector<double> w(n);
    const double ex = -1.0 / (gamma - 1.0);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(n); ++i)
        w[i] = std::min(cap, wmin * std::pow(u01(splitmix64(ws + uint64_t(i))), ex));
    Alias al;
    al.build(w);
    // The edge set is the first m distinct non-loop pairs of the draw stream
    // t = 0, 1, 2, ...  Draw T pairs in parallel, keep each pair's first
    // draw index, and cut the stream where the m-th distinct pair appears;
    // grow T when it holds fewer than m distinct pairs.
    uint64_t T = m + m / 8 + 1024;
    std::vector<KeyT> keys;
    while (true) {
        keys.resize(T);
        #pragma omp parallel for schedule(static)
        for (int64_t t = 0; t < int64_t(T); ++t) {
            uint32_t a = al.draw(splitmix64(es + 2 * uint64_t(t)));
            uint32_t b = al.draw(splitmix64(es + 2 * uint64_t(t) + 1));
            if (a > b) std::swap(a, b);
            keys[t].key = a == b ? ~0ull : (uint64_t(a) << 32) | b;
            keys[t].t = uint64_t(t);
        }
        __gnu_parallel::sort(keys.begin(), keys.end());
        uint64_t u = 0;
        for (uint64_t i = 0; i < T; ++i) {
            if (keys[i].key == ~0ull) break;
            if (i == 0 || keys[i].key != keys[i - 1].key) keys[u++] = keys[i];
        }
        if (u >= m) {
            keys.resize(u);
            // keep the m pairs with the smallest first-draw index
            std::nth_element(keys.begin(), keys.begin() + (m - 1), keys.end(),
                             [](const KeyT &x, const KeyT &y) { return x.t < y.t; });
            keys.resize(m);
            break;
        }
        T = T + T / 4 + (m - u) * 2;
    }
    std::vector<uint32_t> src(2 * m), dst(2 * m);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(m); ++i) {
        uint32_t a = uint32_t(keys[i].key >> 32), b = uint32_t(keys[i].key);
        src[2 * i] = a; dst[2 * i] = b;
        src[2 * i + 1] = b; dst[2 * i + 1] = a;
    }
    std::vector<KeyT>().swap(keys);
    return graph_from_arcs(n, src, dst, g);
}

void gen_random_query(uint32_t k, double p, uint64_t seed, std::vector<uint32_t> &src,
                      std::vector<uint32_t> &dst) {
    src.clear();
    dst.clear();
    const uint64_t base = splitmix64(seed ^ 0x5155455259ull);
    uint64_t ctr = 0;
    std::vector<std::vector<char>> adj(k, std::vector<char>(k, 0));
    for (uint32_t i = 1; i < k; ++i) {  // random attachment spanning tree
        uint32_t j = uint32_t(splitmix64(base + ctr++) % i);
        adj[i][j] = adj[j][i] = 1;
    }
    for (uint32_t a = 0; a < k; ++a)
        for (uint32_t b = a + 1; b < k; ++b) {
            double r = u01(splitmix64(base + ctr++));
            if (!adj[a][b] && r < p) adj[a][b] = adj[b][a] = 1;
        }
    for (uint32_t a = 0; a < k; ++a)
        for (uint32_t b = 0; b < k; ++b)
            if (adj[a][b]) { src.push_back(a); dst.push_back(b); }
}

}  // namespace cuts
