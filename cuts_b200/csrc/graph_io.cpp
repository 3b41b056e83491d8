// graph_io.cpp -- graph text loader, CSR construction and writer.
//
// The loader keeps the reference's parse semantics (util.cpp:19-52): line 1
// is V (std::stoi: leading whitespace, optional sign, digits, anything after
// ignored), then one arc per line split at the first TAB, lines without a
// TAB skipped, duplicate arcs collapsed, self-loops kept.  Unlike the
// reference (std::set per vertex, one thread) it parses in parallel and
// builds the CSR with a counting sort.  Where the reference has undefined
// behaviour (an endpoint outside [0, V), an unparsable number) it reports
// CUTS_ERR_PARSE instead.
#include <algorithm>
#include <atomic>
#include <charconv>
#include <cctype>
#include <climits>
#include <cstdio>
#include <cstring>
#include <memory>
#include <fcntl.h>
#include <omp.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "host.hpp"

namespace cuts {

static thread_local std::string g_err;

int set_error(int code, const std::string &msg) {
    g_err = msg;
    return code;
}
const char *last_error() { return g_err.c_str(); }

uint32_t HostGraph::max_degree() const {
    uint32_t m = 0;
    for (uint32_t v = 0; v < n; ++v) m = std::max(m, std::max(out_deg(v), in_deg(v)));
    return m;
}

// std::stoi prefix semantics; false when no digits or the value overflows int.
static bool parse_int(const char *s, const char *e, long long &out) {
    while (s < e && std::isspace((unsigned char)*s)) ++s;
    bool neg = false;
    if (s < e && (*s == '+' || *s == '-')) { neg = *s == '-'; ++s; }
    if (s >= e || !std::isdigit((unsigned char)*s)) return false;
    long long v = 0;
    while (s < e && std::isdigit((unsigned char)*s)) {
        v = v * 10 + (*s - '0');
        if (v > (long long)INT_MAX + 1) return false;
        ++s;
    }
    v = neg ? -v : v;
    if (v > INT_MAX || v < INT_MIN) return false;
    out = v;
    return true;
}

static void build_one_csr(uint32_t n, const std::vector<uint32_t> &key,
                          const std::vector<uint32_t> &val, std::vector<uint64_t> &off,
                          std::vector<uint32_t> &adj) {
    const uint64_t m = key.size();
    std::unique_ptr<std::atomic<uint64_t>[]> cnt(new std::atomic<uint64_t>[size_t(n) + 1]);
    #pragma omp parallel for schedule(static)
    for (int64_t v = 0; v <= int64_t(n); ++v) cnt[v].store(0, std::memory_order_relaxed);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(m); ++i) cnt[key[i]].fetch_add(1, std::memory_order_relaxed);
    std::vector<uint64_t> raw(size_t(n) + 1, 0);
    for (uint32_t v = 0; v < n; ++v) raw[v + 1] = raw[v] + cnt[v].load(std::memory_order_relaxed);
    #pragma omp parallel for schedule(static)
    for (int64_t v = 0; v < int64_t(n); ++v) cnt[v].store(raw[v], std::memory_order_relaxed);
    std::vector<uint32_t> tmp(m ? m : 1);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(m); ++i)
        tmp[cnt[key[i]].fetch_add(1, std::memory_order_relaxed)] = val[i];
    // sort + dedup each list; record the deduplicated length
    std::vector<uint64_t> len(size_t(n) + 1, 0);
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < int64_t(n); ++v) {
        uint32_t *b = tmp.data() + raw[v], *e = tmp.data() + raw[v + 1];
        std::sort(b, e);
        len[v + 1] = uint64_t(std::unique(b, e) - b);
    }
    off.assign(size_t(n) + 1, 0);
    for (uint32_t v = 0; v < n; ++v) off[v + 1] = off[v] + len[v + 1];
    adj.resize(off[n]);
    #pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < int64_t(n); ++v)
        std::memcpy(adj.data() + off[v], tmp.data() + raw[v], len[v + 1] * sizeof(uint32_t));
}

// Every arc has its reverse (lists strictly increasing).  Vertices ordered
// by (degree, id): reversal maps the arcs going down one-to-one into the
// arcs going up once each down arc's reverse is found, so only down arcs are
// searched -- in the lower vertex's, shorter, list -- and the two kinds are
// counted: equal counts mean every up arc's reverse exists too.
static bool check_symmetric(const HostGraph &g) {
    std::atomic<bool> ok{true};
    uint64_t up = 0, down = 0;
    #pragma omp parallel for schedule(dynamic, 1024) reduction(+ : up, down)
    for (int64_t u = 0; u < int64_t(g.n); ++u) {
        if (!ok.load(std::memory_order_relaxed)) continue;
        const uint64_t du = g.out_off[u + 1] - g.out_off[u];
        for (uint64_t a = g.out_off[u]; a < g.out_off[u + 1]; ++a) {
            const uint32_t v = g.out_adj[a];
            if (v == uint32_t(u)) continue;
            const uint64_t dv = g.out_off[v + 1] - g.out_off[v];
            if (!(dv < du || (dv == du && v < uint32_t(u)))) {
                ++up;
                continue;
            }
            ++down;
            const uint32_t *b = g.out_adj.data() + g.out_off[v], *e = g.out_adj.data() + g.out_off[v + 1];
            if (!std::binary_search(b, e, uint32_t(u))) { ok.store(false); break; }
        }
    }
    return ok.load() && up == down;
}

int graph_from_arcs(uint32_t n, std::vector<uint32_t> &src, std::vector<uint32_t> &dst,
                    HostGraph &g) {
    if (src.size() != dst.size()) return set_error(CUTS_ERR_ARG, "src/dst length mismatch");
    for (size_t i = 0; i < src.size(); ++i)
        if (src[i] >= n || dst[i] >= n)
            return set_error(CUTS_ERR_ARG, "arc endpoint out of range");
    g = HostGraph();
    g.n = n;
    build_one_csr(n, src, dst, g.out_off, g.out_adj);
    g.arcs = g.out_off[n];
    g.symmetric = check_symmetric(g);
    if (!g.symmetric) build_one_csr(n, dst, src, g.in_off, g.in_adj);
    std::vector<uint32_t>().swap(src);
    std::vector<uint32_t>().swap(dst);
    return CUTS_OK;
}

int graph_from_csr(uint32_t n, const uint64_t *out_off, const uint32_t *out_adj,
                   const uint64_t *in_off, const uint32_t *in_adj, HostGraph &g) {
    if (!out_off || (n > 0 && !out_adj && out_off[n] > 0))
        return set_error(CUTS_ERR_ARG, "null CSR array");
    if (in_adj && !in_off) return set_error(CUTS_ERR_ARG, "in_adj without in_off");
    if (in_off && !in_adj && n > 0 && in_off[n] > 0)
        return set_error(CUTS_ERR_ARG, "in_off without in_adj");
    g = HostGraph();
    g.n = n;
    auto adopt = [&](const uint64_t *off, const uint32_t *adj, std::vector<uint64_t> &o,
                     std::vector<uint32_t> &a) -> int {
        if (off[0] != 0) return set_error(CUTS_ERR_ARG, "CSR offsets must start at 0");
        o.assign(off, off + size_t(n) + 1);
        if (off[n] > 0) a.assign(adj, adj + off[n]);
        std::atomic<int> bad{0};
        #pragma omp parallel for schedule(dynamic, 4096)
        for (int64_t v = 0; v < int64_t(n); ++v) {
            if (o[v + 1] < o[v]) { bad = 1; continue; }
            for (uint64_t x = o[v]; x < o[v + 1]; ++x) {
                if (a[x] >= n || (x > o[v] && a[x] <= a[x - 1])) { bad = 2; break; }
            }
        }
        if (bad == 1) return set_error(CUTS_ERR_ARG, "CSR offsets not monotone");
        if (bad == 2) return set_error(CUTS_ERR_ARG, "CSR list not strictly sorted or out of range");
        return CUTS_OK;
    };
    int rc = adopt(out_off, out_adj, g.out_off, g.out_adj);
    if (rc) return rc;
    g.arcs = g.out_off[n];
    if (in_off) {
        rc = adopt(in_off, in_adj, g.in_off, g.in_adj);
        if (rc) return rc;
        if (g.in_off[n] != g.arcs) return set_error(CUTS_ERR_ARG, "in/out arc counts differ");
        g.symmetric = g.in_off == g.out_off && g.in_adj == g.out_adj;
        if (g.symmetric) {
            std::vector<uint64_t>().swap(g.in_off);
            std::vector<uint32_t>().swap(g.in_adj);
        }
    } else {
        if (!check_symmetric(g))
            return set_error(CUTS_ERR_ARG, "in-lists omitted but the graph is not symmetric");
        g.symmetric = true;
    }
    return CUTS_OK;
}

// The file's bytes, mapped read-only (the page cache, no copy); unmapped on
// destruction.
struct MappedFile {
    const char *data = nullptr;
    size_t size = 0;
    ~MappedFile() {
        if (data) munmap(const_cast<char *>(data), size);
    }
};

int load_graph_text(const std::string &path, HostGraph &g) {
    MappedFile mf;
    {
        const int fd = open(path.c_str(), O_RDONLY);
        if (fd < 0) return set_error(CUTS_ERR_IO, "load graph file failed: " + path);
        struct stat st;
        if (fstat(fd, &st) != 0 || !S_ISREG(st.st_mode)) {
            close(fd);
            return set_error(CUTS_ERR_IO, "load graph file failed (not a regular file): " + path);
        }
        mf.size = size_t(st.st_size);
        if (mf.size) {
            void *m = mmap(nullptr, mf.size, PROT_READ, MAP_PRIVATE | MAP_POPULATE, fd, 0);
            if (m == MAP_FAILED) {
                close(fd);
                return set_error(CUTS_ERR_IO, "cannot map " + path);
            }
            mf.data = static_cast<const char *>(m);
        }
        close(fd);
    }
    if (!mf.size) return set_error(CUTS_ERR_PARSE, "first line must hold the vertex count: " + path);
    const char *p = mf.data, *end = mf.data + mf.size;
    const char *nl = static_cast<const char *>(std::memchr(p, '\n', size_t(end - p)));
    long long V;
    if (!parse_int(p, nl ? nl : end, V) || V < 0)
        return set_error(CUTS_ERR_PARSE, "first line must hold the vertex count: " + path);
    const char *body = nl ? nl + 1 : end;
    // split the body into per-thread ranges at line starts
    int T = std::max(1, omp_get_max_threads());
    size_t blen = size_t(end - body);
    if (blen < (size_t(1) << 20)) T = 1;
    std::vector<const char *> cut(T + 1);
    cut[0] = body;
    cut[T] = end;
    for (int t = 1; t < T; ++t) {
        const char *c = body + blen * t / T;
        if (c < cut[t - 1]) c = cut[t - 1];
        const char *q = static_cast<const char *>(std::memchr(c, '\n', size_t(end - c)));
        cut[t] = q ? q + 1 : end;
    }
    std::vector<std::vector<uint32_t>> ls(T), ld(T);
    std::vector<int> err(T, 0);
    #pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        const char *s = cut[t], *e = cut[t + 1];
        // filled through locals and moved out at the end: vectors side by
        // side in ls / ld would share cache lines between the threads
        std::vector<uint32_t> vs, vd;
        vs.reserve(size_t(e - s) / 8);
        vd.reserve(size_t(e - s) / 8);
        while (s < e) {
            const char *le = static_cast<const char *>(std::memchr(s, '\n', size_t(e - s)));
            if (!le) le = e;
            const char *tab = static_cast<const char *>(std::memchr(s, '\t', size_t(le - s)));
            if (tab) {
                long long a, b;
                if (!parse_int(s, tab, a) || !parse_int(tab + 1, le, b)) { err[t] = 1; break; }
                if (a < 0 || b < 0 || a >= V || b >= V) { err[t] = 2; break; }
                vs.push_back(uint32_t(a));
                vd.push_back(uint32_t(b));
            }
            s = le + 1;
        }
        ls[t] = std::move(vs);
        ld[t] = std::move(vd);
    }
    for (int t = 0; t < T; ++t) {
        if (err[t] == 1) return set_error(CUTS_ERR_PARSE, "unparsable arc line in " + path);
        if (err[t] == 2) return set_error(CUTS_ERR_PARSE, "arc endpoint outside [0, V) in " + path);
    }
    std::vector<size_t> at(size_t(T) + 1, 0);
    for (int t = 0; t < T; ++t) at[t + 1] = at[t] + ls[t].size();
    std::vector<uint32_t> src(at[T]), dst(at[T]);
    #pragma omp parallel for num_threads(T) schedule(static, 1)
    for (int t = 0; t < T; ++t) {
        std::copy(ls[t].begin(), ls[t].end(), src.begin() + at[t]);
        std::copy(ld[t].begin(), ld[t].end(), dst.begin() + at[t]);
        std::vector<uint32_t>().swap(ls[t]);
        std::vector<uint32_t>().swap(ld[t]);
    }
    return graph_from_arcs(uint32_t(V), src, dst, g);
}

int write_graph_text(const std::string &path, const HostGraph &g) {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return set_error(CUTS_ERR_IO, "cannot write " + path);
    std::vector<char> buf(1 << 22);
    size_t pos = 0;
    auto flush = [&]() { std::fwrite(buf.data(), 1, pos, f); pos = 0; };
    auto put_u = [&](uint64_t x) {
        auto r = std::to_chars(buf.data() + pos, buf.data() + buf.size(), x);
        pos = size_t(r.ptr - buf.data());
    };
    put_u(g.n);
    buf[pos++] = '\n';
    for (uint32_t u = 0; u < g.n; ++u) {
        for (uint64_t a = g.out_off[u]; a < g.out_off[u + 1]; ++a) {
            if (pos + 32 > buf.size()) flush();
            put_u(u);
            buf[pos++] = '\t';
            put_u(g.out_adj[a]);
            buf[pos++] = '\n';
        }
    }
    flush();
    std::fclose(f);
    return CUTS_OK;
}

// Binary CSR cache: "CUTSCSR1", n, arcs, symmetric flag, then out_off[n+1],
// out_adj[arcs] and, for a directed graph, in_off[n+1], in_adj[arcs]
// (little-endian u64 / u32).  Loading it skips text parsing and sorting.
static const char kCsrMagic[8] = {'C', 'U', 'T', 'S', 'C', 'S', 'R', '1'};

int save_graph_binary(const std::string &path, const HostGraph &g) {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) return set_error(CUTS_ERR_IO, "cannot write " + path);
    const uint64_t hdr[3] = {g.n, g.arcs, g.symmetric ? 1ull : 0ull};
    bool ok = std::fwrite(kCsrMagic, 1, 8, f) == 8 && std::fwrite(hdr, 8, 3, f) == 3;
    auto put = [&](const void *p, size_t sz, size_t cnt) {
        ok = ok && (cnt == 0 || std::fwrite(p, sz, cnt, f) == cnt);
    };
    put(g.out_off.data(), 8, size_t(g.n) + 1);
    put(g.out_adj.data(), 4, g.arcs);
    if (!g.symmetric) {
        put(g.in_off.data(), 8, size_t(g.n) + 1);
        put(g.in_adj.data(), 4, g.arcs);
    }
    std::fclose(f);
    return ok ? CUTS_OK : set_error(CUTS_ERR_IO, "short write to " + path);
}

int load_graph_binary(const std::string &path, HostGraph &g) {
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return set_error(CUTS_ERR_IO, "load graph file failed: " + path);
    std::unique_ptr<FILE, int (*)(FILE *)> hold(f, std::fclose);
    char magic[8];
    uint64_t hdr[3];
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, kCsrMagic, 8) != 0 ||
        std::fread(hdr, 8, 3, f) != 3 || hdr[0] > 0xFFFFFFFFull)
        return set_error(CUTS_ERR_PARSE, "not a cuts binary CSR file: " + path);
    g = HostGraph();
    g.n = uint32_t(hdr[0]);
    g.arcs = hdr[1];
    g.symmetric = hdr[2] != 0;
    auto get = [&](auto &vec, size_t cnt) {
        vec.resize(cnt);
        return cnt == 0 || std::fread(vec.data(), sizeof(vec[0]), cnt, f) == cnt;
    };
    bool ok = get(g.out_off, size_t(g.n) + 1) && get(g.out_adj, g.arcs);
    if (ok && !g.symmetric) ok = get(g.in_off, size_t(g.n) + 1) && get(g.in_adj, g.arcs);
    if (!ok || g.out_off[0] != 0 || g.out_off[g.n] != g.arcs)
        return set_error(CUTS_ERR_PARSE, "truncated or inconsistent binary CSR: " + path);
    for (uint64_t a = 0; a < g.arcs; ++a)
        if (g.out_adj[a] >= g.n) return set_error(CUTS_ERR_PARSE, "arc endpoint out of range in " + path);
    return CUTS_OK;
}

}  // namespace cuts
