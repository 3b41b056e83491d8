// ref_load_main.cpp -- runs the reference's own data-graph loader.
//
// TEST / MEASUREMENT INFRASTRUCTURE ONLY.  Linked against the reference's
// unmodified graph.cpp / util.cpp / score.cpp / common.cpp (compiled in
// place by oracle/Makefile into oracle/_ref/ref_load).  For each data-graph
// file it constructs the reference's Graph(1, path) -- file_reader's
// std::set parse (util.cpp:19-52) plus the CSR and signature build
// (graph.cpp:18-61).
//
//   ref_load <path>...         prints "<path> V=<n> E=<arcs> seconds=<t>",
//                              the baseline for this repository's loader
//   ref_load --csr <path>...   prints, per file, the CSR the reference built:
//                              "V E", then four lines -- out-offsets,
//                              out-neighbours, in-offsets, in-neighbours --
//                              space separated (the loader parity fixtures)
#include "graph.h"

#include <chrono>
#include <cstdio>
#include <cstring>

static void print_row(const unsigned int *a, unsigned int n) {
    for (unsigned int i = 0; i < n; ++i) std::printf(i ? " %u" : "%u", a[i]);
    std::printf("\n");
}

int main(int argc, char **argv) {
    const bool csr = argc > 1 && std::strcmp(argv[1], "--csr") == 0;
    for (int a = csr ? 2 : 1; a < argc; ++a) {
        const auto t0 = std::chrono::steady_clock::now();
        Graph g(1, argv[a]);
        const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (!csr) {
            std::printf("%s V=%u E=%u seconds=%.3f\n", argv[a], g.V, g.E, s);
            continue;
        }
        std::printf("%u %u\n", g.V, g.E);
        print_row(g.neighbors_offset, g.V + 1);
        print_row(g.neighbors, g.neighbors_offset[g.V]);
        print_row(g.r_neighbors_offset, g.V + 1);
        print_row(g.r_neighbors, g.r_neighbors_offset[g.V]);
    }
    return 0;
}
