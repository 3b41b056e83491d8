// ref_load_main.cpp -- times the reference's own data-graph loader.
//
// TEST / MEASUREMENT INFRASTRUCTURE ONLY.  Linked against the reference's
// unmodified graph.cpp / util.cpp / score.cpp / common.cpp (compiled in
// place by oracle/Makefile into oracle/_ref/ref_load).  For each data-graph
// file it constructs the reference's Graph(1, path) -- file_reader's
// std::set parse (util.cpp:19-52) plus the CSR and signature build
// (graph.cpp:18-61) -- and prints "<path> V=<n> E=<arcs> seconds=<t>", the
// baseline for this repository's parallel loader.
#include "graph.h"

#include <chrono>
#include <cstdio>

int main(int argc, char **argv) {
    for (int a = 1; a < argc; ++a) {
        const auto t0 = std::chrono::steady_clock::now();
        Graph g(1, argv[a]);
        const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::printf("%s V=%u E=%u seconds=%.3f\n", argv[a], g.V, g.E, s);
    }
    return 0;
}
