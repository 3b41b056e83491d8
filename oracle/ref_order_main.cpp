// ref_order_main.cpp -- test harness around the reference's own host code.
//
// TEST INFRASTRUCTURE ONLY.  Linked against the reference's unmodified
// graph.cpp / score.cpp / util.cpp / common.cpp (compiled in place by
// oracle/Makefile into oracle/_ref/ref_order).  For each query file given
// on the command line it constructs the reference's Graph(0, path)
// (graph.cpp:18-61, which runs sort_search_order, graph.cpp:62-134) and
// prints one line:
//     <path> order=<o0,o1,...> P=<i:j,j;...> C=<i:j,j;...>
// so the oracle's and the product's orders can be compared with the
// reference's byte for byte.
#include "graph.h"

#include <cstdio>

int main(int argc, char **argv) {
    for (int a = 1; a < argc; ++a) {
        Graph q(0, argv[a]);
        std::printf("%s order=", argv[a]);
        for (unsigned i = 0; i < q.V; ++i) std::printf(i ? ",%u" : "%u", q.order_sequence[i]);
        std::printf(" P=");
        for (unsigned i = 0; i < q.V; ++i) {
            std::printf(i ? ";%u:" : "%u:", i);
            for (unsigned x = q.parents_offset[i]; x < q.parents_offset[i + 1]; ++x)
                std::printf(x > q.parents_offset[i] ? ",%u" : "%u", q.parents[x]);
        }
        std::printf(" C=");
        for (unsigned i = 0; i < q.V; ++i) {
            std::printf(i ? ";%u:" : "%u:", i);
            for (unsigned x = q.children_offset[i]; x < q.children_offset[i + 1]; ++x)
                std::printf(x > q.children_offset[i] ? ",%u" : "%u", q.children[x]);
        }
        std::printf("\n");
    }
    return 0;
}
