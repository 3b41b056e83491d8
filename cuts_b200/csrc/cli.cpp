// cli.cpp -- the `cuts` command, a client of the C ABI.
//
//   cuts <data_graph_path> <query_graph_path> [trunks]
//
// Same argv, progress lines and result line "<data>,<query>,<ms>ms,<count>"
// as the reference (main.cu:24-46, host_funcs.cu:39-171).  The match dump
// to ./ans.txt, hard-coded off in the reference (main.cu:31), is enabled by
// the environment variable CUTS_WRITE_TO_DISK=1.  Errors print the message
// and exit(-1), as the reference's chkerr does (host_funcs.cu:20-27); an
// invalid trunks value (the reference divides by zero) is such an error.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>

#include "../../include/cuts_b200.h"

int main(int argc, char **argv) {
    if (argc < 3) {
        std::cout << "args data_graph path,query_graph_path,first depth trunks(optional)" << std::endl;
        std::exit(-1);
    }
    const char *wenv = std::getenv("CUTS_WRITE_TO_DISK");
    const int write_to_disk = wenv && std::strcmp(wenv, "0") != 0 && wenv[0] != 0;
    uint32_t trunks = 0;
    if (argc > 3) {
        const long t = std::atol(argv[3]);
        if (t <= 0) {
            std::cout << "invalid trunks: " << argv[3] << " (must be a positive integer)" << std::endl;
            std::exit(-1);
        }
        trunks = uint32_t(t);
    }
    uint64_t count = 0;
    float ms = 0;
    const int rc = cuts_search(argv[2], argv[1], write_to_disk, trunks, &count, &ms);
    if (rc != CUTS_OK) {
        std::cout << cuts_last_error() << std::endl;
        std::exit(-1);
    }
    return 0;
}
