// asdm_gen.out — the seeded workload generators as a host-only program
// (compiled from csrc/host_graph.cpp with g++; it links neither CUDA nor
// libasdm_b200.so).  A process that times another implementation on these
// workloads can write its input files with it without loading this library.
//
//   asdm_gen.out graph   <n> <m> <gamma> <labels> <zipf_s> <seed> <out.graph>
//   asdm_gen.out queries <n> <m> <gamma> <labels> <zipf_s> <seed> <list> <dir>
//
// `graph` writes the Chung-Lu data graph in 't/v/e' text; `queries` rebuilds
// the same graph and writes one random-walk query per line of <list>
// ("<size> <seed> <density> <name>"; density 0 any, 1 dense, 2 sparse) to
// <dir>/<name>.  No counterpart in the reference, which ships its query sets
// as files.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>

#include "asdm.h"

namespace {

[[noreturn]] void die(const char *what, int rc) {
    std::cerr << what << ": " << asdm_last_error() << " (status " << rc << ")" << std::endl;
    std::exit(1);
}

[[noreturn]] void usage() {
    std::cerr << "usage: asdm_gen.out graph <n> <m> <gamma> <labels> <zipf_s> <seed> <out.graph>\n"
                 "       asdm_gen.out queries <n> <m> <gamma> <labels> <zipf_s> <seed> <list> <dir>"
              << std::endl;
    std::exit(2);
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 9) usage();
    const std::string what = argv[1];
    const uint32_t n = (uint32_t)std::strtoul(argv[2], nullptr, 10);
    const uint64_t m = std::strtoull(argv[3], nullptr, 10);
    const double gamma = std::strtod(argv[4], nullptr);
    const uint32_t labels = (uint32_t)std::strtoul(argv[5], nullptr, 10);
    const double zipf = std::strtod(argv[6], nullptr);
    const uint64_t seed = std::strtoull(argv[7], nullptr, 10);
    asdm_host_graph *g = nullptr;
    int rc = asdm_gen_chung_lu(n, m, gamma, labels, zipf, seed, &g);
    if (rc != ASDM_OK) die("graph generator", rc);
    if (what == "graph") {
        if ((rc = asdm_host_graph_write(g, argv[8])) != ASDM_OK) die("graph write", rc);
    } else if (what == "queries" && argc >= 10) {
        std::ifstream list(argv[8]);
        if (!list) {
            std::cerr << "cannot open " << argv[8] << std::endl;
            return 1;
        }
        std::string line;
        while (std::getline(list, line)) {
            std::istringstream is(line);
            uint32_t size = 0;
            uint64_t qseed = 0;
            int density = 0;
            std::string name;
            if (!(is >> size >> qseed >> density >> name)) continue;
            asdm_host_graph *q = nullptr;
            if ((rc = asdm_gen_query(g, size, density, qseed, &q)) != ASDM_OK) die("query generator", rc);
            const std::string path = std::string(argv[9]) + "/" + name;
            if ((rc = asdm_host_graph_write(q, path.c_str())) != ASDM_OK) die("query write", rc);
            asdm_host_graph_free(q);
        }
    } else {
        usage();
    }
    asdm_host_graph_free(g);
    return 0;
}
