// prepare.out — drop-in for the reference's plan-cache precomputation
// (executable/prepare.cpp:12-73): `prepare.out -q <query> -d <data> -s <card>`.
//
// The reference samples cardinalities of query-vertex subsets and writes its
// DP structures plus the subset->cardinality map.  Here the cache holds the
// *exact* match counts of every connected induced sub-query with at most six
// vertices (counted on the GPU, capped at 1e9 and at 1 s each), keyed by the
// same bitmask (bit u = query vertex u); ASDMatch.out -s reads it back and the
// planner uses those cardinalities for the prefixes it considers.  The file
// has no bag records (the reference's reader expects its own bags; this
// library reads both layouts).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <vector>
#include <algorithm>

#include "asdm.h"

namespace {

std::string option(int argc, char **argv, const char *flag) {
    for (int i = 1; i < argc; ++i)
        if (std::strcmp(argv[i], flag) == 0) return i + 1 < argc ? argv[i + 1] : "";
    return "";
}

[[noreturn]] void die(const char *what, int rc) {
    std::cerr << what << ": " << asdm_last_error() << " (status " << rc << ")" << std::endl;
    std::exit(rc == ASDM_ERR_IO ? 255 : 1);
}

}  // namespace

int main(int argc, char **argv) {
    const std::string qpath = option(argc, argv, "-q"), dpath = option(argc, argv, "-d");
    const std::string cpath = option(argc, argv, "-s");
    asdm_host_graph *q = nullptr, *g = nullptr;
    int rc = asdm_host_graph_load(qpath.c_str(), &q);
    if (rc == ASDM_ERR_IO) { std::cout << "Can not open file " << qpath << " ." << std::endl; return 255; }
    if (rc) die("query", rc);
    rc = asdm_host_graph_load(dpath.c_str(), &g);
    if (rc == ASDM_ERR_IO) { std::cout << "Can not open file " << dpath << " ." << std::endl; return 255; }
    if (rc) die("data graph", rc);
    uint32_t gn, gl, qn, ql;
    uint64_t gm2, qm2;
    asdm_host_graph_info(g, &gn, &gm2, &gl);
    asdm_host_graph_info(q, &qn, &qm2, &ql);
    const uint32_t *goff, *gnbr, *glab, *qoff, *qnbr, *qlab;
    asdm_host_graph_csr(g, &goff, &gnbr, &glab);
    asdm_host_graph_csr(q, &qoff, &qnbr, &qlab);
    asdm_graph *dg = nullptr;
    if ((rc = asdm_graph_upload(goff, gnbr, glab, gn, gm2, gl, &dg))) die("upload", rc);
    asdm_cs *cs = nullptr;
    int nonempty = 0;
    if ((rc = asdm_candidate_space(dg, qoff, qnbr, qlab, qn, &cs, &nonempty))) die("candidate space", rc);
    asdm_cs_free(cs);
    if (!nonempty) return 0;  // buildCandCFL() == false: the reference returns before writing

    auto t0 = std::chrono::steady_clock::now();
    asdm_card *card = nullptr;
    asdm_card_create(&card);
    const uint32_t maxk = qn < 6 ? qn : 6;
    auto adjacent = [&](uint32_t a, uint32_t b) {
        for (uint32_t e = qoff[a]; e < qoff[a + 1]; ++e)
            if (qnbr[e] == b) return true;
        return false;
    };
    // connected subsets grown one neighbour at a time (each visited once)
    std::vector<uint64_t> frontier;
    std::vector<char> seen_small;
    std::vector<uint64_t> all;
    for (uint32_t u = 0; u < qn; ++u) frontier.push_back(1ull << u);
    for (uint32_t k = 1; k <= maxk && !frontier.empty(); ++k) {
        std::vector<uint64_t> next;
        for (uint64_t m : frontier) {
            all.push_back(m);
            if (k == maxk) continue;
            for (uint32_t u = 0; u < qn; ++u) {
                if (!(m >> u & 1)) continue;
                for (uint32_t e = qoff[u]; e < qoff[u + 1]; ++e) {
                    const uint64_t m2 = m | (1ull << qnbr[e]);
                    if (m2 != m) next.push_back(m2);
                }
            }
        }
        std::sort(next.begin(), next.end());
        next.erase(std::unique(next.begin(), next.end()), next.end());
        frontier.swap(next);
    }
    for (uint64_t m : all) {
        std::vector<uint32_t> verts, labels, edges;
        for (uint32_t u = 0; u < qn; ++u)
            if (m >> u & 1) verts.push_back(u);
        for (uint32_t a = 0; a < verts.size(); ++a) {
            labels.push_back(qlab[verts[a]]);
            for (uint32_t b = a + 1; b < verts.size(); ++b)
                if (adjacent(verts[a], verts[b])) {
                    edges.push_back(a);
                    edges.push_back(b);
                }
        }
        asdm_host_graph *sq = nullptr;
        if ((rc = asdm_host_graph_from_edges((uint32_t)verts.size(), labels.data(), edges.size() / 2, edges.data(), &sq)))
            die("sub-query", rc);
        const uint32_t *so, *sn, *sl;
        uint32_t sqn;
        uint64_t sqm2;
        asdm_host_graph_info(sq, &sqn, &sqm2, nullptr);
        asdm_host_graph_csr(sq, &so, &sn, &sl);
        asdm_run_opts o{};
        o.mode = ASDM_MODE_COUNT;
        o.time_limit_s = 1.0;
        o.count_limit = 1000000000ull;
        asdm_run_stats st{};
        rc = asdm_count_query(dg, so, sn, sl, sqn, &o, &st);
        if (rc != ASDM_OK && rc != ASDM_ERR_LIMIT && rc != ASDM_ERR_TIMEOUT && rc != ASDM_ERR_OVERFLOW) die("count", rc);
        double value = (double)st.count;
        if (rc == ASDM_ERR_LIMIT || rc == ASDM_ERR_OVERFLOW) value = (double)o.count_limit;
        if (rc == ASDM_ERR_TIMEOUT) value = std::max(value, 1.0);  // a lower bound: what was counted in time
        asdm_card_set(card, m, value);
        asdm_host_graph_free(sq);
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if ((rc = asdm_card_write(card, cpath.c_str(), secs))) die("write", rc);
    asdm_card_free(card);
    asdm_graph_free(dg);
    asdm_host_graph_free(q);
    asdm_host_graph_free(g);
    return 0;
}
