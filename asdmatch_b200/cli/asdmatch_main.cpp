// ASDMatch.out — drop-in for the reference's matching executable
// (main.cpp:11-147), running the matching and counting path on the B200
// through libasdm_b200.so.
//
//   ASDMatch.out -q <query> -d <data> [-s <card>] [-m <KB>] [-r <report>] [-c <csv>]
//                [-e <embeddings>] [-t <seconds>]
//
// Flags as in the reference (utility/command.cpp:7-29): the value is the token
// after the flag, "" when absent; -m is read with atoi and 0 means 16e5 KB
// (main.cpp:21-23); -r redirects the text report (main.cpp:28-30); -c writes
// the |Vg| x |Vq| local-count CSV (main.cpp:135-146), which the reference
// produces only when built with ALL_LEVEL + LOCAL_COUNT.  Extensions: -e
// writes the sorted embedding set in storeMatches format
// (matching/join.cpp:1099-1107), -t sets a device time limit.  -a and -i are
// accepted and ignored, like the reference.  Counts are always exact (the
// reference's ALL_LEVEL semantics); a count of 2^64 or more is reported as
// "Number of matches: overflow (at least 18446744073709551616)".
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "asdm.h"

namespace {

std::string option(int argc, char **argv, const char *flag) {
    for (int i = 1; i < argc; ++i)
        if (std::strcmp(argv[i], flag) == 0) return i + 1 < argc ? argv[i + 1] : "";
    return "";
}

double since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

[[noreturn]] void die(const char *what, int rc) {
    std::cerr << what << ": " << asdm_last_error() << " (status " << rc << ")" << std::endl;
    std::exit(rc == ASDM_ERR_IO ? 255 : 1);
}

}  // namespace

int main(int argc, char **argv) {
    const std::string qpath = option(argc, argv, "-q"), dpath = option(argc, argv, "-d");
    const std::string report = option(argc, argv, "-r"), csv = option(argc, argv, "-c");
    const std::string emb = option(argc, argv, "-e"), card = option(argc, argv, "-s");
    int memKB = std::atoi(option(argc, argv, "-m").c_str());
    if (memKB == 0) memKB = 16e5;
    const double tlimit = std::atof(option(argc, argv, "-t").c_str());

    asdm_host_graph *q = nullptr, *g = nullptr;
    int rc = asdm_host_graph_load(qpath.c_str(), &q);
    if (rc == ASDM_ERR_IO) { std::cout << "Can not open file " << qpath << " ." << std::endl; return 255; }
    if (rc) die("query", rc);
    rc = asdm_host_graph_load(dpath.c_str(), &g);
    if (rc == ASDM_ERR_IO) { std::cout << "Can not open file " << dpath << " ." << std::endl; return 255; }
    if (rc) die("data graph", rc);

    std::ofstream outFile;
    if (!report.empty()) outFile.open(report);
    std::ostream &out = report.empty() ? std::cout : outFile;

    uint32_t gn = 0, gl = 0, qn = 0, ql = 0;
    uint64_t gm2 = 0, qm2 = 0;
    asdm_host_graph_info(g, &gn, &gm2, &gl);
    asdm_host_graph_info(q, &qn, &qm2, &ql);
    const uint32_t *goff, *gnbr, *glab, *qoff, *qnbr, *qlab;
    asdm_host_graph_csr(g, &goff, &gnbr, &glab);
    asdm_host_graph_csr(q, &qoff, &qnbr, &qlab);
    asdm_graph *dg = nullptr;
    if ((rc = asdm_graph_upload(goff, gnbr, glab, gn, gm2, gl, &dg))) die("upload", rc);

    auto t0 = std::chrono::steady_clock::now();
    asdm_cs *cs = nullptr;
    int nonempty = 0;
    if ((rc = asdm_candidate_space(dg, qoff, qnbr, qlab, qn, &cs, &nonempty))) die("candidate space", rc);
    if (!nonempty) return 0;  // buildCandCFL() == false: the reference returns silently
    out << "Filtering time (s): " << since(t0) << std::endl;
    out << "FHD time (s): " << 0.0 << std::endl;
    asdm_card *cache = nullptr;
    if (!card.empty()) {
        // -s: the plan cache replaces cardinality estimation (main.cpp:88-99)
        if ((rc = asdm_card_load(card.c_str(), &cache))) die("card", rc);
        double secs = 0;
        asdm_card_info(cache, nullptr, nullptr, &secs);
        out << "dp time: " << secs << std::endl;
    }
    t0 = std::chrono::steady_clock::now();
    asdm_plan *plan = nullptr;
    if ((rc = cache ? asdm_plan_create_card(cs, cache, &plan) : asdm_plan_create(cs, nullptr, &plan))) die("plan", rc);
    asdm_card_free(cache);
    out << "Planning Time: " << since(t0) << std::endl;
    double cost = 0.0;
    asdm_plan_cost(plan, &cost);
    out << "cost: " << cost << std::endl;

    asdm_run_opts o{};
    o.mode = ASDM_MODE_COUNT;
    o.budget_bytes = (uint64_t)1024 * (uint64_t)memKB;
    o.time_limit_s = tlimit;
    std::vector<uint64_t> local;
    if (!csv.empty()) {
        o.mode |= ASDM_MODE_LOCAL;
        local.assign((uint64_t)gn * qn, 0);
        o.local_counts = local.data();
    }
    asdm_run_stats st{};
    std::vector<uint32_t> rows;
    t0 = std::chrono::steady_clock::now();
    if (!emb.empty()) {
        // size the buffer with a counting pass first
        asdm_run_opts c = o;
        c.mode = ASDM_MODE_COUNT;
        c.local_counts = nullptr;
        if ((rc = asdm_run_plan(cs, plan, &c, &st))) die("count", rc);
        rows.assign(st.count * qn, 0);
        o.mode |= ASDM_MODE_EMBED;
        o.embeddings = rows.data();
        o.emb_capacity = st.count;
    }
    rc = asdm_run_plan(cs, plan, &o, &st);
    if (rc == ASDM_ERR_OVERFLOW) {
        // the count is at least 2^64: a uint64 cannot hold it (the reference's
        // size_t would wrap); the report says so instead of a wrapped number
        out << "Execution Time: " << since(t0) << std::endl;
        out << "Number of matches: overflow (at least 18446744073709551616)" << std::endl;
        out << "Number of intersections: " << st.intersections << std::endl;
        asdm_plan_free(plan);
        asdm_cs_free(cs);
        asdm_graph_free(dg);
        asdm_host_graph_free(q);
        asdm_host_graph_free(g);
        return 0;
    }
    if (rc) die("enumeration", rc);
    out << "Execution Time: " << since(t0) << std::endl;
    out << "Number of matches: " << st.count << std::endl;
    out << "Number of fixed attributes: " << 0 << std::endl;
    out << "Number of intersections: " << st.intersections << std::endl;
    out << "Number of fix cases: " << 0 << std::endl;

    if (!csv.empty()) {
        std::ofstream os(csv);
        std::string line;
        for (uint32_t v = 0; v < gn; ++v) {
            line.clear();
            for (uint32_t u = 0; u < qn; ++u) {
                line += std::to_string(local[(uint64_t)v * qn + u]);
                if (u + 1 != qn) line += ',';
            }
            line += '\n';
            os << line;
        }
    }
    if (!emb.empty()) {
        std::ofstream os(emb);
        os << st.emb_rows << "\n";
        std::string line;
        for (uint64_t r = 0; r < st.emb_rows; ++r) {
            line.clear();
            for (uint32_t u = 0; u < qn; ++u) {
                line += std::to_string(rows[r * qn + u]);
                line += ' ';
            }
            line += '\n';
            os << line;
        }
    }
    asdm_plan_free(plan);
    asdm_cs_free(cs);
    asdm_graph_free(dg);
    asdm_host_graph_free(q);
    asdm_host_graph_free(g);
    return 0;
}
