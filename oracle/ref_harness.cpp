// Test infrastructure only: a driver around the reference implementation's own
// matching path, compiled from the reference sources by oracle/ref.mk into
// oracle/_ref/.  Nothing in the product links or calls this file.
//
// It runs the same sequence of reference calls as the reference's ASDMatch.out
// entry point (main.cpp:11-147 of the reference):
//   Graph::loadGraphFromTextFile -> CandidateSpace::buildCandCFL ->
//   setQueryGraphWeights -> buildFHD/HyperTree::buildFromTD -> reorderBags ->
//   smallCard + SubsetStructure::optimalPlanDP/reverseDP (or a .card via -s) ->
//   optCostPlan/simplePlan -> adaptiveShareJoin
// with two harness differences:
//   1. the per-bag trie root vector is sized *after* reorderBags(), because
//      reorderBags may append a virtual global bag and the reference's own
//      entry point sizes it before (main.cpp:51 vs main.cpp:69), which makes
//      adaptiveGlobalJoin index one past the end (matching/adaptive.cpp:304);
//   2. extra outputs for parity checks:
//        -w <file>  candidate space dump: "C <u> <n> v..." lines, then the
//                   reference's CandidateSpace::writeToStream listing
//                   (relation/candidate_space.cpp:489-505);
//        -e <file>  (COLLECT_RESULT builds) the embedding set, sorted, in the
//                   reference's storeMatches format (matching/join.cpp:1099-1107);
//        -b <file>  the data graph in the reference's binary cache format
//                   (Graph::writeToStream, relation/graph.cpp:316-332), then exit.
//   3. many queries against one data graph (-Q <list> -O <dir> [-T s] [-J n]):
//      the data graph is read once; each query of the list file (one path
//      per line) runs in a child process forked from that state, with its
//      report in <dir>/q<k>.out (k = line number, from 0), at most n children
//      at a time, each killed after s seconds.  One line per query on
//      stdout: "Q <k> ok|timeout|signal <n>|exit <n> <wall seconds>".  Every
//      child starts from the same untouched state, as a fresh process would.
//      With -c (LOCAL_COUNT builds) each child writes its CSV to <dir>/q<k>.csv,
//      with -e (COLLECT_RESULT builds) its sorted embedding dump to <dir>/q<k>.emb.
// Build variants select the reference's compile-time modes (config/config.h:38-40):
//   ref_count : ALL_LEVEL                          (exact counts)
//   ref_local : ALL_LEVEL + LOCAL_COUNT            (+ |Vg|x|Vq| CSV via -c)
//   ref_embed : ALL_LEVEL + LOCAL_COUNT + COLLECT_RESULT (+ -e dump)
#include <signal.h>
#include <sys/wait.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <map>
#include <string>
#include <thread>
#include <vector>

#include "adaptive.h"
#include "candidate_space.h"
#include "command.h"
#include "estimator.h"
#include "join.h"
#include "optimizer.h"

static std::string option_after(int argc, char **argv, const char *flag) {
    for (int i = 1; i + 1 < argc; ++i)
        if (std::strcmp(argv[i], flag) == 0) return argv[i + 1];
    return "";
}

static double seconds_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// In list mode with -c, each child's CSV path (<dir>/q<k>.csv).
static std::string g_csv_path;
static std::string g_emb_path;  // list mode: this child's embedding dump

// One query against the loaded data graph g: the reference's ASDMatch.out
// sequence after its graph loads (main.cpp:27-147).
static int run_query(int argc, char **argv, Command &cmd, const std::string &qpath, Graph &g) {
    const std::string cardPath = cmd.getDPStructPath();
    const std::string csDump = option_after(argc, argv, "-w");
    const std::string embDump = g_emb_path.empty() ? option_after(argc, argv, "-e") : g_emb_path;
    int memKB = cmd.getMemoryBudget();
    if (memKB == 0) memKB = 16e5;
    const size_t budget = (size_t)1024 * memKB;

    Graph q;
    q.loadGraphFromTextFile(qpath);
    CandidateSpace cs(q, g);

    auto t0 = std::chrono::steady_clock::now();
    if (!cs.buildCandCFL()) {
        // The reference returns silently here (main.cpp:35-37); the harness
        // reports the empty candidate space explicitly so tests can see it.
        std::cout << "Empty candidate set" << std::endl;
        std::cout << "Number of matches: 0" << std::endl;
        return 0;
    }
    std::cout << "Filtering time (s): " << seconds_since(t0) << std::endl;

    if (!csDump.empty()) {
        std::ofstream os(csDump);
        for (VertexID u = 0; u < q.getNumVertices(); ++u) {
            os << "C " << u << " " << cs.candidateSet[u].size();
            for (VertexID v : cs.candidateSet[u]) os << " " << v;
            os << "\n";
        }
        cs.writeToStream(os);
    }

    cs.setQueryGraphWeights(q);
    t0 = std::chrono::steady_clock::now();
    FHD fhd;
    q.buildFHD(fhd);
    HyperTree t;
    t.buildFromTD(fhd);
    double fhdTime = seconds_since(t0);
    std::cout << "FHD time (s): " << fhdTime << std::endl;

    std::vector<std::vector<VertexID>> result;
    bool *visited = new bool[g.getNumVertices()];
    std::memset(visited, 0, sizeof(bool) * g.getNumVertices());
    VertexID *partMatch = new VertexID[q.getNumVertices()];
    VertexID **candidates = new VertexID *[q.getNumVertices()];
    const ui maxSize = cs.getMaxSize();
    for (ui i = 0; i < q.getNumVertices(); ++i) candidates[i] = new VertexID[maxSize];
    ui *candCount = new ui[q.getNumVertices()];
    std::memset(candCount, 0, sizeof(ui) * q.getNumVertices());

    reorderBags(q, t);
    // Harness difference 1: size the trie roots after the global bag exists.
    std::vector<TrieNode *> nodes(t.numNodes);
    for (ui i = 0; i < t.numNodes; ++i) nodes[i] = new TrieNode();

    std::vector<SubsetStructure> dp;
    ui numNodes = t.numNodes;
    if (t.newGlobalNode) --numNodes;
    double cardTime = 0.0;
    if (cardPath.empty()) {
        smallCard(q, cs);
        dp.resize(numNodes);
        t0 = std::chrono::steady_clock::now();
        for (VertexID nID = 0; nID < numNodes; ++nID) {
            std::vector<VertexID> local(t.nodes[nID].attributes,
                                        t.nodes[nID].attributes + t.nodes[nID].numAttributes);
            SubsetStructure s(local, q, false);
            s.optimalPlanDP(q, cs, visited, partMatch, candidates, candCount);
            s.reverseDP(q, cs);
            dp[nID] = s;
        }
        cardTime = seconds_since(t0);
    } else {
        std::ifstream ifs(cardPath, std::ios::binary);
        dp.resize(numNodes);
        for (VertexID nID = 0; nID < numNodes; ++nID) dp[nID].readFromStream(ifs);
        if (!loadSubsetToCard(ifs)) return 1;
        int scaled = 0;
        ifs.read(reinterpret_cast<char *>(&scaled), sizeof(int));
        cardTime = scaled / 10000.0;
    }
    cardTime += fhdTime;

    bool traverseAll = false;
#if defined(ALL_LEVEL) || defined(COLLECT_RESULT)
    traverseAll = true;
#endif
#ifdef LOCAL_COUNT
    gLocalCount = std::vector<std::vector<size_t>>(g.getNumVertices(),
                                                   std::vector<size_t>(q.getNumVertices(), 0));
#endif
    PrefixNode *pt = nullptr;
    double minCost = 0.0;
    t0 = std::chrono::steady_clock::now();
    if (numNodes != 1)
        optCostPlan(q, t, cs, pt, dp, minCost, 1, true, false);
    else
        simplePlan(q, t, cs, pt, dp, visited, partMatch, candidates, candCount, minCost, nullptr, false);
    std::cout << "Planning Time: " << seconds_since(t0) + cardTime << std::endl;
    std::cout << "cost: " << minCost << std::endl;

    size_t count = 0;
    t0 = std::chrono::steady_clock::now();
    adaptiveShareJoin(q, t, pt, cs, nodes, visited, result, count, traverseAll, budget, false);
    std::cout << "Execution Time: " << seconds_since(t0) << std::endl;
    std::cout << "Number of matches: " << count << std::endl;
    std::cout << "Number of intersections: " << gNumInterSection << std::endl;

#ifdef LOCAL_COUNT
    const std::string csvPath = g_csv_path.empty() ? cmd.getCountPath() : g_csv_path;
    if (!csvPath.empty()) {
        std::ofstream os(csvPath);
        for (VertexID v = 0; v < g.getNumVertices(); ++v) {
            for (VertexID u = 0; u < q.getNumVertices(); ++u) {
                os << gLocalCount[v][u];
                if (u + 1 != q.getNumVertices()) os << ",";
            }
            os << "\n";
        }
    }
#endif
#ifdef COLLECT_RESULT
    if (!embDump.empty()) {
        std::sort(result.begin(), result.end());
        std::ofstream os(embDump);
        storeMatches(result, os);
    }
#endif
    return 0;
}

// Harness difference 3: the queries of a list file, one forked child each.
static int run_list(int argc, char **argv, Command &cmd, Graph &g, const std::string &list) {
    const std::string outDir = option_after(argc, argv, "-O");
    const std::string tArg = option_after(argc, argv, "-T"), jArg = option_after(argc, argv, "-J");
    const double limit = tArg.empty() ? 0.0 : std::stod(tArg);
    const int jobs = std::max(1, jArg.empty() ? 1 : std::stoi(jArg));
    if (outDir.empty()) {
        std::cerr << "-Q needs -O <dir>" << std::endl;
        return 2;
    }
    std::vector<std::string> queries;
    {
        std::ifstream is(list);
        std::string line;
        while (std::getline(is, line))
            if (!line.empty()) queries.push_back(line);
    }
    struct Child { size_t k; std::chrono::steady_clock::time_point t0; bool killed; };
    std::map<pid_t, Child> running;
    size_t next = 0;
    std::cout.setf(std::ios::fixed);
    while (next < queries.size() || !running.empty()) {
        while (next < queries.size() && (int)running.size() < jobs) {
            std::cout.flush();
            const pid_t pid = fork();
            if (pid == 0) {
                const std::string out = outDir + "/q" + std::to_string(next) + ".out";
                if (!std::freopen(out.c_str(), "w", stdout)) _exit(3);
                if (!cmd.getCountPath().empty()) g_csv_path = outDir + "/q" + std::to_string(next) + ".csv";
                if (!option_after(argc, argv, "-e").empty()) g_emb_path = outDir + "/q" + std::to_string(next) + ".emb";
                const int rc = run_query(argc, argv, cmd, queries[next], g);
                std::cout.flush();
                std::fflush(stdout);
                _exit(rc);
            }
            if (pid < 0) {
                std::cerr << "fork failed" << std::endl;
                return 2;
            }
            running[pid] = Child{next, std::chrono::steady_clock::now(), false};
            ++next;
        }
        int wst = 0;
        const pid_t done = waitpid(-1, &wst, WNOHANG);
        if (done > 0) {
            auto it = running.find(done);
            if (it == running.end()) continue;
            const double wall = seconds_since(it->second.t0);
            std::cout << "Q " << it->second.k << " ";
            if (it->second.killed) std::cout << "timeout";
            else if (WIFSIGNALED(wst)) std::cout << "signal " << WTERMSIG(wst);
            else if (WEXITSTATUS(wst) != 0) std::cout << "exit " << WEXITSTATUS(wst);
            else std::cout << "ok";
            std::cout << " " << wall << std::endl;
            running.erase(it);
            continue;
        }
        for (auto &kv : running)
            if (limit > 0 && !kv.second.killed && seconds_since(kv.second.t0) > limit) {
                kill(kv.first, SIGKILL);
                kv.second.killed = true;
            }
        std::this_thread::sleep_for(std::chrono::milliseconds(5));
    }
    return 0;
}

int main(int argc, char **argv) {
    Command cmd(argc, argv);
    const std::string qpath = cmd.getQueryGraphPath();
    const std::string dpath = cmd.getDataGraphPath();
    Graph g;
    const std::string binOut = option_after(argc, argv, "-b");
    if (!binOut.empty()) {
        g.loadGraphFromTextFile(dpath);
        std::ofstream os(binOut, std::ios::binary);
        g.writeToStream(os);
        return 0;
    }
    const std::string list = option_after(argc, argv, "-Q");
    g.loadGraphFromTextFile(dpath);
    if (!list.empty()) return run_list(argc, argv, cmd, g, list);
    return run_query(argc, argv, cmd, qpath, g);
}
