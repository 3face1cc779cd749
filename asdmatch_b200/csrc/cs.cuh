// Candidate space of one query on the device (the product of K1-K3).
#pragma once

#include <functional>
#include <memory>

#include "device.cuh"

// Device arrays of the candidate spaces built together in one group; every
// asdm_cs of the group holds a reference, the last one frees them.
struct CsArena {
    cudaStream_t stream = nullptr;
    uint32_t *d_cand = nullptr;
    uint32_t *d_eoff = nullptr;
    uint32_t *d_elist = nullptr;
    ~CsArena() {
        asdm::dfree(d_cand, stream);
        asdm::dfree(d_eoff, stream);
        asdm::dfree(d_elist, stream);
    }
};

struct asdm_cs {
    asdm_graph *g = nullptr;
    asdm::QueryGraph q;
    bool nonempty = false;
    uint32_t root = 0;                     // CFL root (selectCFLRoot)
    std::vector<uint32_t> bfs_order;       // CFL BFS order (buildCFLBFSTree)
    std::vector<uint32_t> ncand;           // |C(u)|
    std::vector<uint64_t> cand_base;       // C(u) = d_cand + cand_base[u], sorted vertex ids
    uint32_t *d_cand = nullptr;
    // Directed query edge e = q.off[u] + k (u -> q.nbr[e]): for the i-th
    // candidate of u, the candidates of u2 adjacent to it are
    // d_elist[elist_base[e] + off[i] .. elist_base[e] + off[i+1]) with
    // off = d_eoff + eoff_base[e] (ncand[u] + 1 entries, relative to the edge),
    // stored as ascending indices into C(u2).
    std::vector<uint64_t> eoff_base;
    std::vector<uint64_t> elist_base;
    std::vector<uint64_t> etotal;          // entries per directed edge
    uint32_t *d_eoff = nullptr;
    uint32_t *d_elist = nullptr;
    uint64_t build_bytes = 0;              // algorithmic bytes of K1-K3 (roofline)
    float build_ms = 0.f;                  // device time of K1-K3
    uint32_t build_flags = 0;              // ASDM_CS_* bits: which K3 form built the edges, label-run table
    std::shared_ptr<CsArena> arena;        // owns d_cand / d_eoff / d_elist
};

namespace asdm {
// K1-K3 for a group of queries on the same graph (one launch per phase).
int build_batch(const std::vector<asdm_cs *> &group);
}  // namespace asdm

struct asdm_plan {
    std::vector<uint32_t> order;                                   // level -> query vertex
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> back;  // level -> (earlier level j, edge u_j -> u_k)
    std::vector<std::vector<uint32_t>> conf;                       // level -> earlier same-label, non-adjacent levels
    double cost = 0.0;                                             // planner's estimate
};

namespace asdm {
// The planner's greedy order search, in steps, so that a batched caller can
// supply its own cardinalities for the candidates of a step.
struct GreedyState {
    std::vector<uint32_t> order;
    std::vector<char> in;
    uint64_t mask = 0;   // bit u = query vertex u in the prefix
    double N = 0.0;      // estimated partial matches of the prefix
    double cost = 0.0;   // estimated work so far
};
struct GreedyCand {
    uint32_t u;
    double Nu;    // estimated partial matches with u appended
    double work;  // estimated work of the step
    uint32_t B;   // backward edges of u
};
void greedy_start(const asdm_cs &cs, uint32_t start, GreedyState &st);
void greedy_candidates(const asdm_cs &cs, const GreedyState &st, std::vector<GreedyCand> &out);
bool greedy_take(const asdm_cs &cs, GreedyState &st, const std::vector<GreedyCand> &cands);
// Exhaustive search over connected prefixes for queries of at most
// kDpMaxVertices vertices and kDpMaxSubsets connected vertex subsets; false
// when the query is larger (the caller falls back to the greedy search).
// known(S, c) supplies the cardinality of subset S where the caller has one.
constexpr uint32_t kDpMaxVertices = 24;
constexpr size_t kDpMaxSubsets = 1u << 12;
bool connected_subsets(const QueryGraph &q, uint32_t max_size, size_t limit, std::vector<uint64_t> &out);
bool plan_dp(const asdm_cs &cs, const std::function<bool(uint64_t, double &)> &known, std::vector<uint32_t> &order,
             double &cost);
}  // namespace asdm
