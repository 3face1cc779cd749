// Internal declarations shared by the host and device halves of libasdm_b200.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <string>
#include <vector>

#include "asdm.h"

struct asdm_host_graph {
    uint32_t n = 0;
    uint64_t m2 = 0;          // directed edge count (2 x undirected)
    uint32_t nlabels = 0;     // max label + 1
    std::vector<uint32_t> off;  // n + 1 (EdgeID is uint32 in the reference)
    std::vector<uint32_t> nbr;  // m2, sorted by (label, id) per vertex
    std::vector<uint32_t> lab;  // n

    uint32_t deg(uint32_t v) const { return off[v + 1] - off[v]; }
    bool adjacent(uint32_t a, uint32_t b) const;
};

namespace asdm {

// Thread-local error message; returns `code` so callers can `return fail(...)`.
int fail(int code, const char *fmt, ...);
void clear_error();

// Builds the loader layout (label,id-sorted CSR) from an edge list.  Returns
// ASDM_ERR_INVALID on self loops, duplicates or out-of-range ids.
int build_csr(uint32_t n, const uint32_t *labels, uint64_t m, const uint32_t *edges, asdm_host_graph &g);

// Deterministic RNG (splitmix64-seeded xoshiro256**).
struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed);
    uint64_t next();
    double uniform();                  // [0, 1)
    uint64_t below(uint64_t bound);    // [0, bound)
};

// Query-side helpers shared by the candidate space and the planner.
struct QueryGraph {
    uint32_t n = 0;
    std::vector<uint32_t> off, nbr, lab;
    uint32_t deg(uint32_t u) const { return off[u + 1] - off[u]; }
    int slot(uint32_t u, uint32_t w) const {  // position of w in u's neighbour list, -1 if absent
        for (uint32_t e = off[u]; e < off[u + 1]; ++e)
            if (nbr[e] == w) return (int)(e - off[u]);
        return -1;
    }
};
int make_query(const uint32_t *q_offsets, const uint32_t *q_nbrs, const uint32_t *q_labels, uint32_t q_n,
               QueryGraph &q);

constexpr uint32_t kMaxQuery = 32;       // MAX_PATTERN_SIZE (config/config.h:31)
constexpr uint32_t kNone = 0xFFFFFFFFu;

}  // namespace asdm
