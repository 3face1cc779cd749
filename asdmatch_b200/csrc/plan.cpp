// Host planner: chooses the matching order the enumeration kernels follow.
//
// The reference plans with a fractional hypertree decomposition, a sampling
// cardinality estimator and a cost-based DP over bag permutations
// (plan/optimizer.cpp:380-548, plan/estimator.cpp:173-291).  Plans change the
// amount of work, never the count.  This planner uses the candidate space the
// device already built: for a directed query edge e = (u -> u2) the average
// list length a(e) = |candidate edges of e| / |C(u)| estimates how many u2
// candidates extend one u candidate, and a(e)/|C(u2)| is the chance that a
// given u2 candidate survives the extra intersection with e's list.  For every
// start vertex it grows a connected order greedily by the smallest estimated
// number of partial matches, and keeps the order with the smallest total
// estimated work (partial matches expanded + 32-wide list chunks scanned).
#include <algorithm>
#include <cmath>
#include <functional>
#include <memory>
#include <unordered_map>
#include <unordered_set>

#include "cs.cuh"

double card_lookup_or(const asdm_card *c, uint64_t subset, double fallback);

namespace asdm {

namespace {

double avg_len(const asdm_cs &cs, uint32_t from, uint32_t to) {
    const int k = cs.q.slot(from, to);
    const uint32_t e = cs.q.off[from] + (uint32_t)k;
    return cs.ncand[from] ? (double)cs.etotal[e] / (double)cs.ncand[from] : 0.0;
}

}  // namespace

// One step of the greedy order search: every vertex u adjacent to the prefix
// with the model's estimate of the extended prefix's cardinality.
void greedy_candidates(const asdm_cs &cs, const GreedyState &st, std::vector<GreedyCand> &out) {
    const QueryGraph &q = cs.q;
    out.clear();
    std::vector<double> lens;
    for (uint32_t u = 0; u < q.n; ++u) {
        if (st.in[u]) continue;
        double drv = INFINITY;
        lens.clear();
        for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
            const uint32_t j = q.nbr[e];
            if (!st.in[j]) continue;
            const double a = avg_len(cs, j, u);
            lens.push_back(a);
            drv = std::min(drv, a);
        }
        if (lens.empty()) continue;
        double factor = drv;
        bool skipped = false;
        for (double a : lens) {
            if (!skipped && a == drv) { skipped = true; continue; }
            factor *= std::min(1.0, a / std::max(1.0, (double)cs.ncand[u]));
        }
        GreedyCand c;
        c.u = u;
        c.Nu = st.N * factor;
        c.work = st.N * (1.0 + lens.size() * std::ceil(std::max(drv, 1.0) / 32.0));
        c.B = (uint32_t)lens.size();
        out.push_back(c);
    }
}

void greedy_start(const asdm_cs &cs, uint32_t start, GreedyState &st) {
    st.in.assign(cs.q.n, 0);
    st.order.assign(1, start);
    st.in[start] = 1;
    st.mask = 1ull << start;
    st.N = (double)cs.ncand[start];
    st.cost = 0.0;
}

// Takes the candidate with the smallest estimate (more backward edges on a
// tie); false when the prefix cannot grow (the query is disconnected).
bool greedy_take(const asdm_cs &cs, GreedyState &st, const std::vector<GreedyCand> &cands) {
    const GreedyCand *best = nullptr;
    for (const GreedyCand &c : cands)
        if (!best || c.Nu < best->Nu || (c.Nu == best->Nu && c.B > best->B)) best = &c;
    if (!best) {
        st.cost = INFINITY;
        return false;
    }
    st.order.push_back(best->u);
    st.in[best->u] = 1;
    st.mask |= 1ull << best->u;
    st.cost += best->work + (st.order.size() < cs.q.n ? best->Nu : 0.0);
    st.N = std::max(best->Nu, 1e-9);
    return true;
}

namespace {

// With a cardinality cache (`.card`), a prefix whose vertex set is in the
// cache uses the cached cardinality instead of the model's estimate.
void greedy_from(const asdm_cs &cs, const asdm_card *card, uint32_t start, std::vector<uint32_t> &order,
                 double &cost) {
    GreedyState st;
    greedy_start(cs, start, st);
    st.N = card_lookup_or(card, st.mask, st.N);
    std::vector<GreedyCand> cands;
    for (uint32_t k = 1; k < cs.q.n; ++k) {
        greedy_candidates(cs, st, cands);
        for (GreedyCand &c : cands) c.Nu = card_lookup_or(card, st.mask | (1ull << c.u), c.Nu);
        if (!greedy_take(cs, st, cands)) break;
    }
    order = st.order;
    cost = st.cost;
}

}  // namespace

// ---------------------------------------------------------------------------
// Exhaustive order search over connected prefixes (dynamic programming over
// vertex subsets, as the reference's optimalPlanDP does over bag subsets,
// plan/subset_structure.cpp:146-233).  The cost of appending u to a prefix P
// (|P| = l levels, N(P) partial matches, B backward edges whose shortest
// average candidate list holds `drv` entries) follows what the enumeration
// kernel does per partial match of P:
//   inner level:  N(P) * (kOpen + drv * (1 + (B - 1) * kProbe))
//   last level:   N(P) * kLeafOne               when B == 1 (the list length is the count)
//                 N(P) * (kOpen + drv * (1 + (B - 1) * kProbe))   otherwise
// N(S) is exact for one and two vertices (|C(u)|, the candidate-edge total),
// the caller's figure where it has one (a .card entry, a learned estimate),
// else the smallest over last vertices u of N(S - u) times the greedy's
// extension factor.
// When levels n-2 and n-1 each have one backward edge, the enumeration
// counts both in closed form per level-(n-3) partial match (COUNT mode):
//   last two steps:  N(P) * kTail
// Since the vertex left after a prefix of n-1 vertices is fixed, the last
// step is folded into the cost of that prefix.
namespace {
constexpr double kOpen = 4.0;     // opening a level for one partial match (list offsets, driver choice)
constexpr double kProbe = 2.0;    // galloping into one more list, per driver entry
constexpr double kLeafOne = 1.0;  // a one-list last level
constexpr double kTail = 1.0;     // the closed form of the last two levels, per level-(n-3) partial match
}  // namespace

bool connected_subsets(const QueryGraph &q, uint32_t max_size, size_t limit, std::vector<uint64_t> &out) {
    std::vector<uint64_t> nb(q.n, 0);
    for (uint32_t u = 0; u < q.n; ++u)
        for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) nb[u] |= 1ull << q.nbr[e];
    out.clear();
    std::vector<uint64_t> level;
    for (uint32_t u = 0; u < q.n; ++u) level.push_back(1ull << u);
    for (uint32_t k = 1; !level.empty(); ++k) {
        out.insert(out.end(), level.begin(), level.end());
        if (out.size() > limit) return false;
        if (k == max_size) break;
        std::unordered_set<uint64_t> next;
        for (uint64_t S : level) {
            uint64_t ext = 0;
            for (uint64_t r = S; r; r &= r - 1) ext |= nb[__builtin_ctzll(r)];
            ext &= ~S;
            for (; ext; ext &= ext - 1) {
                next.insert(S | (ext & -ext));
                if (out.size() + next.size() > limit) return false;
            }
        }
        level.assign(next.begin(), next.end());
        std::sort(level.begin(), level.end());
    }
    return true;
}

bool plan_dp(const asdm_cs &cs, const std::function<bool(uint64_t, double &)> &known, std::vector<uint32_t> &order,
             double &cost) {
    const QueryGraph &q = cs.q;
    const uint32_t n = q.n;
    if (n > kDpMaxVertices) return false;
    std::vector<uint64_t> subsets;
    if (!connected_subsets(q, n, kDpMaxSubsets, subsets)) return false;
    const uint64_t full = n == 64 ? ~0ull : (1ull << n) - 1;
    if (subsets.empty() || subsets.back() != full) return false;  // disconnected
    std::vector<uint64_t> nb(n, 0);
    for (uint32_t u = 0; u < n; ++u)
        for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) nb[u] |= 1ull << q.nbr[e];
    struct Entry { double N, f; int last; };
    std::unordered_map<uint64_t, Entry> T;
    T.reserve(subsets.size() * 2);
    for (uint64_t S : subsets) {
        const uint32_t k = (uint32_t)__builtin_popcountll(S);
        Entry E{INFINITY, INFINITY, -1};
        if (k == 1) {
            E.N = (double)cs.ncand[__builtin_ctzll(S)];
            E.f = 0.0;
            E.last = (int)__builtin_ctzll(S);
            double c;
            if (known(S, c)) E.N = c;
            T.emplace(S, E);
            continue;
        }
        double derived = INFINITY;
        for (uint64_t r = S; r; r &= r - 1) {
            const uint32_t u = __builtin_ctzll(r);
            const uint64_t P = S & ~(1ull << u);
            if (!(nb[u] & P)) continue;
            auto it = T.find(P);
            if (it == T.end()) continue;  // P not connected
            const Entry &EP = it->second;
            // backward edges of u into P
            double drv = INFINITY, lens[64];
            uint32_t B = 0;
            for (uint64_t b = nb[u] & P; b; b &= b - 1) {
                const double a = avg_len(cs, __builtin_ctzll(b), u);
                lens[B++] = a;
                drv = std::min(drv, a);
            }
            double factor = drv;
            bool skipped = false;
            for (uint32_t i = 0; i < B; ++i) {
                if (!skipped && lens[i] == drv) { skipped = true; continue; }
                factor *= std::min(1.0, lens[i] / std::max(1.0, (double)cs.ncand[u]));
            }
            derived = std::min(derived, EP.N * factor);
            double step = (k == n && B == 1) ? EP.N * kLeafOne : EP.N * (kOpen + drv * (1.0 + (B - 1) * kProbe));
            if (k == n) {
                step = 0.0;  // charged with the prefix of n-1 vertices
            } else if (n >= 3 && k + 1 == n) {
                // u is level n-2; z, the remaining vertex, is the last level
                const uint32_t z = __builtin_ctzll(full & ~S);
                const uint64_t zb = nb[z] & S;
                const uint32_t Bz = (uint32_t)__builtin_popcountll(zb);
                if (B == 1 && Bz == 1) {
                    step = EP.N * kTail;
                } else {
                    double dz = INFINITY;
                    for (uint64_t b = zb; b; b &= b - 1) dz = std::min(dz, avg_len(cs, __builtin_ctzll(b), z));
                    const double Ns = std::max(EP.N * factor, 1e-9);
                    step += Ns * (Bz == 1 ? kLeafOne : kOpen + dz * (1.0 + (Bz - 1) * kProbe));
                }
            }
            if (EP.f + step < E.f) {
                E.f = EP.f + step;
                E.last = (int)u;
            }
        }
        if (k == 2) {
            const uint32_t a = __builtin_ctzll(S), b = __builtin_ctzll(S & (S - 1));
            E.N = (double)cs.etotal[q.off[a] + (uint32_t)q.slot(a, b)];
        } else {
            E.N = derived;
        }
        double c;
        if (known(S, c)) E.N = c;
        E.N = std::max(E.N, 1e-9);
        T.emplace(S, E);
    }
    order.assign(n, 0);
    uint64_t S = full;
    for (uint32_t k = n; k > 0; --k) {
        const Entry &E = T.at(S);
        order[k - 1] = (uint32_t)E.last;
        S &= ~(1ull << E.last);
    }
    cost = T.at(full).f;
    return true;
}

int build_plan(const asdm_cs &cs, const uint32_t *user_order, asdm_plan &p, const asdm_card *card) {
    const QueryGraph &q = cs.q;
    const uint32_t n = q.n;
    if (!cs.nonempty) return fail(ASDM_ERR_INVALID, "cannot plan over an empty candidate space");
    if (user_order) {
        std::vector<uint32_t> given(user_order, user_order + n);
        std::vector<char> seen(n, 0);
        for (uint32_t k = 0; k < n; ++k) {
            if (given[k] >= n || seen[given[k]]) return fail(ASDM_ERR_INVALID, "order is not a permutation");
            seen[given[k]] = 1;
        }
        // An order whose vertex has no earlier neighbour is the reference's
        // Cartesian attribute (cartesianParent, plan/decomposition.cpp:7-88,
        // enumerated by optimizedCartesianProduct, plan/estimator.cpp:41-171).
        // Counts do not depend on the order, so such a vertex is deferred to
        // the first position where an earlier neighbour exists: the order
        // stays the caller's wherever it is connected.
        p.order.clear();
        std::vector<char> in(n, 0), taken(n, 0);
        while (p.order.size() < n) {
            bool placed = false;
            for (uint32_t k = 0; k < n && !placed; ++k) {
                const uint32_t u = given[k];
                if (taken[k]) continue;
                bool linked = p.order.empty();
                for (uint32_t e = q.off[u]; e < q.off[u + 1] && !linked; ++e) linked = in[q.nbr[e]] != 0;
                if (!linked) continue;
                p.order.push_back(u);
                in[u] = 1;
                taken[k] = 1;
                placed = true;
            }
            if (!placed) return fail(ASDM_ERR_INVALID, "query is not connected");
        }
        p.cost = 0;
    } else if (cs.g->tuning.planner == ASDM_PLANNER_DP &&
               plan_dp(cs, [&](uint64_t S, double &c) {
                   c = card_lookup_or(card, S, NAN);
                   return !std::isnan(c);
               }, p.order, p.cost)) {
        // exhaustive search over connected prefixes
    } else {
        double best = INFINITY;
        for (uint32_t s = 0; s < n; ++s) {
            std::vector<uint32_t> o;
            double c;
            greedy_from(cs, card, s, o, c);
            if (o.size() == n && c < best) {
                best = c;
                p.order = o;
            }
        }
        if (p.order.size() != n) return fail(ASDM_ERR_INVALID, "query is not connected");
        p.cost = best;
    }
    std::vector<uint32_t> level(n, 0);
    for (uint32_t k = 0; k < n; ++k) level[p.order[k]] = k;
    p.back.assign(n, {});
    p.conf.assign(n, {});
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t u = p.order[k];
        for (uint32_t j = 0; j < k; ++j) {
            const uint32_t w = p.order[j];
            const int slot = q.slot(w, u);
            if (slot >= 0) p.back[k].push_back({j, q.off[w] + (uint32_t)slot});
            else if (q.lab[w] == q.lab[u]) p.conf[k].push_back(j);
        }
        if (k > 0 && p.back[k].empty()) return fail(ASDM_ERR_INVALID, "order is not connected at level %u", k);
    }
    return ASDM_OK;
}

// A plan over the first `depth` levels only: `order` lists distinct query
// vertices, each after the first adjacent to an earlier one.  Enumerating it
// counts the partial matches of the sub-query these vertices induce inside the
// candidate space, which is what the reference's estimator approximates by
// sampling (cardEstimateLabeled, plan/estimator.cpp:173-291).
int build_prefix_plan(const asdm_cs &cs, const uint32_t *order, uint32_t depth, asdm_plan &p) {
    const QueryGraph &q = cs.q;
    const uint32_t n = q.n;
    if (depth == 0 || depth > n) return fail(ASDM_ERR_INVALID, "prefix depth %u outside 1..%u", depth, n);
    p.order.assign(order, order + depth);
    std::vector<char> seen(n, 0);
    for (uint32_t k = 0; k < depth; ++k) {
        if (p.order[k] >= n || seen[p.order[k]]) return fail(ASDM_ERR_INVALID, "prefix repeats or leaves the query");
        seen[p.order[k]] = 1;
    }
    p.cost = 0;
    p.back.assign(depth, {});
    p.conf.assign(depth, {});
    for (uint32_t k = 0; k < depth; ++k) {
        const uint32_t u = p.order[k];
        for (uint32_t j = 0; j < k; ++j) {
            const uint32_t w = p.order[j];
            const int slot = q.slot(w, u);
            if (slot >= 0) p.back[k].push_back({j, q.off[w] + (uint32_t)slot});
            else if (q.lab[w] == q.lab[u]) p.conf[k].push_back(j);
        }
        if (k > 0 && p.back[k].empty()) return fail(ASDM_ERR_INVALID, "prefix is not connected at level %u", k);
    }
    return ASDM_OK;
}

}  // namespace asdm

using namespace asdm;

extern "C" int asdm_plan_create(const asdm_cs *cs, const uint32_t *order, asdm_plan **out) {
    clear_error();
    if (!cs || !out) return fail(ASDM_ERR_INVALID, "null argument");
    auto p = std::make_unique<asdm_plan>();
    ASDM_TRY(build_plan(*cs, order, *p, nullptr));
    *out = p.release();
    return ASDM_OK;
}

extern "C" int asdm_plan_create_card(const asdm_cs *cs, const asdm_card *card, asdm_plan **out) {
    clear_error();
    if (!cs || !out) return fail(ASDM_ERR_INVALID, "null argument");
    auto p = std::make_unique<asdm_plan>();
    ASDM_TRY(build_plan(*cs, nullptr, *p, card));
    *out = p.release();
    return ASDM_OK;
}

extern "C" int asdm_plan_order(const asdm_plan *p, uint32_t *order) {
    if (!p || !order) return fail(ASDM_ERR_INVALID, "null argument");
    std::copy(p->order.begin(), p->order.end(), order);
    return ASDM_OK;
}

extern "C" int asdm_plan_cost(const asdm_plan *p, double *cost) {
    if (!p || !cost) return fail(ASDM_ERR_INVALID, "null argument");
    *cost = p->cost;
    return ASDM_OK;
}

extern "C" int asdm_plan_free(asdm_plan *p) {
    delete p;
    return ASDM_OK;
}
