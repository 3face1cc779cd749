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
#include <memory>

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

int build_plan(const asdm_cs &cs, const uint32_t *user_order, asdm_plan &p, const asdm_card *card) {
    const QueryGraph &q = cs.q;
    const uint32_t n = q.n;
    if (!cs.nonempty) return fail(ASDM_ERR_INVALID, "cannot plan over an empty candidate space");
    if (user_order) {
        p.order.assign(user_order, user_order + n);
        std::vector<char> seen(n, 0);
        for (uint32_t k = 0; k < n; ++k) {
            if (p.order[k] >= n || seen[p.order[k]]) return fail(ASDM_ERR_INVALID, "order is not a permutation");
            seen[p.order[k]] = 1;
        }
        p.cost = 0;
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

extern "C" int asdm_plan_free(asdm_plan *p) {
    delete p;
    return ASDM_OK;
}
