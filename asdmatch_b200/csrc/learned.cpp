// Learned cardinalities for the planner.
//
// The reference estimates the cardinality of every query-vertex subset it
// plans over by sampling partial matches inside the candidate space
// (cardEstimateLabeled, plan/estimator.cpp:173-291) and stores the results in
// subsetToCard (plan/estimator.cpp:7), which optimalPlanDP reads
// (plan/subset_structure.cpp:146-233).  Here a message-passing network (the
// asdm_estimator, trained on exact partial-match counts that the engine
// produces with asdm_prefix_counts) predicts log(1 + cardinality) of a
// subset's induced sub-query from per-vertex features of the candidate
// space, and the planner's greedy order search asks it about every prefix of
// 3..max_subset vertices.  Prefixes of 1 and 2 vertices stay exact (|C(u)| and
// the candidate-edge total), as smallCard keeps them exact in the reference
// (plan/subset_structure.cpp:97-114).  Plans change; counts never do.
#include <algorithm>
#include <cmath>
#include <memory>
#include <unordered_map>

#include "cs.cuh"

namespace asdm {

int build_plan(const asdm_cs &cs, const uint32_t *user_order, asdm_plan &p, const asdm_card *card = nullptr);
int sample_subsets(asdm_cs &cs, const std::vector<uint64_t> &subsets, uint32_t walks, uint64_t seed,
                   std::vector<double> &est);

namespace {

// Walks per subset when the sampling estimator stands in for a dropped prediction.
constexpr uint32_t kFallbackWalks = 256;

constexpr uint32_t kF = ASDM_EST_FEATURES;
constexpr uint32_t kLabelBuckets = 32;

struct FeatBatch {
    std::vector<float> x;
    std::vector<uint32_t> adj_off{0};
    std::vector<uint32_t> adj;
    std::vector<uint32_t> gid;
};

double edge_avg(const asdm_cs &cs, uint32_t u, uint32_t w) {
    const int k = cs.q.slot(u, w);
    const uint32_t e = cs.q.off[u] + (uint32_t)k;
    return (double)cs.etotal[e] / std::max(1.0, (double)cs.ncand[u]);
}

// Node features of the sub-query induced by `mask` (vertices ascending):
//   [0, 32)  label one-hot (label mod 32)
//   32  log(1+|C(u)|)/16           33  degree inside the subset / 8
//   34  degree in the query / 16
//   35-37  sum / min / max over subset neighbours w of log(1+a(u->w))/16,
//          a(u->w) = candidate edges of (u,w) / |C(u)|
//   38  sum over subset neighbours of log rho(u,w) / 16, rho = a(u->w)/|C(w)|
//   39  (log|C(u)| + sum/2) / 16: summed over the subset, the log of the
//       independence estimate prod |C(u)| * prod_edges rho, over 16
//   40  1                               41  subset size / 16
//   42  cycle rank of the subset / 8    43  other subset vertices with u's label / 8
void subset_features(const asdm_cs &cs, uint64_t mask, uint32_t graph, FeatBatch &b) {
    const QueryGraph &q = cs.q;
    uint32_t verts[64], local[64];
    uint32_t k = 0;
    for (uint32_t u = 0; u < q.n; ++u)
        if (mask >> u & 1ull) {
            local[u] = k;
            verts[k++] = u;
        }
    uint32_t m = 0;
    for (uint32_t i = 0; i < k; ++i)
        for (uint32_t e = q.off[verts[i]]; e < q.off[verts[i] + 1]; ++e)
            if (mask >> q.nbr[e] & 1ull) ++m;
    m /= 2;
    const float cycle = (float)((int)m - (int)k + 1) / 8.f;
    const uint32_t node0 = (uint32_t)b.gid.size();
    const size_t base = b.x.size();
    b.x.resize(base + (size_t)k * kF, 0.f);
    for (uint32_t i = 0; i < k; ++i) {
        const uint32_t u = verts[i];
        float *f = &b.x[base + (size_t)i * kF];
        f[q.lab[u] % kLabelBuckets] = 1.f;
        const double cu = (double)cs.ncand[u];
        f[32] = (float)(std::log1p(cu) / 16.0);
        uint32_t ds = 0, same = 0;
        double sa = 0, mina = 0, maxa = 0, sr = 0;
        for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
            const uint32_t w = q.nbr[e];
            if (!(mask >> w & 1ull)) continue;
            const double a = edge_avg(cs, u, w);
            const double la = std::log1p(a);
            const double rho = a / std::max(1.0, (double)cs.ncand[w]);
            sa += la;
            mina = ds ? std::min(mina, la) : la;
            maxa = ds ? std::max(maxa, la) : la;
            sr += std::log(std::max(rho, 1e-12));
            ++ds;
            b.adj.push_back(node0 + local[w]);
        }
        for (uint32_t j = 0; j < k; ++j)
            if (j != i && q.lab[verts[j]] == q.lab[u]) ++same;
        f[33] = ds / 8.f;
        f[34] = q.deg(u) / 16.f;
        f[35] = (float)(sa / 16.0);
        f[36] = (float)(mina / 16.0);
        f[37] = (float)(maxa / 16.0);
        f[38] = (float)(sr / 16.0);
        f[39] = (float)((std::log(std::max(cu, 1.0)) + 0.5 * sr) / 16.0);
        f[40] = 1.f;
        f[41] = k / 16.f;
        f[42] = cycle;
        f[43] = same / 8.f;
        b.adj_off.push_back((uint32_t)b.adj.size());
    }
    b.gid.insert(b.gid.end(), k, graph);
}

// Learned log(1 + cardinality) -> cardinality.
double from_log(float y) { return std::expm1((double)std::min(std::max(y, 0.f), 60.f)); }

// A subset has at most prod |C(u)| partial matches.
bool in_range(const asdm_cs &cs, uint64_t mask, double card) {
    if (!std::isfinite(card) || card < 0) return false;
    double log_bound = 0;
    for (uint64_t r = mask; r; r &= r - 1) log_bound += std::log(std::max(1.0, (double)cs.ncand[__builtin_ctzll(r)]));
    return std::log1p(card) <= log_bound + 1e-9;
}

// Predictions for a list of (query, subset) requests, in chunks that bound
// the estimator's device workspace.
int predict(asdm_estimator *e, const std::vector<const asdm_cs *> &qs, const std::vector<uint64_t> &masks,
            std::vector<double> &out) {
    constexpr size_t kChunk = 1u << 17;
    out.assign(masks.size(), 0.0);
    std::vector<float> y;
    for (size_t at = 0; at < masks.size(); at += kChunk) {
        const size_t end = std::min(masks.size(), at + kChunk);
        FeatBatch b;
        for (size_t r = at; r < end; ++r) subset_features(*qs[r], masks[r], (uint32_t)(r - at), b);
        y.assign(end - at, 0.f);
        ASDM_TRY(asdm_est_predict(e, (int)b.gid.size(), (int)(end - at), b.x.data(), b.adj_off.data(),
                                  b.adj.empty() ? nullptr : b.adj.data(), b.gid.data(), y.data()));
        for (size_t r = at; r < end; ++r) out[r] = from_log(y[r - at]);
    }
    return ASDM_OK;
}

}  // namespace

namespace {

// Greedy order search for every start of every query, in lockstep; learned
// estimates for prefixes of 3..kmax vertices.
int greedy_batch_learned(const std::vector<asdm_cs *> &css, asdm_estimator *e, uint32_t kmax,
                         std::vector<asdm_plan> &plans) {
    struct Search {
        uint32_t query;
        GreedyState st;
        std::vector<GreedyCand> cands;
        std::vector<int64_t> req;  // request index per candidate, -1 = model estimate
        bool alive = true;
    };
    std::vector<Search> ss;
    uint32_t maxn = 0;
    for (uint32_t i = 0; i < css.size(); ++i) {
        const asdm_cs &cs = *css[i];
        if (!cs.nonempty) continue;
        maxn = std::max(maxn, cs.q.n);
        for (uint32_t s = 0; s < cs.q.n; ++s) {
            Search x;
            x.query = i;
            greedy_start(cs, s, x.st);
            ss.push_back(std::move(x));
        }
    }
    std::vector<std::unordered_map<uint64_t, uint32_t>> seen(css.size());
    std::vector<const asdm_cs *> rq;
    std::vector<uint64_t> rm;
    std::vector<double> est;
    for (uint32_t k = 1; k < maxn; ++k) {
        rq.clear();
        rm.clear();
        for (auto &m : seen) m.clear();
        for (Search &x : ss) {
            const asdm_cs &cs = *css[x.query];
            if (!x.alive || k >= cs.q.n) continue;
            greedy_candidates(cs, x.st, x.cands);
            x.req.assign(x.cands.size(), -1);
            if (k + 1 < 3 || k + 1 > kmax) continue;
            for (size_t c = 0; c < x.cands.size(); ++c) {
                const uint64_t mk = x.st.mask | (1ull << x.cands[c].u);
                auto it = seen[x.query].find(mk);
                if (it == seen[x.query].end()) {
                    it = seen[x.query].emplace(mk, (uint32_t)rm.size()).first;
                    rq.push_back(&cs);
                    rm.push_back(mk);
                }
                x.req[c] = it->second;
            }
        }
        if (!rm.empty()) ASDM_TRY(predict(e, rq, rm, est));
        for (Search &x : ss) {
            const asdm_cs &cs = *css[x.query];
            if (!x.alive || k >= cs.q.n) continue;
            for (size_t c = 0; c < x.cands.size(); ++c)
                if (x.req[c] >= 0 && in_range(cs, x.st.mask | (1ull << x.cands[c].u), est[(size_t)x.req[c]]))
                    x.cands[c].Nu = est[(size_t)x.req[c]];
            x.alive = greedy_take(cs, x.st, x.cands);
        }
    }
    plans.assign(css.size(), asdm_plan{});
    std::vector<double> best(css.size(), INFINITY);
    std::vector<const Search *> pick(css.size(), nullptr);
    for (const Search &x : ss) {
        const asdm_cs &cs = *css[x.query];
        if (x.st.order.size() == cs.q.n && x.st.cost < best[x.query]) {
            best[x.query] = x.st.cost;
            pick[x.query] = &x;
        }
    }
    for (uint32_t i = 0; i < css.size(); ++i) {
        if (!css[i]->nonempty) continue;
        if (!pick[i]) continue;  // not connected: the plan stays empty
        ASDM_TRY(build_plan(*css[i], pick[i]->st.order.data(), plans[i]));
        plans[i].cost = best[i];
    }
    return ASDM_OK;
}

}  // namespace

// Learned plans for a group of queries: the exhaustive prefix search where a
// query is small enough (every connected subset of 3..kmax vertices
// estimated in one forward pass for the whole group), the lockstep greedy
// search for the rest.
int plan_batch_learned(const std::vector<asdm_cs *> &css, asdm_estimator *e, uint32_t kmax,
                       std::vector<asdm_plan> &plans) {
    if (kmax == 0) kmax = 6;
    plans.assign(css.size(), asdm_plan{});
    std::vector<uint32_t> dp_ids;
    std::vector<asdm_cs *> rest;
    std::vector<uint32_t> rest_ids;
    std::vector<const asdm_cs *> rq;
    std::vector<uint64_t> rm;
    std::vector<std::pair<size_t, size_t>> range(css.size(), {0, 0});  // requests of query i
    std::vector<uint64_t> subsets;
    for (uint32_t i = 0; i < css.size(); ++i) {
        const asdm_cs &cs = *css[i];
        if (!cs.nonempty) continue;
        const bool dp = cs.g->tuning.planner == ASDM_PLANNER_DP && cs.q.n <= kDpMaxVertices &&
                        connected_subsets(cs.q, cs.q.n, kDpMaxSubsets, subsets);
        if (!dp) {
            rest.push_back(css[i]);
            rest_ids.push_back(i);
            continue;
        }
        dp_ids.push_back(i);
        range[i].first = rm.size();
        for (uint64_t S : subsets) {
            const uint32_t k = (uint32_t)__builtin_popcountll(S);
            if (k >= 3 && k <= kmax) {
                rq.push_back(&cs);
                rm.push_back(S);
            }
        }
        range[i].second = rm.size();
    }
    std::vector<double> est;
    if (!rm.empty()) ASDM_TRY(predict(e, rq, rm, est));
    for (uint32_t i : dp_ids) {
        // a prediction outside the possible range (more partial matches than
        // the product of the subset's candidate-set sizes, or not finite) is
        // dropped: the sampling estimator's estimate stands in for it
        std::unordered_map<uint64_t, double> known;
        std::vector<uint64_t> dropped;
        for (size_t r = range[i].first; r < range[i].second; ++r) {
            if (in_range(*css[i], rm[r], est[r])) known.emplace(rm[r], est[r]);
            else dropped.push_back(rm[r]);
        }
        if (!dropped.empty()) {
            std::vector<double> sampled;
            ASDM_TRY(sample_subsets(*css[i], dropped, kFallbackWalks, i, sampled));
            for (size_t k = 0; k < dropped.size(); ++k) known.emplace(dropped[k], sampled[k]);
        }
        std::vector<uint32_t> order;
        double cost = 0;
        const bool ok = plan_dp(*css[i], [&](uint64_t S, double &c) {
            auto it = known.find(S);
            if (it == known.end()) return false;
            c = it->second;
            return true;
        }, order, cost);
        if (!ok) {  // not connected: the plan stays empty
            continue;
        }
        ASDM_TRY(build_plan(*css[i], order.data(), plans[i]));
        plans[i].cost = cost;
    }
    if (!rest.empty()) {
        std::vector<asdm_plan> rp;
        ASDM_TRY(greedy_batch_learned(rest, e, kmax, rp));
        for (size_t k = 0; k < rest.size(); ++k) plans[rest_ids[k]] = std::move(rp[k]);
    }
    return ASDM_OK;
}

}  // namespace asdm

using namespace asdm;

extern "C" int asdm_est_features(const asdm_cs *cs, uint32_t nsub, const uint64_t *masks, float *x, uint32_t *adj_off,
                                 uint32_t *adj, uint64_t adj_capacity, uint32_t *node_graph, uint64_t *n_nodes,
                                 uint64_t *n_adj) {
    clear_error();
    if (!cs || (nsub && !masks)) return fail(ASDM_ERR_INVALID, "null argument");
    if (!cs->nonempty) return fail(ASDM_ERR_INVALID, "empty candidate space");
    const uint64_t all = cs->q.n >= 64 ? ~0ull : ((1ull << cs->q.n) - 1);
    FeatBatch b;
    for (uint32_t i = 0; i < nsub; ++i) {
        if (masks[i] == 0 || (masks[i] & ~all)) return fail(ASDM_ERR_INVALID, "subset %u is empty or leaves the query", i);
        subset_features(*cs, masks[i], i, b);
    }
    if (n_nodes) *n_nodes = b.gid.size();
    if (n_adj) *n_adj = b.adj.size();
    if (!x && !adj_off && !adj && !node_graph) return ASDM_OK;
    if (!x || !adj_off || !node_graph || (b.adj.size() && !adj)) return fail(ASDM_ERR_INVALID, "null output");
    if (b.adj.size() > adj_capacity) return fail(ASDM_ERR_CAPACITY, "%zu adjacency entries", b.adj.size());
    std::copy(b.x.begin(), b.x.end(), x);
    std::copy(b.adj_off.begin(), b.adj_off.end(), adj_off);
    std::copy(b.adj.begin(), b.adj.end(), adj);
    std::copy(b.gid.begin(), b.gid.end(), node_graph);
    return ASDM_OK;
}

extern "C" int asdm_plan_create_learned(uint32_t nq, asdm_cs *const *cs, asdm_estimator *e, uint32_t max_subset,
                                        asdm_plan **plans) {
    clear_error();
    if (nq && (!cs || !e || !plans)) return fail(ASDM_ERR_INVALID, "null argument");
    std::vector<asdm_cs *> css(cs, cs + nq);
    for (uint32_t i = 0; i < nq; ++i) {
        plans[i] = nullptr;
        if (!css[i]) return fail(ASDM_ERR_INVALID, "query %u has no candidate space", i);
        if (!css[i]->nonempty) return fail(ASDM_ERR_INVALID, "cannot plan over an empty candidate space");
    }
    std::vector<asdm_plan> out;
    ASDM_TRY(plan_batch_learned(css, e, max_subset, out));
    for (uint32_t i = 0; i < nq; ++i)
        if (out[i].order.size() != css[i]->q.n) return fail(ASDM_ERR_INVALID, "query %u is not connected", i);
    for (uint32_t i = 0; i < nq; ++i) plans[i] = new asdm_plan(std::move(out[i]));
    return ASDM_OK;
}
