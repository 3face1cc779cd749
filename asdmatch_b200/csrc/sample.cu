// Sampling estimates of partial-match counts on the device.
//
// The reference plans with cardEstimateLabeled (plan/estimator.cpp:173-291):
// it walks the candidate space level by level along an order, draws a sample
// of each level's candidates (the intersection of the candidate-edge lists of
// the level's earlier neighbours, LeapfrogJoin), and scales the partial
// counts by (candidates at the level / candidates sampled), so the estimate
// of each prefix's number of partial matches is unbiased.  Here every sample
// is an independent random walk on the device, one warp per walk: at level k
// the warp computes the level's candidate set exactly (shortest list as
// driver, membership in the other lists by binary search, same-label earlier
// vertices excluded), multiplies the walk's weight by its size and moves to
// one member drawn uniformly.  The weight at depth d is an unbiased estimate
// of the number of partial matches of the first d levels (a walk that meets
// an empty set contributes 0 from there on); the estimate is the mean over
// the walks.
//
// asdm_card_sample fills a cardinality cache (asdm_card) with such estimates
// for the connected induced sub-queries of up to max_subset vertices, which
// the card-guided planner (asdm_plan_create_card) uses for its prefixes: the
// plain form's "sampling estimator" planning, and the learned estimator's
// fallback and judge.
#include <algorithm>
#include <cmath>

#include "cs.cuh"

namespace asdm {
namespace {

struct SLevel {
    const uint32_t *cand;   // C(u)
    uint32_t ncand;
    uint32_t nback, back_first;
    uint32_t nconf, conf_first;
    uint32_t pad;
};

struct SBack {
    const uint32_t *off, *list;  // candidate edges (u_j -> u_k), by candidate index of u_j
    uint32_t level, pad;
};

struct SPrefix {
    uint32_t lv_first, depth;
    double *out;  // the prefix's estimate (mean of the walks' weights)
};

__device__ __forceinline__ uint64_t walk_rand(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

constexpr uint32_t kSampleWarps = 8;

// One warp per walk (walk w belongs to prefix w / walks).
__global__ void __launch_bounds__(kSampleWarps * 32)
    sample_walks(const SPrefix *__restrict__ pre, uint64_t nwalks_total, uint32_t walks, const SLevel *__restrict__ lv,
                 const SBack *__restrict__ bk, const uint32_t *__restrict__ conf, uint64_t seed) {
    __shared__ uint32_t s_idx[kSampleWarps][kMaxQuery], s_vid[kSampleWarps][kMaxQuery];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t *idx = s_idx[wid], *vid = s_vid[wid];
    for (uint64_t w = (uint64_t)blockIdx.x * kSampleWarps + wid; w < nwalks_total;
         w += (uint64_t)gridDim.x * kSampleWarps) {
        const SPrefix p = pre[w / walks];
        const SLevel *L = lv + p.lv_first;
        uint64_t rs = walk_rand(seed ^ (w * 0xD1B54A32D192ED03ull));
        double weight = (double)L[0].ncand;
        if (L[0].ncand == 0) weight = 0.0;
        if (lane == 0 && weight > 0.0) {
            const uint32_t x = (uint32_t)(rs % L[0].ncand);
            idx[0] = x;
            vid[0] = L[0].cand[x];
        }
        __syncwarp();
        for (uint32_t k = 1; k < p.depth && weight > 0.0; ++k) {
            const SLevel l = L[k];
            // driver: the shortest list
            uint32_t dlen = 0xFFFFFFFFu, dslot = 0;
            for (uint32_t b = 0; b < l.nback; ++b) {
                const SBack sb = bk[l.back_first + b];
                const uint32_t i = idx[sb.level];
                const uint32_t len = sb.off[i + 1] - sb.off[i];
                if (len < dlen) { dlen = len; dslot = b; }
            }
            const SBack db = bk[l.back_first + dslot];
            const uint32_t *drv = db.list + db.off[idx[db.level]];
            // count the level's candidates, then draw one
            auto member = [&](uint32_t x) {
                bool ok = true;
                for (uint32_t b = 0; b < l.nback && ok; ++b) {
                    if (b == dslot) continue;
                    const SBack sb = bk[l.back_first + b];
                    const uint32_t i = idx[sb.level];
                    const uint32_t s0 = sb.off[i], len = sb.off[i + 1] - s0;
                    const uint32_t q = lower_bound_u32(sb.list + s0, len, x);
                    ok = q < len && sb.list[s0 + q] == x;
                }
                if (ok && l.nconf) {
                    const uint32_t v = l.cand[x];
                    for (uint32_t c = 0; c < l.nconf && ok; ++c) ok = v != vid[conf[l.conf_first + c]];
                }
                return ok;
            };
            uint32_t cnt = 0;
            for (uint32_t i0 = 0; i0 < dlen; i0 += 32) {
                const uint32_t i = i0 + lane;
                cnt += __popc(__ballot_sync(0xffffffffu, i < dlen && member(drv[i])));
            }
            if (cnt == 0) {
                weight = 0.0;
                break;
            }
            weight *= (double)cnt;
            rs = walk_rand(rs);
            uint32_t r = (uint32_t)(rs % cnt), pick = 0;
            for (uint32_t i0 = 0; i0 < dlen; i0 += 32) {
                const uint32_t i = i0 + lane;
                const uint32_t m = __ballot_sync(0xffffffffu, i < dlen && member(drv[i]));
                const uint32_t c = __popc(m);
                if (r < c) {
                    // lane holding the r-th set bit
                    uint32_t mm = m;
                    for (uint32_t t = 0; t < r; ++t) mm &= mm - 1;
                    pick = i0 + __ffs(mm) - 1;
                    break;
                }
                r -= c;
            }
            if (lane == 0) {
                idx[k] = drv[pick];
                vid[k] = l.cand[drv[pick]];
            }
            __syncwarp();
        }
        if (lane == 0 && weight > 0.0) atomicAdd(p.out, weight / (double)walks);
        __syncwarp();
    }
}

// A connected order of the vertices of S (bit u = query vertex u): from the
// vertex with the fewest candidates, always the vertex with the most earlier
// neighbours next (ties: fewer candidates, then the lower id).
std::vector<uint32_t> subset_order(const asdm_cs &cs, uint64_t S) {
    const QueryGraph &q = cs.q;
    std::vector<uint32_t> order;
    uint64_t in = 0;
    uint32_t start = kNone;
    for (uint64_t r = S; r; r &= r - 1) {
        const uint32_t u = (uint32_t)__builtin_ctzll(r);
        if (start == kNone || cs.ncand[u] < cs.ncand[start]) start = u;
    }
    order.push_back(start);
    in |= 1ull << start;
    while (in != S) {
        uint32_t best = kNone, best_links = 0;
        for (uint64_t r = S & ~in; r; r &= r - 1) {
            const uint32_t u = (uint32_t)__builtin_ctzll(r);
            uint32_t links = 0;
            for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) links += (in >> q.nbr[e]) & 1u;
            if (!links) continue;
            if (best == kNone || links > best_links || (links == best_links && cs.ncand[u] < cs.ncand[best])) {
                best = u;
                best_links = links;
            }
        }
        if (best == kNone) break;  // S not connected
        order.push_back(best);
        in |= 1ull << best;
    }
    return order;
}

}  // namespace

// Sampling estimates of the partial-match counts of the given vertex subsets
// (connected; bit u = query vertex u), `walks` walks each.
int sample_subsets(asdm_cs &cs, const std::vector<uint64_t> &subsets, uint32_t walks, uint64_t seed,
                   std::vector<double> &est) {
    asdm_graph *G = cs.g;
    cudaStream_t s = G->stream;
    const QueryGraph &q = cs.q;
    est.assign(subsets.size(), 0.0);
    if (!cs.nonempty || subsets.empty() || walks == 0) return ASDM_OK;
    std::vector<SLevel> lv;
    std::vector<SBack> bk;
    std::vector<uint32_t> cf;
    std::vector<SPrefix> pre;
    for (uint64_t S : subsets) {
        const std::vector<uint32_t> order = subset_order(cs, S);
        if (order.size() != (size_t)__builtin_popcountll(S)) return fail(ASDM_ERR_INVALID, "subset is not connected");
        SPrefix p{(uint32_t)lv.size(), (uint32_t)order.size(), nullptr};
        for (uint32_t k = 0; k < order.size(); ++k) {
            const uint32_t u = order[k];
            SLevel l{cs.d_cand + cs.cand_base[u], cs.ncand[u], 0, (uint32_t)bk.size(), 0, 0, 0};
            for (uint32_t j = 0; j < k; ++j) {
                const uint32_t w = order[j];
                const int slot = q.slot(w, u);
                if (slot >= 0) {
                    const uint32_t e = q.off[w] + (uint32_t)slot;
                    bk.push_back(SBack{cs.d_eoff + cs.eoff_base[e], cs.d_elist + cs.elist_base[e], j, 0});
                    ++l.nback;
                }
            }
            l.conf_first = (uint32_t)cf.size();
            for (uint32_t j = 0; j < k; ++j)
                if (q.lab[order[j]] == q.lab[u] && q.slot(order[j], u) < 0) cf.push_back(j);
            l.nconf = (uint32_t)cf.size() - l.conf_first;
            lv.push_back(l);
        }
        pre.push_back(p);
    }
    if (bk.empty()) bk.push_back(SBack{});
    if (cf.empty()) cf.push_back(0);
    SLevel *d_lv = nullptr;
    SBack *d_bk = nullptr;
    uint32_t *d_cf = nullptr;
    SPrefix *d_pre = nullptr;
    double *d_out = nullptr;
    int rc = ASDM_OK;
    do {
        if ((rc = dalloc(&d_lv, lv.size(), s)) || (rc = dalloc(&d_bk, bk.size(), s)) ||
            (rc = dalloc(&d_cf, cf.size(), s)) || (rc = dalloc(&d_pre, pre.size(), s)) ||
            (rc = dalloc(&d_out, pre.size(), s)))
            break;
        for (size_t k = 0; k < pre.size(); ++k) pre[k].out = d_out + k;
        if (cudaMemsetAsync(d_out, 0, pre.size() * sizeof(double), s) != cudaSuccess ||
            cudaMemcpyAsync(d_lv, lv.data(), lv.size() * sizeof(SLevel), cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(d_bk, bk.data(), bk.size() * sizeof(SBack), cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(d_cf, cf.data(), cf.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemcpyAsync(d_pre, pre.data(), pre.size() * sizeof(SPrefix), cudaMemcpyHostToDevice, s) !=
                cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "sampling upload failed");
            break;
        }
        const uint64_t total = (uint64_t)walks * pre.size();
        const unsigned grid = (unsigned)std::min<uint64_t>((total + kSampleWarps - 1) / kSampleWarps,
                                                           (uint64_t)G->num_sms * 16);
        sample_walks<<<grid, kSampleWarps * 32, 0, s>>>(d_pre, total, walks, d_lv, d_bk, d_cf, seed);
        ::asdm::count_launch();
        if (cudaGetLastError() != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "sampling kernel failed");
            break;
        }
        if (cudaMemcpyAsync(est.data(), d_out, pre.size() * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            rc = fail(ASDM_ERR_CUDA, "sampling readback failed");
    } while (false);
    cudaStreamSynchronize(s);  // the uploads read host vectors
    dfree(d_lv, s);
    dfree(d_bk, s);
    dfree(d_cf, s);
    dfree(d_pre, s);
    dfree(d_out, s);
    return rc;
}

}  // namespace asdm

using namespace asdm;

extern "C" int asdm_sample_subsets(asdm_cs *cs, uint32_t nsub, const uint64_t *masks, uint32_t walks, uint64_t seed,
                                   double *est) {
    clear_error();
    if (!cs || (nsub && (!masks || !est))) return fail(ASDM_ERR_INVALID, "null argument");
    for (uint32_t i = 0; i < nsub; ++i) {
        est[i] = 0.0;
        if (masks[i] == 0 || (cs->q.n < 64 && (masks[i] >> cs->q.n) != 0))
            return fail(ASDM_ERR_INVALID, "subset %u names a vertex outside the query", i);
    }
    if (!cs->nonempty || nsub == 0) return ASDM_OK;
    std::vector<double> out;
    ASDM_TRY(sample_subsets(*cs, std::vector<uint64_t>(masks, masks + nsub), walks ? walks : 512, seed, out));
    std::copy(out.begin(), out.end(), est);
    return ASDM_OK;
}

extern "C" int asdm_card_sample(asdm_cs *cs, uint32_t max_subset, uint32_t walks, uint64_t seed, asdm_card **out) {
    clear_error();
    if (!cs || !out) return fail(ASDM_ERR_INVALID, "null argument");
    *out = nullptr;
    if (max_subset == 0) max_subset = 6;
    if (walks == 0) walks = 512;
    asdm_card *card = nullptr;
    ASDM_TRY(asdm_card_create(&card));
    if (cs->nonempty) {
        // the largest subset size whose connected subsets stay within the planner's limit
        std::vector<uint64_t> subsets;
        uint32_t k = std::min<uint32_t>(max_subset, cs->q.n);
        while (k >= 3 && !connected_subsets(cs->q, k, kDpMaxSubsets, subsets)) --k;
        std::vector<uint64_t> pick;
        for (uint64_t S : subsets)
            if (__builtin_popcountll(S) >= 3) pick.push_back(S);
        std::vector<double> est;
        const int rc = sample_subsets(*cs, pick, walks, seed, est);
        if (rc != ASDM_OK) {
            asdm_card_free(card);
            return rc;
        }
        for (size_t i = 0; i < pick.size(); ++i) asdm_card_set(card, pick[i], est[i]);
    }
    *out = card;
    return ASDM_OK;
}
