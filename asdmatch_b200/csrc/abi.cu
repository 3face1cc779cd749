// Remaining C-ABI entry points: batched set intersection (K4 as a standalone
// primitive), the multi-query front end and the version string.
#include <algorithm>
#include <atomic>
#include <memory>

#include "cs.cuh"

namespace asdm {
namespace {

constexpr uint32_t kFull = 0xffffffffu;

// Warp per intersection problem: the shortest list drives, every lane takes
// one driver element per round and looks it up in the other lists from cursors
// that advance with the driver (leapfrog seek; utility/compute_set_intersection.cpp:177-233):
// a list whose unread part is at most kMergeRatio times the driver's is merged
// a window of 32 entries at a time, a longer one is galloped by every lane
// (the reference's merge/gallop switch, :9-30).
constexpr uint32_t kMergeRatio = 8;
__global__ void __launch_bounds__(256) intersect_kernel(const uint32_t *__restrict__ values,
                                                        const uint64_t *__restrict__ list_off,
                                                        const uint32_t *__restrict__ list_first, uint32_t nsets,
                                                        const uint64_t *__restrict__ out_off, uint32_t *__restrict__ out,
                                                        uint32_t *__restrict__ out_count) {
    __shared__ uint32_t cur_s[8][32];
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t *cur = cur_s[w];
    const uint32_t nwarps = gridDim.x * (blockDim.x >> 5);
    for (uint32_t s = blockIdx.x * (blockDim.x >> 5) + w; s < nsets; s += nwarps) {
        const uint32_t first = list_first[s], k = list_first[s + 1] - list_first[s];
        if (k == 0) {
            if (lane == 0) out_count[s] = 0;
            continue;
        }
        uint32_t len = 0xFFFFFFFFu;
        uint64_t start = 0;
        if (lane < k) {
            start = list_off[first + lane];
            len = (uint32_t)(list_off[first + lane + 1] - start);
            cur[lane] = 0;
        }
        uint32_t key = len, who = lane;
        for (int o = 16; o; o >>= 1) {
            const uint32_t k2 = __shfl_xor_sync(kFull, key, o), w2 = __shfl_xor_sync(kFull, who, o);
            if (k2 < key || (k2 == key && w2 < who)) { key = k2; who = w2; }
        }
        __syncwarp();
        const uint64_t dstart = __shfl_sync(kFull, start, who);
        const uint32_t *dl = values + dstart;
        uint32_t produced = 0;
        for (uint32_t p0 = 0; p0 < key; p0 += 32) {
            const uint32_t p = p0 + lane;
            const bool valid = p < key;
            const uint32_t x = valid ? dl[p] : 0xFFFFFFFFu;
            const uint32_t lastlane = min(31u, key - 1 - p0);
            bool ok = valid;
            for (uint32_t j = 0; j < k; ++j) {
                if (j == who) continue;
                const uint64_t sj = __shfl_sync(kFull, start, j);
                const uint32_t lj = __shfl_sync(kFull, len, j);
                const uint32_t *lst = values + sj;
                const uint32_t cj = cur[j];
                uint32_t nc;
                if ((uint64_t)(lj - cj) <= (uint64_t)kMergeRatio * (key - p0)) {
                    ok = warp_merge_member(lst, cj, lj, x, ok, lastlane, lane, nc) && ok;
                } else {
                    const uint32_t q = valid ? gallop_lb(lst, cj, lj, x) : lj;
                    ok = ok && q < lj && lst[q] == x;
                    nc = __shfl_sync(kFull, q, lastlane);
                }
                __syncwarp();
                if (lane == 0) cur[j] = nc;
                __syncwarp();
            }
            const uint32_t m = __ballot_sync(kFull, ok);
            if (ok) out[out_off[s] + produced + __popc(m & ((1u << lane) - 1))] = x;
            produced += __popc(m);
        }
        if (lane == 0) out_count[s] = produced;
    }
}

}  // namespace
}  // namespace asdm

namespace asdm {
static std::atomic<unsigned long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
}  // namespace asdm

using namespace asdm;

extern "C" uint64_t asdm_kernel_launches(void) { return asdm::g_launches.load(); }

extern "C" int asdm_graph_stream(asdm_graph *g, void **stream) {
    if (!g || !stream) return fail(ASDM_ERR_INVALID, "null argument");
    *stream = (void *)g->stream;
    return ASDM_OK;
}

extern "C" int asdm_graph_set_tuning(asdm_graph *g, const asdm_tuning *t) {
    if (!g || !t) return fail(ASDM_ERR_INVALID, "null argument");
    if (t->enum_min_blocks < 1 || t->enum_min_blocks > 6)
        return fail(ASDM_ERR_INVALID, "enum_min_blocks must be 1 to 6");
    if (t->lane_leaf_max > 4096) return fail(ASDM_ERR_INVALID, "lane_leaf_max must be <= 4096");
    if (t->root_block_min < 1 || t->root_block_min > 256) return fail(ASDM_ERR_INVALID, "root_block_min must be 1..256");
    if (t->planner != ASDM_PLANNER_DP && t->planner != ASDM_PLANNER_GREEDY)
        return fail(ASDM_ERR_INVALID, "planner must be ASDM_PLANNER_DP or ASDM_PLANNER_GREEDY");
    if (t->padded_cap_log2 < 20 || t->padded_cap_log2 > 34) return fail(ASDM_ERR_INVALID, "padded_cap_log2 must be 20..34");
    if (t->merge_ratio > 1024) return fail(ASDM_ERR_INVALID, "merge_ratio must be <= 1024");
    g->tuning = *t;
    return ASDM_OK;
}

extern "C" int asdm_graph_get_tuning(const asdm_graph *g, asdm_tuning *t) {
    if (!g || !t) return fail(ASDM_ERR_INVALID, "null argument");
    *t = g->tuning;
    return ASDM_OK;
}

extern "C" int asdm_cs_edge_totals(const asdm_cs *cs, uint64_t *totals) {
    if (!cs || !totals) return fail(ASDM_ERR_INVALID, "null argument");
    const uint32_t ne = cs->q.off[cs->q.n];
    for (uint32_t e = 0; e < ne; ++e) totals[e] = cs->nonempty ? cs->etotal[e] : 0;
    return ASDM_OK;
}

extern "C" int asdm_cs_stats(const asdm_cs *cs, uint64_t *build_bytes, double *build_ms) {
    if (!cs) return fail(ASDM_ERR_INVALID, "null argument");
    if (build_bytes) *build_bytes = cs->build_bytes;
    if (build_ms) *build_ms = cs->build_ms;
    return ASDM_OK;
}

namespace asdm {
__device__ __forceinline__ unsigned long long digest_mix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Sum over i of mix(tag, i, a[i]): independent of the order threads add in.
__global__ void digest_kernel(const uint32_t *__restrict__ a, uint64_t n, unsigned long long tag,
                              unsigned long long *__restrict__ out) {
    unsigned long long acc = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        acc += digest_mix64(tag * 0x9E3779B97F4A7C15ull + i * 0xD1B54A32D192ED03ull + a[i]);
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(out, acc);
}
}  // namespace asdm

extern "C" int asdm_cs_digest(const asdm_cs *cs, uint64_t *digest, uint32_t *flags) {
    clear_error();
    if (!cs || !digest) return fail(ASDM_ERR_INVALID, "null argument");
    *digest = 0;
    if (flags) *flags = cs->build_flags;
    if (!cs->nonempty) return ASDM_OK;
    cudaStream_t s = cs->g->stream;
    unsigned long long *d = nullptr;
    ASDM_TRY(dalloc(&d, 1, s));
    int rc = cudaMemsetAsync(d, 0, sizeof(unsigned long long), s) == cudaSuccess ? ASDM_OK
                                                                                  : fail(ASDM_ERR_CUDA, "digest reset");
    const QueryGraph &q = cs->q;
    auto run = [&](const uint32_t *a, uint64_t n, unsigned long long tag) {
        if (rc != ASDM_OK || n == 0) return;
        const unsigned grid = (unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
        digest_kernel<<<grid, 256, 0, s>>>(a, n, tag, d);
        ::asdm::count_launch();
        if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "digest kernel failed");
    };
    for (uint32_t u = 0; u < q.n; ++u) run(cs->d_cand + cs->cand_base[u], cs->ncand[u], 1 + u);
    for (uint32_t u = 0; u < q.n; ++u)
        for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
            run(cs->d_eoff + cs->eoff_base[e], cs->ncand[u] + 1ull, 1000 + 2ull * e);
            run(cs->d_elist + cs->elist_base[e], cs->etotal[e], 1001 + 2ull * e);
        }
    unsigned long long h = 0;
    if (rc == ASDM_OK && (cudaMemcpyAsync(&h, d, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                          cudaStreamSynchronize(s) != cudaSuccess))
        rc = fail(ASDM_ERR_CUDA, "digest readback failed");
    dfree(d, s);
    cudaStreamSynchronize(s);
    *digest = h;
    return rc;
}

extern "C" const char *asdm_version(void) { return "asdmatch-b200 0.1 (sm_100a)"; }

extern "C" int asdm_intersect_batch(const uint32_t *values, const uint64_t *list_off, uint64_t nlists,
                                    const uint32_t *list_first, uint32_t nsets, const uint64_t *out_off, uint32_t *out,
                                    uint32_t *out_count) {
    clear_error();
    if (!list_off || !list_first || !out_off || !out_count || (nsets && !out)) return fail(ASDM_ERR_INVALID, "null argument");
    if (nsets == 0) return ASDM_OK;
    if (list_first[nsets] > nlists) return fail(ASDM_ERR_INVALID, "list index out of range");
    uint64_t out_total = 0;
    for (uint32_t s = 0; s < nsets; ++s) {
        const uint32_t k = list_first[s + 1] - list_first[s];
        if (list_first[s + 1] < list_first[s] || k > 32) return fail(ASDM_ERR_INVALID, "set %u: 0..32 lists supported", s);
        uint64_t mn = k ? ~0ull : 0;
        for (uint32_t j = 0; j < k; ++j) {
            const uint64_t l = list_off[list_first[s] + j + 1] - list_off[list_first[s] + j];
            if (l >= 0xFFFFFFFFull) return fail(ASDM_ERR_INVALID, "list too long");
            mn = std::min(mn, l);
        }
        if (out_off[s] + mn > out_off[s + 1]) return fail(ASDM_ERR_INVALID, "output slot %u smaller than its shortest list", s);
        out_total = std::max(out_total, out_off[s + 1]);
    }
    const uint64_t nvals = list_off[nlists];
    int dev = 0, sms = 0;
    ASDM_TRY(device_setup(&dev, &sms));
    cudaStream_t s;
    ASDM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    uint32_t *d_vals = nullptr, *d_first = nullptr, *d_out = nullptr, *d_cnt = nullptr;
    uint64_t *d_loff = nullptr, *d_ooff = nullptr;
    int rc = ASDM_OK;
    do {
        if ((rc = dalloc(&d_vals, nvals, s)) || (rc = dalloc(&d_loff, nlists + 1, s)) ||
            (rc = dalloc(&d_first, nsets + 1, s)) || (rc = dalloc(&d_ooff, nsets + 1, s)) ||
            (rc = dalloc(&d_out, out_total, s)) || (rc = dalloc(&d_cnt, nsets, s)))
            break;
        if ((nvals && cudaMemcpyAsync(d_vals, values, nvals * 4, cudaMemcpyHostToDevice, s)) ||
            cudaMemcpyAsync(d_loff, list_off, (nlists + 1) * 8, cudaMemcpyHostToDevice, s) ||
            cudaMemcpyAsync(d_first, list_first, (nsets + 1) * 4, cudaMemcpyHostToDevice, s) ||
            cudaMemcpyAsync(d_ooff, out_off, (nsets + 1) * 8, cudaMemcpyHostToDevice, s)) {
            rc = fail(ASDM_ERR_CUDA, "upload failed");
            break;
        }
        const unsigned grid = (unsigned)std::min<uint64_t>((nsets + 7) / 8, (uint64_t)sms * 16);
        intersect_kernel<<<grid, 256, 0, s>>>(d_vals, d_loff, d_first, nsets, d_ooff, d_out, d_cnt);
        ::asdm::count_launch();
        if (cudaGetLastError() != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "intersection launch failed");
            break;
        }
        if ((out_total && cudaMemcpyAsync(out, d_out, out_total * 4, cudaMemcpyDeviceToHost, s)) ||
            cudaMemcpyAsync(out_count, d_cnt, nsets * 4, cudaMemcpyDeviceToHost, s) || cudaStreamSynchronize(s)) {
            rc = fail(ASDM_ERR_CUDA, "intersection failed: %s", cudaGetErrorString(cudaGetLastError()));
            break;
        }
    } while (false);
    dfree(d_vals, s); dfree(d_loff, s); dfree(d_first, s); dfree(d_ooff, s); dfree(d_out, s); dfree(d_cnt, s);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    return rc;
}

namespace asdm {
int build_plan(const asdm_cs &cs, const uint32_t *user_order, asdm_plan &p, const asdm_card *card = nullptr);
int build_prefix_plan(const asdm_cs &cs, const uint32_t *order, uint32_t depth, asdm_plan &p);
int run_batch_count(asdm_graph *G, const std::vector<asdm_cs *> &cs, const std::vector<const asdm_plan *> &plans,
                    double time_limit_s, uint64_t count_limit, uint64_t *counts, int *status, asdm_run_stats *agg,
                    uint64_t *const *local_out, uint64_t *cycles = nullptr, double query_time_s = 0.0,
                    bool settled = false);
int settle_queries(asdm_graph *G, const std::vector<asdm_cs *> &cs, const std::vector<char> &full,
                   std::vector<uint32_t> &live, uint64_t count_limit, uint64_t *counts, int *status,
                   asdm_run_stats *agg, uint64_t *const *local_out);
int plan_batch_learned(const std::vector<asdm_cs *> &css, asdm_estimator *e, uint32_t kmax,
                       std::vector<asdm_plan> &plans);
}  // namespace asdm

// Candidate-space state a group may hold at once (state words, storage and
// candidate arrays: 12 bytes per data vertex of each query vertex's label).
static constexpr uint64_t kGroupStateBytes = 32ull << 30;

static int run_batch_impl(asdm_graph *g, uint32_t nq, const uint32_t *q_sizes, const uint64_t *q_off_base,
                          const uint32_t *q_offsets, const uint64_t *q_nbr_base, const uint32_t *q_nbrs,
                          const uint64_t *q_lab_base, const uint32_t *q_labels, double time_limit_s,
                          uint64_t count_limit, const asdm_card *const *cards, asdm_estimator *est,
                          uint32_t est_kmax, uint64_t *counts, int *status, asdm_run_stats *stats,
                          uint64_t *const *local_out, double query_time_s = 0.0) {
    clear_error();
    if (stats) *stats = asdm_run_stats{};
    if (!g || (nq && (!q_sizes || !q_off_base || !q_offsets || !q_nbr_base || !q_nbrs || !q_lab_base || !q_labels ||
                      !counts || !status)))
        return fail(ASDM_ERR_INVALID, "null argument");
    std::vector<std::unique_ptr<asdm_cs>> all(nq);
    std::vector<uint64_t> state(nq, 0);
    for (uint32_t i = 0; i < nq; ++i) {
        counts[i] = 0;
        status[i] = ASDM_OK;
        auto c = std::make_unique<asdm_cs>();
        c->g = g;
        const int rc = make_query(q_offsets + q_off_base[i], q_nbrs + q_nbr_base[i], q_labels + q_lab_base[i],
                                  q_sizes[i], c->q);
        if (rc != ASDM_OK) {
            status[i] = rc;
            continue;
        }
        for (uint32_t u = 0; u < c->q.n; ++u) {
            const uint32_t l = c->q.lab[u];
            if (l < g->d.nlabels) state[i] += 12ull * (g->h_vbl_off[l + 1] - g->h_vbl_off[l]);
        }
        if (local_out) {
            state[i] += 8ull * g->d.n * c->q.n;  // the query's local-count block
            if (local_out[i]) std::fill(local_out[i], local_out[i] + (uint64_t)g->d.n * c->q.n, 0ull);
        }
        all[i] = std::move(c);
    }
    int worst = ASDM_OK;
    for (uint32_t i = 0; i < nq && worst != ASDM_ERR_CUDA; ++i)
        if (status[i] != ASDM_OK && worst == ASDM_OK) worst = status[i];
    uint32_t i = 0;
    while (i < nq) {
        // next group: consecutive valid queries within the state budget
        std::vector<uint32_t> ids;
        uint64_t bytes = 0;
        for (; i < nq; ++i) {
            if (!all[i]) continue;
            if (!ids.empty() && bytes + state[i] > kGroupStateBytes) break;
            ids.push_back(i);
            bytes += state[i];
        }
        if (ids.empty()) continue;
        std::vector<asdm_cs *> group;
        for (uint32_t id : ids) group.push_back(all[id].get());
        int rc = build_batch(group);
        if (rc != ASDM_OK) {
            for (uint32_t id : ids) status[id] = rc;
            if (worst == ASDM_OK) worst = rc;
            if (rc == ASDM_ERR_CUDA) break;
            continue;
        }
        // queries the tree program or an overflow bound settles need no plan:
        // settle first, then plan (cost model, .card or learned) the rest
        asdm_run_stats gs{};
        std::vector<uint32_t> open;
        {
            std::vector<uint32_t> live;
            for (uint32_t k = 0; k < ids.size(); ++k)
                if (group[k]->nonempty) live.push_back(k);  // an empty space counts 0, like the reference's early return
            std::vector<char> full(ids.size(), 1);
            std::vector<uint64_t> sc(ids.size(), 0);
            std::vector<int> sst(ids.size(), ASDM_OK);
            std::vector<uint64_t *> slo;
            if (local_out)
                for (uint32_t id : ids) slo.push_back(local_out[id]);
            const std::vector<uint32_t> before = live;
            rc = settle_queries(g, group, full, live, count_limit, sc.data(), sst.data(), &gs,
                                local_out ? slo.data() : nullptr);
            if (rc != ASDM_OK) {
                for (uint32_t id : ids) status[id] = rc;
                if (worst == ASDM_OK) worst = rc;
                if (rc == ASDM_ERR_CUDA) break;
                continue;
            }
            std::vector<char> still(ids.size(), 0);
            for (uint32_t k : live) still[k] = 1;
            for (uint32_t k : before) {
                if (still[k]) continue;
                counts[ids[k]] = sc[k];
                status[ids[k]] = sst[k];
                if (sst[k] != ASDM_OK && worst == ASDM_OK) worst = sst[k];
            }
            open = live;
        }
        std::vector<asdm_cs *> open_cs;
        for (uint32_t k : open) open_cs.push_back(group[k]);
        std::vector<asdm_plan> plans(open.size());
        std::vector<asdm_cs *> run_cs;
        std::vector<const asdm_plan *> run_plans;
        std::vector<uint32_t> run_ids;
        int learned_rc = ASDM_OK;
        if (est && !open_cs.empty()) learned_rc = plan_batch_learned(open_cs, est, est_kmax, plans);
        for (size_t j = 0; j < open.size(); ++j) {
            const uint32_t k = open[j];
            int prc;
            if (!est) prc = build_plan(*group[k], nullptr, plans[j], cards ? cards[ids[k]] : nullptr);
            else if (learned_rc != ASDM_OK) prc = learned_rc;
            else if (plans[j].order.size() != group[k]->q.n) prc = fail(ASDM_ERR_INVALID, "query is not connected");
            else prc = ASDM_OK;
            if (prc != ASDM_OK) {
                status[ids[k]] = prc;
                if (worst == ASDM_OK) worst = prc;
                continue;
            }
            run_cs.push_back(group[k]);
            run_plans.push_back(&plans[j]);
            run_ids.push_back(ids[k]);
        }
        std::vector<uint64_t> c(run_ids.size());
        std::vector<int> st(run_ids.size());
        std::vector<uint64_t *> lo;
        if (local_out)
            for (uint32_t id : run_ids) lo.push_back(local_out[id]);
        {
            asdm_run_stats es{};
            rc = run_batch_count(g, run_cs, run_plans, time_limit_s, count_limit, c.data(), st.data(), &es,
                                 local_out ? lo.data() : nullptr, nullptr, query_time_s, /*settled=*/true);
            gs.count += es.count;
            gs.intersections += es.intersections;
            gs.list_bytes += es.list_bytes;
            gs.tasks += es.tasks;
            gs.kernel_ms += es.kernel_ms;
            gs.tails_lane += es.tails_lane;
            gs.tails_warp += es.tails_warp;
            gs.busy_warp_ms += es.busy_warp_ms;
            gs.idle_warp_ms += es.idle_warp_ms;
        }
        if (stats) {
            stats->count += gs.count;
            stats->intersections += gs.intersections;
            stats->list_bytes += gs.list_bytes;
            stats->tasks += gs.tasks;
            stats->kernel_ms += gs.kernel_ms;
            stats->tails_lane += gs.tails_lane;
            stats->tails_warp += gs.tails_warp;
            stats->busy_warp_ms += gs.busy_warp_ms;
            stats->idle_warp_ms += gs.idle_warp_ms;
            for (asdm_cs *gc : group) {
                stats->build_ms += gc->build_ms;
                stats->build_bytes += gc->build_bytes;
            }
        }
        for (size_t k = 0; k < run_ids.size(); ++k) {
            counts[run_ids[k]] = c[k];
            status[run_ids[k]] = st[k];
            if (st[k] != ASDM_OK && worst == ASDM_OK) worst = st[k];
        }
        if (rc != ASDM_OK && worst == ASDM_OK) worst = rc;
        for (uint32_t id : ids) all[id].reset();
        if (rc == ASDM_ERR_CUDA) break;
    }
    return worst;
}

extern "C" int asdm_run_batch(asdm_graph *g, uint32_t nq, const uint32_t *q_sizes, const uint64_t *q_off_base,
                              const uint32_t *q_offsets, const uint64_t *q_nbr_base, const uint32_t *q_nbrs,
                              const uint64_t *q_lab_base, const uint32_t *q_labels, double time_limit_s,
                              uint64_t *counts, int *status, asdm_run_stats *stats) {
    return run_batch_impl(g, nq, q_sizes, q_off_base, q_offsets, q_nbr_base, q_nbrs, q_lab_base, q_labels,
                          time_limit_s, 0, nullptr, nullptr, 0, counts, status, stats, nullptr);
}

extern "C" int asdm_run_batch_ex(asdm_graph *g, uint32_t nq, const uint32_t *q_sizes, const uint64_t *q_off_base,
                                 const uint32_t *q_offsets, const uint64_t *q_nbr_base, const uint32_t *q_nbrs,
                                 const uint64_t *q_lab_base, const uint32_t *q_labels, const asdm_batch_opts *opts,
                                 uint64_t *counts, int *status, uint64_t *const *local_counts, asdm_run_stats *stats) {
    if (!opts) return fail(ASDM_ERR_INVALID, "null options");
    return run_batch_impl(g, nq, q_sizes, q_off_base, q_offsets, q_nbr_base, q_nbrs, q_lab_base, q_labels,
                          opts->time_limit_s, opts->count_limit, opts->cards, opts->estimator,
                          opts->learned_max_subset, counts, status, stats, local_counts, opts->query_time_limit_s);
}

extern "C" int asdm_run_batch_local(asdm_graph *g, uint32_t nq, const uint32_t *q_sizes, const uint64_t *q_off_base,
                                    const uint32_t *q_offsets, const uint64_t *q_nbr_base, const uint32_t *q_nbrs,
                                    const uint64_t *q_lab_base, const uint32_t *q_labels, double time_limit_s,
                                    uint64_t *counts, int *status, uint64_t *const *local_counts,
                                    asdm_run_stats *stats) {
    if (nq && !local_counts) return fail(ASDM_ERR_INVALID, "null local-count array");
    return run_batch_impl(g, nq, q_sizes, q_off_base, q_offsets, q_nbr_base, q_nbrs, q_lab_base, q_labels,
                          time_limit_s, 0, nullptr, nullptr, 0, counts, status, stats, local_counts);
}

// Partial-match counts of many prefixes of one query in one batched launch.
extern "C" int asdm_prefix_counts(asdm_cs *cs, uint32_t nprefix, const uint32_t *orders, const uint32_t *depths,
                                  double time_limit_s, uint64_t count_limit, uint64_t *counts, int *status) {
    clear_error();
    if (!cs || (nprefix && (!orders || !depths || !counts || !status))) return fail(ASDM_ERR_INVALID, "null argument");
    const uint32_t n = cs->q.n;
    std::vector<asdm_plan> plans(nprefix);
    std::vector<asdm_cs *> run_cs;
    std::vector<const asdm_plan *> run_plans;
    std::vector<uint32_t> run_ids;
    int worst = ASDM_OK;
    for (uint32_t i = 0; i < nprefix; ++i) {
        counts[i] = 0;
        status[i] = build_prefix_plan(*cs, orders + (uint64_t)i * n, depths[i], plans[i]);
        if (status[i] != ASDM_OK) {
            if (worst == ASDM_OK) worst = status[i];
            continue;
        }
        if (!cs->nonempty) continue;  // an empty candidate space has no partial matches
        if (depths[i] == 1) {
            counts[i] = cs->ncand[orders[(uint64_t)i * n]];
            if (count_limit && counts[i] > count_limit) status[i] = ASDM_ERR_LIMIT;
            continue;
        }
        run_cs.push_back(cs);
        run_plans.push_back(&plans[i]);
        run_ids.push_back(i);
    }
    if (run_ids.empty()) return worst;
    std::vector<uint64_t> c(run_ids.size());
    std::vector<int> st(run_ids.size());
    const int rc = run_batch_count(cs->g, run_cs, run_plans, time_limit_s, count_limit, c.data(), st.data(), nullptr,
                                   nullptr);
    for (size_t k = 0; k < run_ids.size(); ++k) {
        counts[run_ids[k]] = c[k];
        status[run_ids[k]] = st[k];
        if (st[k] != ASDM_OK && worst == ASDM_OK) worst = st[k];
    }
    if (rc != ASDM_OK && (worst == ASDM_OK || rc == ASDM_ERR_CUDA)) worst = rc;
    return worst;
}

// Candidate spaces of many queries, built in groups (one K1-K3 launch per
// phase per group), for callers that plan between filtering and enumeration.
extern "C" int asdm_candidate_space_batch(asdm_graph *g, uint32_t nq, const uint32_t *q_sizes,
                                          const uint64_t *q_off_base, const uint32_t *q_offsets,
                                          const uint64_t *q_nbr_base, const uint32_t *q_nbrs,
                                          const uint64_t *q_lab_base, const uint32_t *q_labels, asdm_cs **out,
                                          int *nonempty, int *status) {
    clear_error();
    if (!g || (nq && (!q_sizes || !q_off_base || !q_offsets || !q_nbr_base || !q_nbrs || !q_lab_base || !q_labels ||
                      !out || !nonempty || !status)))
        return fail(ASDM_ERR_INVALID, "null argument");
    std::vector<std::unique_ptr<asdm_cs>> all(nq);
    std::vector<uint64_t> state(nq, 0);
    int worst = ASDM_OK;
    for (uint32_t i = 0; i < nq; ++i) {
        out[i] = nullptr;
        nonempty[i] = 0;
        auto c = std::make_unique<asdm_cs>();
        c->g = g;
        status[i] = make_query(q_offsets + q_off_base[i], q_nbrs + q_nbr_base[i], q_labels + q_lab_base[i], q_sizes[i],
                               c->q);
        if (status[i] != ASDM_OK) {
            if (worst == ASDM_OK) worst = status[i];
            continue;
        }
        for (uint32_t u = 0; u < c->q.n; ++u) {
            const uint32_t l = c->q.lab[u];
            if (l < g->d.nlabels) state[i] += 12ull * (g->h_vbl_off[l + 1] - g->h_vbl_off[l]);
        }
        all[i] = std::move(c);
    }
    uint32_t i = 0;
    while (i < nq) {
        std::vector<uint32_t> ids;
        uint64_t bytes = 0;
        for (; i < nq; ++i) {
            if (!all[i]) continue;
            if (!ids.empty() && bytes + state[i] > kGroupStateBytes) break;
            ids.push_back(i);
            bytes += state[i];
        }
        if (ids.empty()) continue;
        std::vector<asdm_cs *> group;
        for (uint32_t id : ids) group.push_back(all[id].get());
        const int rc = build_batch(group);
        for (uint32_t id : ids) {
            status[id] = rc;
            if (rc == ASDM_OK) {
                nonempty[id] = all[id]->nonempty ? 1 : 0;
                out[id] = all[id].release();
            } else {
                all[id].reset();
            }
        }
        if (rc != ASDM_OK && worst == ASDM_OK) worst = rc;
        if (rc == ASDM_ERR_CUDA) break;
    }
    return worst;
}

// One persistent launch over candidate spaces and plans the caller built.
extern "C" int asdm_run_planned_profile(uint32_t nq, asdm_cs *const *cs, const asdm_plan *const *plans,
                                        const asdm_batch_opts *opts, uint64_t *counts, int *status,
                                        asdm_run_stats *stats, uint64_t *cycles) {
    clear_error();
    if (stats) *stats = asdm_run_stats{};
    if (nq && (!cs || !plans || !counts || !status)) return fail(ASDM_ERR_INVALID, "null argument");
    asdm_graph *g = nullptr;
    std::vector<asdm_cs *> run_cs;
    std::vector<const asdm_plan *> run_plans;
    std::vector<uint32_t> run_ids;
    int worst = ASDM_OK;
    for (uint32_t i = 0; i < nq; ++i) {
        counts[i] = 0;
        status[i] = ASDM_OK;
        if (!cs[i] || !plans[i]) {
            status[i] = fail(ASDM_ERR_INVALID, "query %u has no candidate space or plan", i);
        } else if (g && cs[i]->g != g) {
            status[i] = fail(ASDM_ERR_INVALID, "query %u is on another graph", i);
        } else if (plans[i]->order.size() != cs[i]->q.n) {
            status[i] = fail(ASDM_ERR_INVALID, "plan %u does not match its query", i);
        }
        if (status[i] != ASDM_OK) {
            if (worst == ASDM_OK) worst = status[i];
            continue;
        }
        g = cs[i]->g;
        if (!cs[i]->nonempty) continue;
        run_cs.push_back(cs[i]);
        run_plans.push_back(plans[i]);
        run_ids.push_back(i);
    }
    if (run_ids.empty()) return worst;
    std::vector<uint64_t> c(run_ids.size());
    std::vector<int> st(run_ids.size());
    const double tl = opts ? opts->time_limit_s : 0.0;
    const uint64_t cl = opts ? opts->count_limit : 0;
    const double qt = opts ? opts->query_time_limit_s : 0.0;
    std::vector<uint64_t> cy(cycles ? run_ids.size() : 0);
    const int rc = run_batch_count(g, run_cs, run_plans, tl, cl, c.data(), st.data(), stats, nullptr,
                                   cycles ? cy.data() : nullptr, qt);
    if (cycles)
        for (uint32_t i = 0; i < nq; ++i) cycles[i] = 0;
    for (size_t k = 0; k < run_ids.size(); ++k) {
        counts[run_ids[k]] = c[k];
        status[run_ids[k]] = st[k];
        if (cycles) cycles[run_ids[k]] = cy[k];
        if (st[k] != ASDM_OK && worst == ASDM_OK) worst = st[k];
    }
    if (rc != ASDM_OK && (worst == ASDM_OK || rc == ASDM_ERR_CUDA)) worst = rc;
    return worst;
}

extern "C" int asdm_run_planned(uint32_t nq, asdm_cs *const *cs, const asdm_plan *const *plans,
                                const asdm_batch_opts *opts, uint64_t *counts, int *status, asdm_run_stats *stats) {
    return asdm_run_planned_profile(nq, cs, plans, opts, counts, status, stats, nullptr);
}
