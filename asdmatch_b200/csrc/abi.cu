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
// one driver element per round and gallops in the other lists from cursors
// that advance with the driver (leapfrog seek; utility/compute_set_intersection.cpp:177-233).
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
                const uint32_t q = valid ? gallop_lb(lst, cur[j], lj, x) : lj;
                ok = ok && q < lj && lst[q] == x;
                const uint32_t nc = __shfl_sync(kFull, q, lastlane);
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

extern "C" int asdm_cs_stats(const asdm_cs *cs, uint64_t *build_bytes, double *build_ms) {
    if (!cs) return fail(ASDM_ERR_INVALID, "null argument");
    if (build_bytes) *build_bytes = cs->build_bytes;
    if (build_ms) *build_ms = cs->build_ms;
    return ASDM_OK;
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

extern "C" int asdm_run_batch(asdm_graph *g, uint32_t nq, const uint32_t *q_sizes, const uint64_t *q_off_base,
                              const uint32_t *q_offsets, const uint64_t *q_nbr_base, const uint32_t *q_nbrs,
                              const uint64_t *q_lab_base, const uint32_t *q_labels, double time_limit_s,
                              uint64_t *counts, int *status) {
    clear_error();
    if (!g || (nq && (!q_sizes || !q_off_base || !q_offsets || !q_nbr_base || !q_nbrs || !q_lab_base || !q_labels ||
                      !counts || !status)))
        return fail(ASDM_ERR_INVALID, "null argument");
    int worst = ASDM_OK;
    for (uint32_t i = 0; i < nq; ++i) {
        asdm_run_opts o{};
        o.mode = ASDM_MODE_COUNT;
        o.time_limit_s = time_limit_s;
        asdm_run_stats st{};
        const int rc = asdm_count_query(g, q_offsets + q_off_base[i], q_nbrs + q_nbr_base[i], q_labels + q_lab_base[i],
                                        q_sizes[i], &o, &st);
        status[i] = rc;
        counts[i] = rc == ASDM_OK ? st.count : 0;
        if (rc != ASDM_OK && worst == ASDM_OK) worst = rc;
        if (rc == ASDM_ERR_CUDA) break;
    }
    return worst;
}
