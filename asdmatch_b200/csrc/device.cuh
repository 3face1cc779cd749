// Device-side structures and helpers shared by the sm_100a kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "internal.h"

#define ASDM_CUDA(call)                                                                              \
    do {                                                                                             \
        cudaError_t e__ = (call);                                                                    \
        if (e__ != cudaSuccess)                                                                      \
            return ::asdm::fail(e__ == cudaErrorMemoryAllocation ? ASDM_ERR_OOM : ASDM_ERR_CUDA,     \
                                "%s: %s (%s:%d)", #call, cudaGetErrorString(e__), __FILE__, __LINE__); \
    } while (0)

#define ASDM_TRY(call)                   \
    do {                                 \
        int rc__ = (call);               \
        if (rc__ != ASDM_OK) return rc__; \
    } while (0)

namespace asdm {

// Device view of a data graph.  Adjacency lists are sorted by (label, id);
// each list is split into label runs (run_lab ascending, run_start the first
// edge of the run, the run ends at the next run's start or at off[v+1]).
struct DevGraph {
    uint32_t n = 0, nlabels = 0;
    uint64_t m2 = 0, nruns = 0;
    const uint32_t *off = nullptr;           // n + 1
    const uint32_t *nbr = nullptr;           // m2
    const uint32_t *lab = nullptr;           // n
    const uint32_t *pos_in_label = nullptr;  // n: rank of v among vertices of its label
    const uint32_t *vbl_off = nullptr;       // nlabels + 1
    const uint32_t *vbl = nullptr;           // n: vertices grouped by label, id order
    const uint32_t *run_off = nullptr;       // n + 1
    const uint32_t *run_lab = nullptr;       // nruns
    const uint32_t *run_start = nullptr;     // nruns
    const uint32_t *nbr_rank = nullptr;      // m2: pos_in_label of nbr[k]
    const uint2 *rank_info = nullptr;        // n, in vbl order: {degree, bit (l mod 32) per neighbour label l}
    // n x (nlabels + 1), or null: row v holds, for every label l, the first
    // edge of v whose neighbour has label >= l (then off[v+1]); the run of l is
    // [row[l], row[l+1]).  Built when it fits kLabPosCap bytes.
    const uint32_t *lab_pos = nullptr;
};

constexpr uint64_t kLabPosCap = 1ull << 30;

// [b, e) edge range of label l in w's adjacency (empty if w has no such neighbour).
__device__ __forceinline__ void label_run(const DevGraph &g, uint32_t w, uint32_t l, uint32_t &b, uint32_t &e) {
    if (g.lab_pos) {
        // one row of the dense table: both ends in one or two sectors
        if (l < g.nlabels) {
            const uint32_t *r = g.lab_pos + (uint64_t)w * (g.nlabels + 1) + l;
            b = r[0];
            e = r[1];
        } else {
            b = e = 0;
        }
        return;
    }
    uint32_t lo = g.run_off[w], hi = g.run_off[w + 1];
    const uint32_t end = hi;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (g.run_lab[mid] < l) lo = mid + 1; else hi = mid;
    }
    if (lo < end && g.run_lab[lo] == l) {
        b = g.run_start[lo];
        e = (lo + 1 < end) ? g.run_start[lo + 1] : g.off[w + 1];
    } else {
        b = e = 0;
    }
}

// First index in [lo, n) with a[i] >= x: exponential probe from lo, then
// binary search (the leapfrog seek of the leapfrog-triejoin paper).
__device__ __forceinline__ uint32_t gallop_lb(const uint32_t *__restrict__ a, uint32_t lo, uint32_t n, uint32_t x) {
    if (lo >= n || a[lo] >= x) return lo;
    uint32_t prev = lo, step = 1, hi = n;
    while (true) {
        uint32_t nxt = prev + step;
        if (nxt >= n) { hi = n; break; }
        if (a[nxt] >= x) { hi = nxt; break; }
        prev = nxt;
        step <<= 1;
    }
    lo = prev + 1;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

#ifdef __CUDACC__
// Warp-cooperative merge probe, the counterpart of galloping for lists of
// similar length (the reference switches from galloping to a linear merge when
// the lengths differ by less than 50x, utility/compute_set_intersection.cpp:9-30).
// Lane i holds x_i; x ascends over lanes 0..last, lanes past `last` hold
// 0xFFFFFFFF.  Every entry of a[0, cur) is below x_0.  The warp reads a[cur, n)
// one window of 32 entries at a time (one coalesced 128-byte load) and each
// lane finds the number of window entries below its x in five shuffle steps.
// A lane is settled by the first window whose last entry is >= its x.  The
// loop ends when x_last is settled, or when no lane with `want` set is still
// unsettled.  Returns whether x_i is in a (meaningful where `want` is set);
// *ncur gets a position p <= lower_bound(a, x_last) with every a[0, p) below
// x_last, the cursor of the next round of drivers.
__device__ __forceinline__ bool warp_merge_member(const uint32_t *__restrict__ a, uint32_t cur, uint32_t n, uint32_t x,
                                                  bool want, uint32_t last, uint32_t lane, uint32_t &ncur) {
    constexpr uint32_t full = 0xffffffffu;
    const uint32_t xl = __shfl_sync(full, x, last);
    bool hit = false;
    uint32_t c = cur;
    ncur = n;
    while (c < n) {
        const uint32_t j = c + lane;
        const uint32_t y = j < n ? a[j] : 0xFFFFFFFFu;
        uint32_t r = 0;  // entries of the window below x (at most 31 here)
#pragma unroll
        for (uint32_t s = 16; s; s >>= 1) {
            const uint32_t yv = __shfl_sync(full, y, r + s - 1);
            if (yv < x) r += s;
        }
        const uint32_t yr = __shfl_sync(full, y, r);
        const uint32_t ylast = __shfl_sync(full, y, 31);
        hit = hit || (want && lane <= last && yr == x);
        const uint32_t rl = __shfl_sync(full, r, last);
        if (ylast >= xl) {
            ncur = c + rl;
            break;
        }
        // every entry of this window is below x_last
        if (!__any_sync(full, want && x > ylast)) {
            ncur = min(c + 32, n);
            break;
        }
        c += 32;
    }
    return hit;
}
#endif

__device__ __forceinline__ uint32_t lower_bound_u32(const uint32_t *__restrict__ a, uint32_t n, uint32_t x) {
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Exclusive prefix sum of n values (uint32 or uint64 input) into uint64
// output; out[n] receives the total when out has n + 1 slots and
// with_total is set.  Temporary memory comes from the stream-ordered pool.
int scan_exclusive_u32(const uint32_t *in, uint64_t *out, uint64_t n, bool with_total, cudaStream_t s);
int scan_exclusive_u64(const uint64_t *in, uint64_t *out, uint64_t n, bool with_total, cudaStream_t s);

// Stream-ordered allocation helpers with error reporting.
template <typename T>
int dalloc(T **p, uint64_t count, cudaStream_t s) {
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMallocAsync((void **)p, count * sizeof(T), s);
    if (e != cudaSuccess)
        return fail(e == cudaErrorMemoryAllocation ? ASDM_ERR_OOM : ASDM_ERR_CUDA, "device allocation of %llu bytes: %s",
                    (unsigned long long)(count * sizeof(T)), cudaGetErrorString(e));
    return ASDM_OK;
}
template <typename T>
void dfree(T *&p, cudaStream_t s) {
    if (p) cudaFreeAsync((void *)p, s);
    p = nullptr;
}

int device_setup(int *device, int *num_sms);

// Number of kernels this library has launched (all threads, all devices).
void count_launch();

}  // namespace asdm

// Pinned host memory for descriptor uploads: a copy from pageable memory
// first waits for the stream, a copy from pinned memory does not.  Memory
// handed out stays valid until the next reset().
struct PinnedStage {
    std::vector<std::pair<uint8_t *, size_t>> chunks;
    size_t cur = 0, off = 0;
    void reset() { cur = 0; off = 0; }
    void *put(const void *src, size_t bytes) {
        const size_t need = (bytes + 63) & ~size_t(63);
        while (cur < chunks.size() && off + need > chunks[cur].second) { ++cur; off = 0; }
        if (cur == chunks.size()) {
            uint8_t *p = nullptr;
            const size_t sz = std::max<size_t>(need, 4u << 20);
            if (cudaMallocHost((void **)&p, sz) != cudaSuccess) return nullptr;
            chunks.emplace_back(p, sz);
            off = 0;
        }
        uint8_t *dst = chunks[cur].first + off;
        if (bytes) std::memcpy(dst, src, bytes);
        off += need;
        return dst;
    }
    ~PinnedStage() {
        for (auto &c : chunks) cudaFreeHost(c.first);
    }
};

struct asdm_graph {
    asdm_tuning tuning{1, 96, ASDM_PLANNER_DP, 64, 33, 8};         // kernel knobs (asdm_graph_set_tuning)
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    asdm::DevGraph d;
    uint32_t *buf = nullptr;               // one allocation backing every DevGraph array
    std::vector<uint32_t> h_vbl_off;       // host copy of the label offsets
    uint32_t max_deg = 0;
    PinnedStage stage;                     // descriptor uploads of the candidate-space build
};

namespace asdm {
// Host-to-device copy on the graph's stream through its pinned stage (a plain
// copy when pinned memory is not available).
inline cudaError_t upload_async(asdm_graph *G, void *dst, const void *src, size_t bytes) {
    if (!bytes) return cudaSuccess;
    const void *p = G->stage.put(src, bytes);
    return cudaMemcpyAsync(dst, p ? p : src, bytes, cudaMemcpyHostToDevice, G->stream);
}
}  // namespace asdm
