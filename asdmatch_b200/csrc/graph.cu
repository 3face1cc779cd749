// Data-graph upload: CSR copy, (label, id)-order check and the per-vertex
// label-run index, built on the device.  The host adds the vertices-by-label
// grouping (Graph::loadGraphFromTextFile, relation/graph.cpp:132-144) with a
// counting sort, since it needs the id order preserved inside each label.
#include <algorithm>
#include <memory>

#include "device.cuh"

namespace asdm {

int device_setup(int *device, int *num_sms) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return fail(ASDM_ERR_CUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
    ASDM_CUDA(cudaGetDevice(device));
    ASDM_CUDA(cudaDeviceGetAttribute(num_sms, cudaDevAttrMultiProcessorCount, *device));
    // keep freed stream-ordered allocations in the pool instead of returning
    // them to the driver at every synchronisation
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, *device) == cudaSuccess) {
        uint64_t keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    return ASDM_OK;
}

namespace {

// Warp per vertex: checks (label, id) order and ids/labels in range; counts
// label runs.
__global__ void check_and_count_runs(DevGraph g, uint32_t *__restrict__ runs, uint32_t *__restrict__ bad) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t v = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); v < g.n; v += nwarps) {
        const uint32_t b = g.off[v], e = g.off[v + 1];
        uint32_t count = 0;
        for (uint32_t base = b; base < e; base += 32) {
            const uint32_t i = base + lane;
            bool boundary = false, ok = true;
            if (i < e) {
                const uint32_t x = g.nbr[i];
                if (x >= g.n) {
                    ok = false;
                } else {
                    const uint32_t lx = g.lab[x];
                    if (i == b) {
                        boundary = true;
                    } else {
                        const uint32_t y = g.nbr[i - 1];
                        const uint32_t ly = y < g.n ? g.lab[y] : 0xFFFFFFFFu;
                        boundary = lx != ly;
                        ok = (ly < lx) || (ly == lx && y < x);
                    }
                    ok = ok && x != v;
                }
            }
            count += __popc(__ballot_sync(0xffffffffu, boundary));
            if (__any_sync(0xffffffffu, !ok) && lane == 0) atomicExch(bad, 1u);
        }
        if (lane == 0) runs[v] = count;
    }
}

__global__ void write_runs(DevGraph g, const uint64_t *__restrict__ run_pos, uint32_t *__restrict__ run_lab,
                           uint32_t *__restrict__ run_start) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t v = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); v < g.n; v += nwarps) {
        const uint32_t b = g.off[v], e = g.off[v + 1];
        uint64_t out = run_pos[v];
        for (uint32_t base = b; base < e; base += 32) {
            const uint32_t i = base + lane;
            bool boundary = false;
            uint32_t lx = 0;
            if (i < e) {
                lx = g.lab[g.nbr[i]];
                boundary = (i == b) || lx != g.lab[g.nbr[i - 1]];
            }
            const uint32_t mask = __ballot_sync(0xffffffffu, boundary);
            if (boundary) {
                const uint64_t r = out + __popc(mask & ((1u << lane) - 1));
                run_lab[r] = lx;
                run_start[r] = i;
            }
            out += __popc(mask);
        }
    }
}

__global__ void nbr_ranks(DevGraph g, uint32_t *__restrict__ rank) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < g.m2; k += (uint64_t)gridDim.x * blockDim.x)
        rank[k] = g.pos_in_label[g.nbr[k]];
}

// Per vertex, stored at its place in the vertices-by-label order: degree and
// a mask with bit (l mod 32) set for every label l among its neighbours.
__global__ void rank_infos(DevGraph g, uint2 *__restrict__ info) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < g.n; v += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t mask = 0;
        for (uint32_t r = g.run_off[v]; r < g.run_off[v + 1]; ++r) mask |= 1u << (g.run_lab[r] & 31u);
        info[g.vbl_off[g.lab[v]] + g.pos_in_label[v]] = make_uint2(g.off[v + 1] - g.off[v], mask);
    }
}

// Dense label-run table: one thread per (vertex, label) entry.
__global__ void write_lab_pos(DevGraph g, uint32_t *__restrict__ lab_pos) {
    const uint32_t stride = g.nlabels + 1;
    const uint64_t total = (uint64_t)g.n * stride;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(t / stride), l = (uint32_t)(t - (uint64_t)v * stride);
        uint32_t lo = g.run_off[v], hi = g.run_off[v + 1];
        const uint32_t end = hi;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (g.run_lab[mid] < l) lo = mid + 1; else hi = mid;
        }
        lab_pos[t] = lo < end ? g.run_start[lo] : g.off[v + 1];
    }
}

__global__ void narrow_u64(const uint64_t *__restrict__ in, uint32_t *__restrict__ out, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = (uint32_t)in[i];
}

}  // namespace
}  // namespace asdm

using namespace asdm;

extern "C" int asdm_graph_upload(const uint32_t *offsets, const uint32_t *nbrs, const uint32_t *labels, uint32_t n,
                                 uint64_t m2, uint32_t nlabels, asdm_graph **out) {
    clear_error();
    if (!offsets || !labels || !out || (m2 && !nbrs)) return fail(ASDM_ERR_INVALID, "null argument");
    if (n == 0 || n >= 0xFFFFFFFFu) return fail(ASDM_ERR_INVALID, "vertex count %u unsupported", n);
    if (m2 >= 0xFFFFFFFFull) return fail(ASDM_ERR_INVALID, "edge count too large for 32-bit offsets");
    if (offsets[0] != 0 || (uint64_t)offsets[n] != m2) return fail(ASDM_ERR_INVALID, "offsets do not span 0..m2");
    uint32_t max_deg = 0;
    for (uint32_t v = 0; v < n; ++v) {
        if (offsets[v + 1] < offsets[v]) return fail(ASDM_ERR_INVALID, "offsets not monotone at %u", v);
        max_deg = std::max(max_deg, offsets[v + 1] - offsets[v]);
        if (labels[v] >= nlabels) return fail(ASDM_ERR_INVALID, "label of vertex %u >= nlabels", v);
    }
    auto g = std::make_unique<asdm_graph>();
    ASDM_TRY(device_setup(&g->device, &g->num_sms));
    ASDM_CUDA(cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking));
    cudaStream_t s = g->stream;
    // host: vertices grouped by label (stable), rank inside the label
    g->h_vbl_off.assign((size_t)nlabels + 1, 0);
    for (uint32_t v = 0; v < n; ++v) g->h_vbl_off[labels[v] + 1]++;
    for (uint32_t l = 0; l < nlabels; ++l) g->h_vbl_off[l + 1] += g->h_vbl_off[l];
    std::vector<uint32_t> vbl(n), pos(n);
    {
        std::vector<uint32_t> fill(g->h_vbl_off.begin(), g->h_vbl_off.end() - 1);
        for (uint32_t v = 0; v < n; ++v) {
            uint32_t l = labels[v];
            pos[v] = fill[l] - g->h_vbl_off[l];
            vbl[fill[l]++] = v;
        }
    }
    g->max_deg = max_deg;
    // one backing allocation for the fixed-size arrays
    const uint64_t fixed = (uint64_t)(n + 1) + m2 + n + n + (nlabels + 1) + n + (n + 1) + m2 + 1 + 2ull * n;
    ASDM_CUDA(cudaMalloc((void **)&g->buf, fixed * sizeof(uint32_t)));
    uint32_t *p = g->buf;
    uint32_t *d_off = p; p += n + 1;
    uint32_t *d_nbr = p; p += m2;
    uint32_t *d_lab = p; p += n;
    uint32_t *d_pos = p; p += n;
    uint32_t *d_vbl_off = p; p += nlabels + 1;
    uint32_t *d_vbl = p; p += n;
    uint32_t *d_run_off = p; p += n + 1;
    uint32_t *d_nbr_rank = p; p += m2;
    if ((p - g->buf) & 1) ++p;  // 8-byte alignment for the uint2 array
    uint2 *d_rank_info = reinterpret_cast<uint2 *>(p);
    ASDM_CUDA(cudaMemcpyAsync(d_off, offsets, (n + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    if (m2) ASDM_CUDA(cudaMemcpyAsync(d_nbr, nbrs, m2 * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    ASDM_CUDA(cudaMemcpyAsync(d_lab, labels, n * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    ASDM_CUDA(cudaMemcpyAsync(d_pos, pos.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    ASDM_CUDA(cudaMemcpyAsync(d_vbl_off, g->h_vbl_off.data(), (nlabels + 1) * sizeof(uint32_t),
                              cudaMemcpyHostToDevice, s));
    ASDM_CUDA(cudaMemcpyAsync(d_vbl, vbl.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, s));
    DevGraph &d = g->d;
    d.n = n;
    d.nlabels = nlabels;
    d.m2 = m2;
    d.off = d_off;
    d.nbr = d_nbr;
    d.lab = d_lab;
    d.pos_in_label = d_pos;
    d.vbl_off = d_vbl_off;
    d.vbl = d_vbl;
    d.run_off = d_run_off;
    // label runs
    uint32_t *runs = nullptr, *bad = nullptr;
    uint64_t *run_pos = nullptr;
    ASDM_TRY(dalloc(&runs, n, s));
    ASDM_TRY(dalloc(&bad, 1, s));
    ASDM_TRY(dalloc(&run_pos, (uint64_t)n + 1, s));
    ASDM_CUDA(cudaMemsetAsync(bad, 0, sizeof(uint32_t), s));
    const unsigned blocks = (unsigned)std::min<uint64_t>((n + 7) / 8, (uint64_t)g->num_sms * 16);
    check_and_count_runs<<<blocks, 256, 0, s>>>(d, runs, bad);
    ::asdm::count_launch();
    ASDM_CUDA(cudaGetLastError());
    ASDM_TRY(scan_exclusive_u32(runs, run_pos, n, true, s));
    uint32_t h_bad = 0;
    uint64_t nruns = 0;
    ASDM_CUDA(cudaMemcpyAsync(&h_bad, bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    ASDM_CUDA(cudaMemcpyAsync(&nruns, run_pos + n, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
    ASDM_CUDA(cudaStreamSynchronize(s));
    if (h_bad) {
        dfree(runs, s); dfree(bad, s); dfree(run_pos, s);
        cudaStreamSynchronize(s);
        cudaFree(g->buf);
        cudaStreamDestroy(g->stream);
        return fail(ASDM_ERR_INVALID, "adjacency lists must be sorted by (label, id), loop-free and in range");
    }
    uint32_t *run_buf = nullptr;
    ASDM_CUDA(cudaMalloc((void **)&run_buf, std::max<uint64_t>(2 * nruns, 1) * sizeof(uint32_t)));
    uint32_t *d_run_lab = run_buf, *d_run_start = run_buf + nruns;
    narrow_u64<<<(unsigned)std::min<uint64_t>((n + 256) / 256, 4096), 256, 0, s>>>(run_pos, d_run_off, (uint64_t)n + 1);
    ::asdm::count_launch();
    write_runs<<<blocks, 256, 0, s>>>(d, run_pos, d_run_lab, d_run_start);
    ::asdm::count_launch();
    ASDM_CUDA(cudaGetLastError());
    d.run_lab = d_run_lab;
    d.run_start = d_run_start;
    d.nruns = nruns;
    if (m2) {
        nbr_ranks<<<(unsigned)std::min<uint64_t>((m2 + 255) / 256, (uint64_t)g->num_sms * 32), 256, 0, s>>>(d, d_nbr_rank);
        ::asdm::count_launch();
    }
    rank_infos<<<(unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)g->num_sms * 32), 256, 0, s>>>(d, d_rank_info);
    ::asdm::count_launch();
    ASDM_CUDA(cudaGetLastError());
    d.nbr_rank = d_nbr_rank;
    d.rank_info = d_rank_info;
    const uint64_t lp_words = (uint64_t)n * (nlabels + 1);
    if (n && lp_words * sizeof(uint32_t) <= kLabPosCap) {
        uint32_t *lp = nullptr;
        if (cudaMalloc((void **)&lp, lp_words * sizeof(uint32_t)) == cudaSuccess) {
            write_lab_pos<<<(unsigned)std::min<uint64_t>((lp_words + 255) / 256, (uint64_t)g->num_sms * 32), 256, 0, s>>>(
                d, lp);
            ::asdm::count_launch();
            ASDM_CUDA(cudaGetLastError());
            d.lab_pos = lp;
        } else {
            cudaGetLastError();  // no room: label runs are searched instead
        }
    }
    dfree(runs, s); dfree(bad, s); dfree(run_pos, s);
    ASDM_CUDA(cudaStreamSynchronize(s));
    // the run arrays live in their own allocation; remember it for free()
    g->d.run_lab = d_run_lab;
    *out = g.release();
    return ASDM_OK;
}

extern "C" int asdm_graph_free(asdm_graph *g) {
    if (!g) return ASDM_OK;
    cudaStreamSynchronize(g->stream);
    cudaFree((void *)g->d.run_lab);  // run_lab heads the run allocation
    if (g->d.lab_pos) cudaFree((void *)g->d.lab_pos);
    cudaFree(g->buf);
    cudaStreamDestroy(g->stream);
    delete g;
    return ASDM_OK;
}
