// K1-K3: the CFL candidate space on the device.
//
// Restates CandidateSpace::buildCandCFL (relation/candidate_space.cpp:550-721)
// as the set computation it performs.  For every query vertex u a state word
// per data vertex of u's label holds bit 31 = "passes the label, degree and
// NLC filter" (K1, nlcValid at utility/utils.cpp:30-40) and bit b = "adjacent
// to the storage of u's b-th query neighbour p" (K2).  The storage S(p) that
// the reference scans for p is the top-down candidate set Ctd(p) plus data
// vertex 0 whenever Ctd(p) is smaller than |V_l(p)|: candidateSet[p] is
// resized to |V_l(p)| up front (:555-559), its zero-initialised tail is
// iterated by the range-for loops (:588, :623, :661), and pruned entries stay
// in it until the compaction at :692-703.  Hence
//     Ctd(root) = F(root),   Ctd(u) = F(u) ∩ ⋂_{p ∈ before(u)} N_l(u)(S(p)),
//     C(u) = F(u) ∩ ⋂_{p ∈ N_q(u)} N_l(u)(S(p)),
// computed wave by wave along the CFL BFS order (a vertex's wave is one more
// than the latest wave among its earlier neighbours).  The marking is an
// atomicOr of bit b, so the order of the scans inside a wave does not matter.
// K3 compacts each C(u) in id order and builds the candidate edges
// (buildCandidateEdge(false), :458-487) as CSR lists of indices into C(u2).
#include <algorithm>
#include <memory>
#include <queue>

#include "cs.cuh"

namespace asdm {
namespace {

constexpr uint32_t kFBit = 0x80000000u;
constexpr int kBlock = 256;
constexpr uint32_t kLongRun = 32;

__device__ __forceinline__ uint32_t find_segment(const uint64_t *__restrict__ prefix, uint32_t nseg, uint64_t item) {
    // last s with prefix[s] <= item (prefix has nseg + 1 entries, non-decreasing)
    uint32_t lo = 0, hi = nseg;
    while (hi - lo > 1) {
        uint32_t mid = (lo + hi) >> 1;
        if (prefix[mid] <= item) lo = mid; else hi = mid;
    }
    return lo;
}

// ---- K1: label + degree + NLC filter --------------------------------------
// One segment per (query, query vertex) of a batch.
struct FilterArgs {
    DevGraph g;
    uint32_t *st;
    const uint64_t *seg;      // nseg + 1 prefix of |V_l(u)|
    const uint32_t *lbase;    // vbl_off[l(u)]
    const uint32_t *qdeg;     // deg(u)
    const uint32_t *qnlc;     // (label, count) pairs
    const uint32_t *qnlc_off; // nseg + 1
    uint32_t nq;              // number of segments
    uint32_t *fcount;         // |F(u)|
};

__global__ void __launch_bounds__(kBlock) k1_filter(FilterArgs a) {
    const uint64_t *seg = a.seg;
    const uint64_t total = seg[a.nq];
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total; base += stride) {
        const uint64_t item = base + lane;
        bool pass = false;
        uint32_t u = 0xFFFFFFFFu;
        if (item < total) {
            u = find_segment(seg, a.nq, item);
            const uint32_t i = (uint32_t)(item - seg[u]);
            const uint32_t v = a.g.vbl[a.lbase[u] + i];
            pass = (a.g.off[v + 1] - a.g.off[v]) >= a.qdeg[u];
            for (uint32_t k = a.qnlc_off[u]; pass && k < a.qnlc_off[u + 1]; ++k) {
                uint32_t b, e;
                label_run(a.g, v, a.qnlc[2 * k], b, e);
                pass = (e - b) >= a.qnlc[2 * k + 1];
            }
            a.st[item] = pass ? kFBit : 0u;
        }
        const uint32_t key = pass ? u : 0xFFFFFFFFu;
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        if (pass && (__ffs(peers) - 1) == (int)lane) atomicAdd(&a.fcount[u], (uint32_t)__popc(peers));
    }
}

// ---- K2: neighbour marking passes -------------------------------------------
struct PassDesc {
    const uint32_t *src;  // storage S(p): vertex ids
    uint32_t *st;         // state words of u (indexed by rank inside l(u))
    uint32_t label;       // l(u)
    uint32_t mask;        // bit of p among u's query neighbours
};

__device__ __forceinline__ void mark(const DevGraph &g, uint32_t *st, uint32_t k, uint32_t mask) {
    const uint32_t i = g.pos_in_label[g.nbr[k]];
    const uint32_t s = st[i];
    if ((s & kFBit) && !(s & mask)) atomicOr(&st[i], mask);
}

__global__ void __launch_bounds__(kBlock) k2_pass(DevGraph g, const PassDesc *__restrict__ passes,
                                                  const uint64_t *__restrict__ prefix, uint32_t npass,
                                                  unsigned long long *__restrict__ elems) {
    const uint64_t total = prefix[npass];
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t scanned = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total; base += stride) {
        const uint64_t item = base + lane;
        uint32_t b = 0, e = 0, mask = 0;
        uint32_t *st = nullptr;
        if (item < total) {
            const uint32_t p = find_segment(prefix, npass, item);
            const PassDesc d = passes[p];
            const uint32_t w = d.src[item - prefix[p]];
            label_run(g, w, d.label, b, e);
            st = d.st;
            mask = d.mask;
        }
        scanned += e - b;
        const bool coop = (e - b) > kLongRun;
        uint32_t todo = __ballot_sync(0xffffffffu, coop);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint32_t bb = __shfl_sync(0xffffffffu, b, src), ee = __shfl_sync(0xffffffffu, e, src);
            const uint32_t mm = __shfl_sync(0xffffffffu, mask, src);
            uint32_t *ss = (uint32_t *)__shfl_sync(0xffffffffu, (unsigned long long)st, src);
            for (uint32_t k = bb + lane; k < ee; k += 32) mark(g, ss, k, mm);
        }
        if (!coop)
            for (uint32_t k = b; k < e; ++k) mark(g, st, k, mask);
    }
    for (int o = 16; o; o >>= 1) scanned += __shfl_xor_sync(0xffffffffu, scanned, o);
    if (lane == 0 && scanned) atomicAdd(elems, (unsigned long long)scanned);
}

// ---- K3a: order-preserving compaction of state words into vertex lists ----
constexpr int kItems = 8;
constexpr int kTile = kBlock * kItems;

struct CompDesc {
    const uint32_t *st;
    uint32_t *out;        // vertex ids, capacity len
    uint32_t len;         // |V_l(u)|
    uint32_t need;        // required bits
    uint32_t lbase;       // vbl_off[l(u)]
    uint32_t phantom;     // append data vertex 0 when fewer than len survive
};

__global__ void __launch_bounds__(kBlock) k3_count(const CompDesc *__restrict__ segs, const uint64_t *__restrict__ tile_first,
                                                   uint32_t nseg, uint32_t *__restrict__ tile_cnt) {
    const uint32_t t = blockIdx.x;
    const uint32_t sidx = find_segment(tile_first, nseg, t);
    const CompDesc d = segs[sidx];
    const uint64_t first = (uint64_t)(t - tile_first[sidx]) * kTile;
    uint32_t c = 0;
    for (uint32_t k = threadIdx.x; k < kTile; k += kBlock) {
        const uint64_t i = first + k;
        if (i < d.len && (d.st[i] & d.need) == d.need) ++c;
    }
    __shared__ uint32_t wsum[kBlock / 32];
    for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t s = 0;
        for (int w = 0; w < kBlock / 32; ++w) s += wsum[w];
        tile_cnt[t] = s;
    }
}

__global__ void __launch_bounds__(kBlock) k3_write(const CompDesc *__restrict__ segs, const uint64_t *__restrict__ tile_first,
                                                   uint32_t nseg, const uint64_t *__restrict__ tile_pos,
                                                   const uint32_t *__restrict__ vbl, uint32_t *__restrict__ seg_count) {
    const uint32_t t = blockIdx.x;
    const uint32_t sidx = find_segment(tile_first, nseg, t);
    const CompDesc d = segs[sidx];
    const uint64_t first = (uint64_t)(t - tile_first[sidx]) * kTile;
    const uint64_t my = first + (uint64_t)threadIdx.x * kItems;
    uint32_t flags = 0, c = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint64_t i = my + k;
        if (i < d.len && (d.st[i] & d.need) == d.need) { flags |= 1u << k; ++c; }
    }
    // block exclusive scan of c
    __shared__ uint32_t wsum[kBlock / 32];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = c;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < kBlock / 32 ? wsum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kBlock / 32) wsum[lane] = w;
    }
    __syncthreads();
    uint64_t pos = (tile_pos[t] - tile_pos[tile_first[sidx]]) + (warp ? wsum[warp - 1] : 0) + x - c;
#pragma unroll
    for (int k = 0; k < kItems; ++k)
        if (flags & (1u << k)) d.out[pos++] = vbl[d.lbase + (uint32_t)(my + k)];
    // the last tile of a segment records the segment size
    if (threadIdx.x == 0 && t + 1 == tile_first[sidx + 1]) {
        uint32_t size = (uint32_t)(tile_pos[t + 1] - tile_pos[tile_first[sidx]]);
        if (d.phantom && size < d.len) d.out[size++] = 0;  // the reference's zero-filled storage tail
        seg_count[sidx] = size;
    }
}

// ---- K3b: candidate edges ---------------------------------------------------
struct EdgeDesc {
    const uint32_t *cand_u;  // C(u)
    const uint32_t *map_u2;  // rank in l(u2) -> index in C(u2) or kNone
    uint32_t ncand_u;
    uint32_t label_u2;
};

__global__ void __launch_bounds__(kBlock) k3_scatter_map(const uint32_t *const *__restrict__ cands,
                                                         const uint64_t *__restrict__ cprefix, uint32_t nseg,
                                                         uint32_t *const *__restrict__ maps,
                                                         const uint32_t *__restrict__ pos_in_label) {
    const uint64_t total = cprefix[nseg];
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t u = find_segment(cprefix, nseg, i);
        const uint32_t j = (uint32_t)(i - cprefix[u]);
        maps[u][pos_in_label[cands[u][j]]] = j;
    }
}

template <bool kFill>
__global__ void __launch_bounds__(kBlock) k3_edges(DevGraph g, const EdgeDesc *__restrict__ edges,
                                                   const uint64_t *__restrict__ item_base, uint32_t nedges,
                                                   uint32_t *__restrict__ cnt, const uint64_t *__restrict__ wpos,
                                                   uint32_t *__restrict__ elist, unsigned long long *__restrict__ elems) {
    const uint64_t total = item_base[nedges];
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t scanned = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total; base += stride) {
        const uint64_t item = base + lane;
        uint32_t b = 0, e = 0;
        const uint32_t *map = nullptr;
        if (item < total) {
            const uint32_t ei = find_segment(item_base, nedges, item);
            const EdgeDesc d = edges[ei];
            const uint32_t i = (uint32_t)(item - item_base[ei]);
            if (i < d.ncand_u) label_run(g, d.cand_u[i], d.label_u2, b, e);
            map = d.map_u2;
        }
        scanned += e - b;
        const bool coop = (e - b) > kLongRun;
        uint32_t mine = 0;
        uint64_t out = kFill && item < total ? wpos[item] : 0;
        uint32_t todo = __ballot_sync(0xffffffffu, coop);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint32_t bb = __shfl_sync(0xffffffffu, b, src), ee = __shfl_sync(0xffffffffu, e, src);
            const uint32_t *mm = (const uint32_t *)__shfl_sync(0xffffffffu, (unsigned long long)map, src);
            uint64_t o = __shfl_sync(0xffffffffu, out, src);
            uint32_t c = 0;
            for (uint32_t k0 = bb; k0 < ee; k0 += 32) {
                const uint32_t k = k0 + lane;
                uint32_t idx = kNone;
                if (k < ee) idx = mm[g.pos_in_label[g.nbr[k]]];
                const uint32_t hit = __ballot_sync(0xffffffffu, idx != kNone);
                if (kFill && idx != kNone) elist[o + __popc(hit & ((1u << lane) - 1))] = idx;
                o += __popc(hit);
                c += __popc(hit);
            }
            if ((int)lane == src) mine = c;
        }
        if (!coop) {
            for (uint32_t k = b; k < e; ++k) {
                const uint32_t idx = map[g.pos_in_label[g.nbr[k]]];
                if (idx != kNone) {
                    if (kFill) elist[out++] = idx;
                    ++mine;
                }
            }
        }
        if (!kFill && item < total) cnt[item] = mine;
    }
    if (!kFill) {
        for (int o = 16; o; o >>= 1) scanned += __shfl_xor_sync(0xffffffffu, scanned, o);
        if (lane == 0 && scanned) atomicAdd(elems, (unsigned long long)scanned);
    }
}

__global__ void k3_offsets(const uint64_t *__restrict__ item_base, uint32_t nedges, const uint64_t *__restrict__ wpos,
                           uint32_t *__restrict__ eoff, uint64_t *__restrict__ edge_start, uint32_t *__restrict__ bad) {
    const uint64_t total = item_base[nedges];
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t ei = find_segment(item_base, nedges, i);
        const uint64_t rel = wpos[i] - wpos[item_base[ei]];
        if (rel > 0xFFFFFFFFull) atomicExch(bad, 1u);
        eoff[i] = (uint32_t)rel;
        if (i == item_base[ei]) edge_start[ei] = wpos[i];
    }
}

unsigned grid_for(uint64_t items, int num_sms) {
    uint64_t blocks = (items + kBlock - 1) / kBlock;
    return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(blocks, (uint64_t)num_sms * 32));
}

// Runs one compaction over the given segments; returns per-segment sizes.
int compact(asdm_graph *G, const std::vector<CompDesc> &segs, std::vector<uint32_t> &sizes) {
    cudaStream_t s = G->stream;
    const uint32_t nseg = (uint32_t)segs.size();
    sizes.assign(nseg, 0);
    if (nseg == 0) return ASDM_OK;
    std::vector<uint64_t> tile_first(nseg + 1, 0);
    for (uint32_t i = 0; i < nseg; ++i) tile_first[i + 1] = tile_first[i] + (segs[i].len + kTile - 1) / kTile;
    const uint64_t ntiles = tile_first[nseg];
    if (ntiles == 0) return ASDM_OK;
    CompDesc *d_segs = nullptr;
    uint64_t *d_tf = nullptr, *d_pos = nullptr;
    uint32_t *d_cnt = nullptr, *d_sc = nullptr;
    ASDM_TRY(dalloc(&d_segs, nseg, s));
    ASDM_TRY(dalloc(&d_tf, nseg + 1, s));
    ASDM_TRY(dalloc(&d_cnt, ntiles, s));
    ASDM_TRY(dalloc(&d_pos, ntiles + 1, s));
    ASDM_TRY(dalloc(&d_sc, nseg, s));
    ASDM_CUDA(cudaMemcpyAsync(d_segs, segs.data(), nseg * sizeof(CompDesc), cudaMemcpyHostToDevice, s));
    ASDM_CUDA(cudaMemcpyAsync(d_tf, tile_first.data(), (nseg + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    ASDM_CUDA(cudaMemsetAsync(d_sc, 0, nseg * sizeof(uint32_t), s));
    k3_count<<<(unsigned)ntiles, kBlock, 0, s>>>(d_segs, d_tf, nseg, d_cnt);
    ::asdm::count_launch();
    ASDM_CUDA(cudaGetLastError());
    ASDM_TRY(scan_exclusive_u32(d_cnt, d_pos, ntiles, true, s));
    k3_write<<<(unsigned)ntiles, kBlock, 0, s>>>(d_segs, d_tf, nseg, d_pos, G->d.vbl, d_sc);
    ::asdm::count_launch();
    ASDM_CUDA(cudaGetLastError());
    ASDM_CUDA(cudaMemcpyAsync(sizes.data(), d_sc, nseg * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    ASDM_CUDA(cudaStreamSynchronize(s));
    dfree(d_segs, s); dfree(d_tf, s); dfree(d_cnt, s); dfree(d_pos, s); dfree(d_sc, s);
    return ASDM_OK;
}

int run_passes(asdm_graph *G, const std::vector<PassDesc> &passes, const std::vector<uint64_t> &lens,
               unsigned long long *d_elems) {
    cudaStream_t s = G->stream;
    const uint32_t np = (uint32_t)passes.size();
    if (np == 0) return ASDM_OK;
    std::vector<uint64_t> prefix(np + 1, 0);
    for (uint32_t i = 0; i < np; ++i) prefix[i + 1] = prefix[i] + lens[i];
    if (prefix[np] == 0) return ASDM_OK;
    PassDesc *d_p = nullptr;
    uint64_t *d_prefix = nullptr;
    ASDM_TRY(dalloc(&d_p, np, s));
    ASDM_TRY(dalloc(&d_prefix, np + 1, s));
    ASDM_CUDA(cudaMemcpyAsync(d_p, passes.data(), np * sizeof(PassDesc), cudaMemcpyHostToDevice, s));
    ASDM_CUDA(cudaMemcpyAsync(d_prefix, prefix.data(), (np + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    k2_pass<<<grid_for(prefix[np], G->num_sms), kBlock, 0, s>>>(G->d, d_p, d_prefix, np, d_elems);
    ::asdm::count_launch();
    ASDM_CUDA(cudaGetLastError());
    dfree(d_p, s);
    dfree(d_prefix, s);
    return ASDM_OK;
}

struct Scratch {
    cudaStream_t s;
    std::vector<void *> ptrs;
    ~Scratch() {
        for (void *p : ptrs) cudaFreeAsync(p, s);
    }
    template <typename T>
    int alloc(T **p, uint64_t n) {
        int rc = dalloc(p, n, s);
        if (rc == ASDM_OK) ptrs.push_back((void *)*p);
        return rc;
    }
    template <typename T>
    int upload(T **p, const std::vector<T> &h) {
        ASDM_TRY(alloc(p, h.size()));
        if (!h.empty()) ASDM_CUDA(cudaMemcpyAsync(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, s));
        return ASDM_OK;
    }
};

// Host-side plan of one query's CFL build.
struct QPlan {
    asdm_cs *cs;
    uint32_t seg0;                  // first segment (query vertex 0)
    bool empty = false;
    std::vector<uint32_t> lsize, lbase, rank, order, wave;
};

}  // namespace

// Candidate spaces of a group of queries on one graph, one launch per phase
// for the whole group.  Every phase is the single-query computation applied
// to all (query, query vertex) segments at once.
int build_batch(const std::vector<asdm_cs *> &group) {
    if (group.empty()) return ASDM_OK;
    asdm_graph *G = group[0]->g;
    const DevGraph &g = G->d;
    cudaStream_t s = G->stream;
    Scratch scr{s, {}};
    cudaEvent_t ev0, ev1;
    ASDM_CUDA(cudaEventCreate(&ev0));
    ASDM_CUDA(cudaEventCreate(&ev1));
    ASDM_CUDA(cudaEventRecord(ev0, s));
    const uint32_t Q = (uint32_t)group.size();
    std::vector<QPlan> P(Q);
    uint32_t nseg = 0;
    for (uint32_t qi = 0; qi < Q; ++qi) {
        QPlan &qp = P[qi];
        qp.cs = group[qi];
        const QueryGraph &q = qp.cs->q;
        qp.seg0 = nseg;
        nseg += q.n;
        qp.lsize.assign(q.n, 0);
        qp.lbase.assign(q.n, 0);
        for (uint32_t u = 0; u < q.n; ++u) {
            const uint32_t l = q.lab[u];
            if (l < g.nlabels) {
                qp.lbase[u] = G->h_vbl_off[l];
                qp.lsize[u] = G->h_vbl_off[l + 1] - G->h_vbl_off[l];
            }
        }
    }
    // segment tables
    std::vector<uint64_t> seg(nseg + 1, 0);
    std::vector<uint32_t> lbase(nseg), qdeg(nseg), qnlc, qnlc_off(nseg + 1, 0);
    for (const QPlan &qp : P) {
        const QueryGraph &q = qp.cs->q;
        for (uint32_t u = 0; u < q.n; ++u) {
            const uint32_t sg = qp.seg0 + u;
            seg[sg + 1] = seg[sg] + qp.lsize[u];
            lbase[sg] = qp.lbase[u];
            qdeg[sg] = q.deg(u);
            for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                const uint32_t l = q.lab[q.nbr[e]];
                if (qnlc.size() > 2 * qnlc_off[sg] && qnlc[qnlc.size() - 2] == l) qnlc.back()++;
                else { qnlc.push_back(l); qnlc.push_back(1); }
            }
            qnlc_off[sg + 1] = (uint32_t)(qnlc.size() / 2);
        }
    }
    uint32_t *st = nullptr, *d_fcount = nullptr, *d_lbase = nullptr, *d_qdeg = nullptr, *d_qnlc = nullptr,
             *d_qnlc_off = nullptr;
    uint64_t *d_seg = nullptr;
    unsigned long long *d_elems = nullptr;
    ASDM_TRY(scr.alloc(&st, seg[nseg]));
    ASDM_TRY(scr.upload(&d_seg, seg));
    ASDM_TRY(scr.upload(&d_lbase, lbase));
    ASDM_TRY(scr.upload(&d_qdeg, qdeg));
    if (qnlc.empty()) qnlc.push_back(0);
    ASDM_TRY(scr.upload(&d_qnlc, qnlc));
    ASDM_TRY(scr.upload(&d_qnlc_off, qnlc_off));
    ASDM_TRY(scr.alloc(&d_fcount, nseg));
    ASDM_TRY(scr.alloc(&d_elems, 2));
    ASDM_CUDA(cudaMemsetAsync(d_fcount, 0, nseg * sizeof(uint32_t), s));
    ASDM_CUDA(cudaMemsetAsync(d_elems, 0, 2 * sizeof(unsigned long long), s));
    if (seg[nseg]) {
        FilterArgs fa{g, st, d_seg, d_lbase, d_qdeg, d_qnlc, d_qnlc_off, nseg, d_fcount};
        k1_filter<<<grid_for(seg[nseg], G->num_sms), kBlock, 0, s>>>(fa);
        ::asdm::count_launch();
        ASDM_CUDA(cudaGetLastError());
    }
    std::vector<uint32_t> fcount(nseg, 0);
    ASDM_CUDA(cudaMemcpyAsync(fcount.data(), d_fcount, nseg * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    ASDM_CUDA(cudaStreamSynchronize(s));

    uint32_t maxwave = 0;
    for (QPlan &qp : P) {
        asdm_cs &cs = *qp.cs;
        const QueryGraph &q = cs.q;
        const uint32_t nq = q.n;
        // Root: the three smallest |V_l(u)|/deg(u) kept in a max-heap, then the
        // first strict minimum of |F(u)|/deg(u) in pop order (selectCFLRoot,
        // relation/candidate_space.cpp:723-763; same container and comparator).
        auto cmp = [](const std::pair<uint32_t, double> &x, const std::pair<uint32_t, double> &y) {
            return x.second < y.second;
        };
        std::priority_queue<std::pair<uint32_t, double>, std::vector<std::pair<uint32_t, double>>, decltype(cmp)> pq(cmp);
        for (uint32_t u = 0; u < nq; ++u) pq.emplace(u, qp.lsize[u] / (double)q.deg(u));
        while (pq.size() > 3) pq.pop();
        uint32_t root = 0;
        double best = g.n;
        while (!pq.empty()) {
            const uint32_t u = pq.top().first;
            pq.pop();
            const double score = fcount[qp.seg0 + u] / (double)q.deg(u);
            if (score < best) { best = score; root = u; }
        }
        cs.root = root;
        // BFS levels with discovery order over (label,id)-sorted query
        // neighbours (buildCFLBFSTree, :765-816); rank = position in that order
        qp.rank.assign(nq, kNone);
        qp.order.clear();
        std::vector<uint32_t> frontier{root};
        qp.rank[root] = 0;
        uint32_t r = 1;
        while (!frontier.empty()) {
            std::vector<uint32_t> next;
            for (uint32_t u : frontier) {
                qp.order.push_back(u);
                for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                    const uint32_t w = q.nbr[e];
                    if (qp.rank[w] == kNone) { qp.rank[w] = r++; next.push_back(w); }
                }
            }
            frontier.swap(next);
        }
        cs.bfs_order = qp.order;
        cs.ncand.assign(nq, 0);
        cs.cand_base.assign(nq + 1, 0);
        cs.nonempty = false;
        qp.empty = qp.order.size() != nq;  // unreached query vertices get no candidates
        for (uint32_t u = 0; u < nq; ++u) qp.empty |= fcount[qp.seg0 + u] == 0;
        qp.wave.assign(nq, 0);
        if (qp.empty) continue;
        for (uint32_t u : qp.order) {
            for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                const uint32_t p = q.nbr[e];
                if (qp.rank[p] < qp.rank[u]) qp.wave[u] = std::max(qp.wave[u], qp.wave[p] + 1);
            }
            maxwave = std::max(maxwave, qp.wave[u]);
        }
    }
    // storage S(u) = Ctd(u) (+ vertex 0), capacity |V_l(u)| + 1 per segment
    std::vector<uint64_t> sbase(nseg + 1, 0);
    for (const QPlan &qp : P)
        for (uint32_t u = 0; u < qp.cs->q.n; ++u) sbase[qp.seg0 + u + 1] = sbase[qp.seg0 + u] + qp.lsize[u] + 1;
    uint32_t *sbuf = nullptr;
    ASDM_TRY(scr.alloc(&sbuf, sbase[nseg]));
    std::vector<uint64_t> slen(nseg, 0);
    for (uint32_t w = 0; w <= maxwave; ++w) {
        std::vector<PassDesc> passes;
        std::vector<uint64_t> lens;
        std::vector<CompDesc> segs;
        std::vector<uint32_t> seg_ids;
        for (const QPlan &qp : P) {
            if (qp.empty) continue;
            const QueryGraph &q = qp.cs->q;
            for (uint32_t u : qp.order) {
                if (qp.wave[u] != w) continue;
                const uint32_t su = qp.seg0 + u;
                uint32_t need = kFBit;
                for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                    const uint32_t p = q.nbr[e];
                    if (qp.rank[p] >= qp.rank[u]) continue;
                    const uint32_t bit = 1u << (e - q.off[u]);
                    need |= bit;
                    passes.push_back(PassDesc{sbuf + sbase[qp.seg0 + p], st + seg[su], q.lab[u], bit});
                    lens.push_back(slen[qp.seg0 + p]);
                }
                segs.push_back(CompDesc{st + seg[su], sbuf + sbase[su], qp.lsize[u], need, qp.lbase[u], 1});
                seg_ids.push_back(su);
            }
        }
        ASDM_TRY(run_passes(G, passes, lens, d_elems));
        std::vector<uint32_t> sizes;
        ASDM_TRY(compact(G, segs, sizes));
        for (size_t i = 0; i < seg_ids.size(); ++i) slen[seg_ids[i]] = sizes[i];
    }
    // remaining passes (neighbours later in the BFS order), all queries at once
    {
        std::vector<PassDesc> passes;
        std::vector<uint64_t> lens;
        for (const QPlan &qp : P) {
            if (qp.empty) continue;
            const QueryGraph &q = qp.cs->q;
            for (uint32_t u = 0; u < q.n; ++u)
                for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                    const uint32_t p = q.nbr[e];
                    if (qp.rank[p] < qp.rank[u]) continue;
                    passes.push_back(PassDesc{sbuf + sbase[qp.seg0 + p], st + seg[qp.seg0 + u], q.lab[u],
                                              1u << (e - q.off[u])});
                    lens.push_back(slen[qp.seg0 + p]);
                }
        }
        ASDM_TRY(run_passes(G, passes, lens, d_elems));
    }
    // final candidate sets into the group's arena
    auto arena = std::make_shared<CsArena>();
    arena->stream = s;
    ASDM_TRY(dalloc(&arena->d_cand, seg[nseg], s));
    {
        std::vector<CompDesc> segs;
        std::vector<uint32_t> seg_ids;
        for (const QPlan &qp : P) {
            if (qp.empty) continue;
            const QueryGraph &q = qp.cs->q;
            for (uint32_t u = 0; u < q.n; ++u) {
                const uint32_t all = q.deg(u) ? ((q.deg(u) == 32 ? 0xFFFFFFFFu : (1u << q.deg(u)) - 1u)) : 0u;
                const uint32_t su = qp.seg0 + u;
                segs.push_back(CompDesc{st + seg[su], arena->d_cand + seg[su], qp.lsize[u], kFBit | all, qp.lbase[u], 0});
                seg_ids.push_back(su);
            }
        }
        std::vector<uint32_t> sizes;
        ASDM_TRY(compact(G, segs, sizes));
        std::vector<uint32_t> ncand(nseg, 0);
        for (size_t i = 0; i < seg_ids.size(); ++i) ncand[seg_ids[i]] = sizes[i];
        for (QPlan &qp : P) {
            if (qp.empty) continue;
            asdm_cs &cs = *qp.cs;
            bool ok = true;
            for (uint32_t u = 0; u < cs.q.n; ++u) {
                cs.ncand[u] = ncand[qp.seg0 + u];
                cs.cand_base[u] = seg[qp.seg0 + u];
                ok &= cs.ncand[u] > 0;
            }
            cs.cand_base[cs.q.n] = seg[qp.seg0 + cs.q.n];
            qp.empty = !ok;
        }
    }
    // candidate edges: rank-in-label -> candidate index maps (reuse st)
    ASDM_CUDA(cudaMemsetAsync(st, 0xFF, seg[nseg] * sizeof(uint32_t), s));
    {
        std::vector<const uint32_t *> cands;
        std::vector<uint32_t *> maps;
        std::vector<uint64_t> cpre{0};
        for (const QPlan &qp : P) {
            if (qp.empty) continue;
            for (uint32_t u = 0; u < qp.cs->q.n; ++u) {
                const uint32_t su = qp.seg0 + u;
                cands.push_back(arena->d_cand + seg[su]);
                maps.push_back(st + seg[su]);
                cpre.push_back(cpre.back() + qp.cs->ncand[u]);
            }
        }
        if (cpre.back()) {
            const uint32_t **d_cands = nullptr;
            uint32_t **d_maps = nullptr;
            uint64_t *d_cpre = nullptr;
            ASDM_TRY(scr.upload(&d_cands, cands));
            ASDM_TRY(scr.upload(&d_maps, maps));
            ASDM_TRY(scr.upload(&d_cpre, cpre));
            k3_scatter_map<<<grid_for(cpre.back(), G->num_sms), kBlock, 0, s>>>(d_cands, d_cpre, (uint32_t)cands.size(),
                                                                               d_maps, g.pos_in_label);
            ::asdm::count_launch();
            ASDM_CUDA(cudaGetLastError());
        }
    }
    std::vector<EdgeDesc> edges;
    std::vector<uint64_t> item_base{0};
    std::vector<uint32_t> edge_first(Q, 0);
    for (uint32_t qi = 0; qi < Q; ++qi) {
        const QPlan &qp = P[qi];
        edge_first[qi] = (uint32_t)edges.size();
        if (qp.empty) continue;
        const asdm_cs &cs = *qp.cs;
        const QueryGraph &q = cs.q;
        for (uint32_t u = 0; u < q.n; ++u)
            for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                const uint32_t u2 = q.nbr[e];
                edges.push_back(EdgeDesc{arena->d_cand + seg[qp.seg0 + u], st + seg[qp.seg0 + u2], cs.ncand[u], q.lab[u2]});
                item_base.push_back(item_base.back() + cs.ncand[u] + 1);
            }
    }
    const uint32_t ne = (uint32_t)edges.size();
    const uint64_t nitems = item_base.back();
    std::vector<uint64_t> estart(ne, 0);
    uint64_t total = 0;
    if (ne) {
        EdgeDesc *d_edges = nullptr;
        uint64_t *d_ib = nullptr, *d_wpos = nullptr, *d_estart = nullptr;
        uint32_t *d_bad = nullptr;
        ASDM_TRY(scr.upload(&d_edges, edges));
        ASDM_TRY(scr.upload(&d_ib, item_base));
        ASDM_TRY(scr.alloc(&d_wpos, nitems + 1));
        ASDM_TRY(scr.alloc(&d_estart, ne));
        ASDM_TRY(scr.alloc(&d_bad, 1));
        ASDM_TRY(dalloc(&arena->d_eoff, nitems, s));
        ASDM_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(uint32_t), s));
        const unsigned egrid = grid_for(nitems, G->num_sms);
        k3_edges<false><<<egrid, kBlock, 0, s>>>(g, d_edges, d_ib, ne, arena->d_eoff, nullptr, nullptr, d_elems + 1);
        ::asdm::count_launch();
        ASDM_CUDA(cudaGetLastError());
        ASDM_TRY(scan_exclusive_u32(arena->d_eoff, d_wpos, nitems, true, s));
        ASDM_CUDA(cudaMemcpyAsync(&total, d_wpos + nitems, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        ASDM_CUDA(cudaStreamSynchronize(s));
        ASDM_TRY(dalloc(&arena->d_elist, total, s));
        k3_edges<true><<<egrid, kBlock, 0, s>>>(g, d_edges, d_ib, ne, nullptr, d_wpos, arena->d_elist, nullptr);
        ::asdm::count_launch();
        ASDM_CUDA(cudaGetLastError());
        k3_offsets<<<grid_for(nitems, G->num_sms), kBlock, 0, s>>>(d_ib, ne, d_wpos, arena->d_eoff, d_estart, d_bad);
        ::asdm::count_launch();
        ASDM_CUDA(cudaGetLastError());
        uint32_t bad = 0;
        ASDM_CUDA(cudaMemcpyAsync(estart.data(), d_estart, ne * sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        ASDM_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        ASDM_CUDA(cudaStreamSynchronize(s));
        if (bad) return fail(ASDM_ERR_INVALID, "a candidate-edge list exceeds 2^32 entries");
    }
    unsigned long long elems[2] = {0, 0};
    ASDM_CUDA(cudaMemcpyAsync(elems, d_elems, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    ASDM_CUDA(cudaEventRecord(ev1, s));
    ASDM_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    // K2 scans + K3 scans (count and fill read the same runs) + K1 state words
    const uint64_t bytes = 4ull * (elems[0] + 2 * elems[1]) + 4ull * seg[nseg];
    for (uint32_t qi = 0; qi < Q; ++qi) {
        QPlan &qp = P[qi];
        asdm_cs &cs = *qp.cs;
        cs.build_ms = ms / Q;
        cs.build_bytes = bytes / Q;
        cs.arena = arena;
        cs.d_cand = arena->d_cand;
        cs.d_eoff = arena->d_eoff;
        cs.d_elist = arena->d_elist;
        if (qp.empty) {
            cs.nonempty = false;
            continue;
        }
        cs.nonempty = true;
        const QueryGraph &q = cs.q;
        const uint32_t nq_e = q.off[q.n];
        cs.eoff_base.assign(nq_e, 0);
        cs.elist_base.assign(nq_e, 0);
        cs.etotal.assign(nq_e, 0);
        for (uint32_t k = 0; k < nq_e; ++k) {
            const uint32_t e = edge_first[qi] + k;
            cs.eoff_base[k] = item_base[e];
            cs.elist_base[k] = estart[e];
            const uint64_t end = (e + 1 < ne) ? estart[e + 1] : total;
            cs.etotal[k] = end - estart[e];
        }
    }
    return ASDM_OK;
}

namespace {
}  // namespace
}  // namespace asdm

using namespace asdm;

extern "C" int asdm_candidate_space(asdm_graph *g, const uint32_t *q_offsets, const uint32_t *q_nbrs,
                                    const uint32_t *q_labels, uint32_t q_n, asdm_cs **out, int *nonempty) {
    clear_error();
    if (!g || !out) return fail(ASDM_ERR_INVALID, "null argument");
    auto cs = std::make_unique<asdm_cs>();
    cs->g = g;
    ASDM_TRY(make_query(q_offsets, q_nbrs, q_labels, q_n, cs->q));
    int rc = build_batch({cs.get()});
    if (rc != ASDM_OK) {
        cs.reset();
        cudaStreamSynchronize(g->stream);
        return rc;
    }
    if (nonempty) *nonempty = cs->nonempty ? 1 : 0;
    *out = cs.release();
    return ASDM_OK;
}

extern "C" int asdm_cs_sizes(const asdm_cs *cs, uint32_t *sizes) {
    if (!cs || !sizes) return fail(ASDM_ERR_INVALID, "null argument");
    for (uint32_t u = 0; u < cs->q.n; ++u) sizes[u] = cs->ncand.empty() ? 0 : cs->ncand[u];
    return ASDM_OK;
}

extern "C" int asdm_cs_read(const asdm_cs *cs, uint32_t u, uint32_t *out, uint32_t capacity) {
    if (!cs || !out) return fail(ASDM_ERR_INVALID, "null argument");
    if (u >= cs->q.n) return fail(ASDM_ERR_INVALID, "query vertex %u out of range", u);
    const uint32_t n = cs->ncand.empty() ? 0 : cs->ncand[u];
    if (n > capacity) return fail(ASDM_ERR_CAPACITY, "candidate set of %u has %u entries", u, n);
    if (n == 0) return ASDM_OK;
    ASDM_CUDA(cudaMemcpyAsync(out, cs->d_cand + cs->cand_base[u], n * sizeof(uint32_t), cudaMemcpyDeviceToHost,
                              cs->g->stream));
    ASDM_CUDA(cudaStreamSynchronize(cs->g->stream));
    return ASDM_OK;
}

extern "C" int asdm_cs_read_edges(const asdm_cs *cs, uint32_t u, uint32_t u2, uint32_t *offsets, uint32_t *vertices,
                                  uint64_t capacity, uint64_t *total) {
    if (!cs || !offsets) return fail(ASDM_ERR_INVALID, "null argument");
    if (u >= cs->q.n || u2 >= cs->q.n) return fail(ASDM_ERR_INVALID, "query vertex out of range");
    const int k = cs->q.slot(u, u2);
    if (k < 0) return fail(ASDM_ERR_INVALID, "(%u, %u) is not a query edge", u, u2);
    if (!cs->nonempty) return fail(ASDM_ERR_INVALID, "candidate space is empty");
    const uint32_t e = cs->q.off[u] + (uint32_t)k;
    const uint64_t cnt = cs->etotal[e];
    if (total) *total = cnt;
    if (cnt > capacity) return fail(ASDM_ERR_CAPACITY, "edge list has %llu entries", (unsigned long long)cnt);
    cudaStream_t s = cs->g->stream;
    const uint32_t nu = cs->ncand[u], nu2 = cs->ncand[u2];
    ASDM_CUDA(cudaMemcpyAsync(offsets, cs->d_eoff + cs->eoff_base[e], (nu + 1) * sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, s));
    std::vector<uint32_t> idx(cnt), c2(nu2);
    if (cnt) ASDM_CUDA(cudaMemcpyAsync(idx.data(), cs->d_elist + cs->elist_base[e], cnt * sizeof(uint32_t),
                                       cudaMemcpyDeviceToHost, s));
    ASDM_CUDA(cudaMemcpyAsync(c2.data(), cs->d_cand + cs->cand_base[u2], nu2 * sizeof(uint32_t),
                              cudaMemcpyDeviceToHost, s));
    ASDM_CUDA(cudaStreamSynchronize(s));
    if (vertices)
        for (uint64_t i = 0; i < cnt; ++i) vertices[i] = c2[idx[i]];
    return ASDM_OK;
}

extern "C" int asdm_cs_free(asdm_cs *cs) {
    if (!cs) return ASDM_OK;
    cudaStream_t s = cs->g->stream;
    delete cs;  // the group's arena is freed with its last candidate space
    cudaStreamSynchronize(s);
    return ASDM_OK;
}
