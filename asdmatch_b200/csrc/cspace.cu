// K1-K3: the CFL candidate space on the device.
//
// Restates CandidateSpace::buildCandCFL (relation/candidate_space.cpp:550-721)
// as the set computation it performs.  For every query vertex u, over the
// data vertices of u's label (indexed by their rank inside the label), a
// bitset F(u) holds "passes the label, degree and NLC filter" (K1, nlcValid
// at utility/utils.cpp:30-40) and one bitset per query neighbour p of u holds
// "adjacent to the storage of p" (K2).  The storage S(p) that the reference
// scans for p is the top-down candidate set Ctd(p) plus data vertex 0
// whenever Ctd(p) is smaller than |V_l(p)|: candidateSet[p] is resized to
// |V_l(p)| up front (:555-559), its zero-initialised tail is iterated by the
// range-for loops (:588, :623, :661), and pruned entries stay in it until the
// compaction at :692-703.  Hence
//     Ctd(root) = F(root),   Ctd(u) = F(u) ∩ ⋂_{p ∈ before(u)} N_l(u)(S(p)),
//     C(u) = F(u) ∩ ⋂_{p ∈ N_q(u)} N_l(u)(S(p)),
// computed wave by wave along the CFL BFS order (a vertex's wave is one more
// than the latest wave among its earlier neighbours).  The slot bitset of a
// pass p -> u is computed in pull form: a candidate's bit is set when one of
// its l(p)-neighbours lies in Ctd(p) (the phantom vertex 0 is pushed).
// Compaction ANDs the required bitsets word by word and writes the surviving
// vertices in id order.  K3 builds the candidate edges
// (buildCandidateEdge(false), :458-487) as CSR lists of indices into C(u2),
// looking a neighbour's index up in C(u2)'s membership bitset and per-word
// prefix counts.
#include <algorithm>
#include <map>
#include <memory>
#include <queue>

#include "cs.cuh"

namespace asdm {
namespace {

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

// The same for a warp whose lanes hold ascending items (item = base + lane;
// lanes past the end pass valid = false, and every lane must call): the
// warp's first item is located once, 32 probes per round, and only a lane
// whose item lies past that segment searches on from there.  Segments here
// are long (a query vertex's candidates), so most warps need one search.
__device__ __forceinline__ uint32_t warp_find_segment(const uint64_t *__restrict__ prefix, uint32_t nseg,
                                                      uint64_t base, uint64_t item, bool valid, uint32_t lane) {
    uint32_t lo = 0, hi = nseg;
    while (hi - lo > 32) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t p = lo + lane * step;
        const uint32_t m = __ballot_sync(0xffffffffu, p < hi && prefix[p] <= base);
        const uint32_t nlo = lo + (31 - __clz(m)) * step;
        hi = min(hi, nlo + step);
        lo = nlo;
    }
    const uint32_t p = lo + lane;
    uint32_t s = lo + (31 - __clz(__ballot_sync(0xffffffffu, p < hi && prefix[p] <= base)));
    if (valid && s + 1 < nseg && prefix[s + 1] <= item) {
        uint32_t l2 = s + 1, h2 = nseg;
        while (h2 - l2 > 1) {
            const uint32_t mid = (l2 + h2) >> 1;
            if (prefix[mid] <= item) l2 = mid; else h2 = mid;
        }
        s = l2;
    }
    return s;
}

// ---- K1: label + degree + NLC filter --------------------------------------
// One segment per (query, query vertex) of a group; a segment's items are
// the ranks 0 .. |V_l(u)| - 1 of u's label, padded to a multiple of 32 so
// that a warp's 32 items are one word of F(u).
struct FilterArgs {
    DevGraph g;
    uint32_t *bits;           // bitsets of the group
    const uint64_t *seg;      // nseg + 1 prefix of the padded item counts
    const uint64_t *fword;    // word offset of F(u) in bits
    const uint32_t *lbase;    // vbl_off[l(u)]
    const uint32_t *llen;     // |V_l(u)|
    const uint32_t *qdeg;     // deg(u)
    const uint32_t *qnlc;     // (label, count) pairs
    const uint32_t *qnlc_off; // nseg + 1
    uint32_t nq;              // number of segments
    uint32_t *fcount;         // |F(u)|
};

// A warp takes a run of up to kK1Words words (32 items each) inside one
// segment, so the segment lookup and the query vertex's parameters are read
// once per run.
constexpr uint32_t kK1Words = 32;

__global__ void __launch_bounds__(kBlock) k1_filter(FilterArgs a) {
    const uint64_t total_words = a.seg[a.nq] / 32;
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t nruns = (total_words + kK1Words - 1) / kK1Words;
    for (uint64_t run = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); run < nruns; run += nwarps) {
        uint64_t w = run * kK1Words;
        const uint64_t w_end = min(total_words, w + kK1Words);
        while (w < w_end) {
            const uint32_t u = find_segment(a.seg, a.nq, w * 32);
            const uint64_t seg_w0 = a.seg[u] / 32, seg_w1 = a.seg[u + 1] / 32;
            const uint64_t stop = min(w_end, seg_w1);
            const uint32_t len = a.llen[u], lbase = a.lbase[u], qdeg = a.qdeg[u];
            const uint32_t k0 = a.qnlc_off[u], k1 = a.qnlc_off[u + 1];
            uint32_t total = 0;
            for (; w < stop; ++w) {
                const uint32_t i = (uint32_t)(w - seg_w0) * 32 + lane;
                bool pass = false;
                if (i < len) {
                    // degree and neighbour-label mask of the vertex, in label order
                    const uint2 info = a.g.rank_info[lbase + i];
                    pass = info.x >= qdeg;
                    for (uint32_t k = k0; pass && k < k1; ++k) {
                        const uint32_t l = a.qnlc[2 * k], c = a.qnlc[2 * k + 1];
                        pass = l < a.g.nlabels && ((info.y >> (l & 31u)) & 1u);
                        if (pass && (c > 1 || a.g.nlabels > 32)) {
                            uint32_t b, e;
                            label_run(a.g, a.g.vbl[lbase + i], l, b, e);
                            pass = (e - b) >= c;
                        }
                    }
                }
                const uint32_t word = __ballot_sync(0xffffffffu, pass);
                if (lane == 0) a.bits[a.fword[u] + (w - seg_w0)] = word;
                total += __popc(word);
            }
            if (lane == 0 && total) atomicAdd(&a.fcount[u], total);
        }
    }
}

// F(u) of query vertices whose filter inputs (label, degree, neighbour-label
// counts) repeat an earlier vertex of the group: copied from that vertex's
// bitset instead of filtered again.
struct CopySeg {
    const uint32_t *src;
    uint32_t *dst;
};

__global__ void __launch_bounds__(kBlock) copy_words(const CopySeg *__restrict__ segs, const uint64_t *__restrict__ prefix,
                                                     uint32_t nseg) {
    const uint64_t total = prefix[nseg];
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = find_segment(prefix, nseg, t);
        segs[k].dst[t - prefix[k]] = segs[k].src[t - prefix[k]];
    }
}

// ---- K2: neighbour marking passes -------------------------------------------
// Push form (used for the phantom vertex 0 of a storage): every l(u)-neighbour
// of a listed vertex gets its bit in u's slot bitset.
struct PassDesc {
    const uint32_t *src;   // vertex ids
    uint32_t *mbits;       // u's bitset for p
    uint32_t label;        // l(u)
    uint32_t pad;
    const uint32_t *cond;  // or null: the pass runs only where *cond is nonzero
};

__device__ __forceinline__ void mark(const DevGraph &g, uint32_t *mb, uint32_t k) {
    const uint32_t r = g.nbr_rank[k];
    atomicOr(&mb[r >> 5], 1u << (r & 31u));  // result unused: a fire-and-forget reduction
}

// A warp takes 32 items and marks the concatenation of their label runs 32
// entries at a time, a lane per entry (every lane has a reduction to issue,
// whatever the run lengths).
__global__ void __launch_bounds__(kBlock) k2_pass(DevGraph g, const PassDesc *__restrict__ passes,
                                                  const uint64_t *__restrict__ prefix, uint32_t npass,
                                                  unsigned long long *__restrict__ elems) {
    constexpr uint32_t kWarps = kBlock / 32;
    __shared__ uint64_t s_pre[kWarps][33];   // exclusive prefix of the run lengths (s_pre[32] = total)
    __shared__ uint32_t *s_mb[kWarps][32];
    __shared__ uint32_t s_b[kWarps][32];
    const uint64_t total = prefix[npass];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t scanned = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total; base += stride) {
        const uint64_t pos = base + lane;
        uint32_t b = 0, e = 0;
        if (pos < total) {
            const uint64_t item = pos;
            const uint32_t p = find_segment(prefix, npass, item);
            const PassDesc d = passes[p];
            if (!d.cond || *d.cond) label_run(g, d.src[item - prefix[p]], d.label, b, e);
            s_mb[wid][lane] = d.mbits;
        }
        s_b[wid][lane] = b;
        uint64_t inc = e - b;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= (uint32_t)o) inc += y;
        }
        s_pre[wid][lane + 1] = inc;
        if (lane == 0) s_pre[wid][0] = 0;
        __syncwarp();
        const uint64_t S = s_pre[wid][32];
        scanned += S;
        for (uint64_t j = lane; j < S; j += 32) {
            // owner: the last item whose run starts at or before j
            uint32_t lo = 0, hi = 32;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (s_pre[wid][mid] <= j) lo = mid; else hi = mid;
            }
            mark(g, s_mb[wid][lo], s_b[wid][lo] + (uint32_t)(j - s_pre[wid][lo]));
        }
        __syncwarp();
    }
    if (lane == 0 && scanned) atomicAdd(elems, (unsigned long long)scanned);
}

// Pull form of a marking pass (p -> u): the bit of each candidate x of u
// (F(u) for passes from earlier BFS neighbours, Ctd(u) for the later ones:
// the final AND discards the rest) is set when some neighbour of x with label
// l(p) lies in Ctd(p).  Same bits on those candidates as pushing from S(p);
// the phantom vertex 0 of S(p) is pushed separately.  A warp takes 32 words
// of candidates; each lane scans one candidate's label run, stopping at its
// first member of Ctd(p), and runs left open after kPullLane entries are
// finished by the whole warp 32 entries at a time.
struct PullDesc {
    const uint32_t *xbits;   // candidates to test, by rank in l(u)
    uint32_t *mbits;         // u's slot bitset for p
    const uint32_t *sbits;   // membership of Ctd(p), by rank in l(p)
    uint32_t lbase;          // vbl_off[l(u)]
    uint32_t label;          // l(p)
    uint32_t words;          // words of xbits
    uint32_t pad;
};

constexpr uint32_t kPullLane = 16;

// Position of the n-th (0-based) set bit of w; n < popc(w).
__device__ __forceinline__ uint32_t nth_set_bit(uint32_t w, uint32_t n) {
    uint32_t pos = 0;
#pragma unroll
    for (uint32_t width = 16; width; width >>= 1) {
        const uint32_t low = __popc(w & ((1u << width) - 1u));
        if (n >= low) {
            n -= low;
            w >>= width;
            pos += width;
        }
    }
    return pos;
}

__device__ __forceinline__ bool pull_member(const DevGraph &g, const uint32_t *sb, uint32_t k) {
    const uint32_t z = g.nbr_rank[k];
    return (sb[z >> 5] >> (z & 31u)) & 1u;
}

__global__ void __launch_bounds__(kBlock) k2_pull(DevGraph g, const PullDesc *__restrict__ passes,
                                                  const uint64_t *__restrict__ group_pre, uint32_t npass,
                                                  unsigned long long *__restrict__ elems) {
    constexpr uint32_t kWarps = kBlock / 32;
    __shared__ uint32_t s_out[kWarps][32];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint64_t ngroups = group_pre[npass];
    const uint64_t nwarps = (uint64_t)gridDim.x * kWarps;
    uint64_t scanned = 0;
    s_out[wid][lane] = 0;
    __syncwarp();
    for (uint64_t grp = (uint64_t)blockIdx.x * kWarps + wid; grp < ngroups; grp += nwarps) {
        const uint32_t pi = find_segment(group_pre, npass, grp);
        const PullDesc d = passes[pi];
        const uint32_t w0 = (uint32_t)(grp - group_pre[pi]) * 32;
        const uint32_t f = (w0 + lane < d.words) ? d.xbits[w0 + lane] : 0u;
        // inclusive prefix of the candidates per word
        uint32_t pre = __popc(f);
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, pre, o);
            if (lane >= (uint32_t)o) pre += y;
        }
        const uint32_t total = __shfl_sync(0xffffffffu, pre, 31);
        for (uint32_t t0 = 0; t0 < total; t0 += 32) {
            const uint32_t t = t0 + lane;
            // owner word: the first lane whose inclusive prefix exceeds t
            uint32_t o = 0;
#pragma unroll
            for (uint32_t step = 16; step; step >>= 1) {
                const uint32_t v = __shfl_sync(0xffffffffu, pre, o + step - 1);
                if (v <= t) o += step;
            }
            o = min(o, 31u);
            const uint32_t word = __shfl_sync(0xffffffffu, f, o);
            const uint32_t before = __shfl_sync(0xffffffffu, pre - __popc(f), o);
            const bool mine = t < total;
            uint32_t bit = 0, b = 0, e = 0;
            if (mine) {
                bit = nth_set_bit(word, t - before);
                const uint32_t x = g.vbl[d.lbase + 32 * (w0 + o) + bit];
                label_run(g, x, d.label, b, e);
            }
            bool hit = false;
            const uint32_t stop = min(e, b + kPullLane);
            uint32_t k = b;
            for (; k < stop && !hit; ++k) hit = pull_member(g, d.sbits, k);
            scanned += k - b;
            // runs still open: the whole warp scans them
            uint32_t todo = __ballot_sync(0xffffffffu, mine && !hit && k < e);
            while (todo) {
                const int src = __ffs(todo) - 1;
                todo &= todo - 1;
                const uint32_t kk = __shfl_sync(0xffffffffu, k, src), ee = __shfl_sync(0xffffffffu, e, src);
                bool found = false;
                uint32_t seen = 0;
                for (uint32_t base = kk; base < ee && !found; base += 32) {
                    const uint32_t j = base + lane;
                    found = __any_sync(0xffffffffu, j < ee && pull_member(g, d.sbits, j));
                    seen += min(32u, ee - base);
                }
                if ((int)lane == src) {
                    hit = found;
                    scanned += seen;
                }
            }
            if (hit) atomicOr(&s_out[wid][o], 1u << bit);
        }
        __syncwarp();
        const uint32_t m = s_out[wid][lane];
        if (m) {
            atomicOr(&d.mbits[w0 + lane], m);
            s_out[wid][lane] = 0;
        }
        __syncwarp();
    }
    for (int o = 16; o; o >>= 1) scanned += __shfl_xor_sync(0xffffffffu, scanned, o);
    if (lane == 0 && scanned) atomicAdd(elems, (unsigned long long)scanned);
}

// ---- K3a: compaction of bitsets into vertex lists, word by word ------------
constexpr int kItems = 8;               // words per thread
constexpr int kTile = kBlock * kItems;  // words per tile

struct CompDesc {
    const uint32_t *bits;   // F(u); the bitset of u's query-neighbour slot b at bits + (1 + b) * words
    uint32_t words;         // ceil(|V_l(u)| / 32)
    uint32_t need;          // slots whose bitsets are required
    uint32_t len;           // |V_l(u)|
    uint32_t lbase;         // vbl_off[l(u)]
    uint32_t phantom;       // append data vertex 0 when fewer than len survive
    uint32_t pad;
    uint2 *cmem;            // or null: per word of the result, {membership bits, result size before it}
    uint32_t *sbits;        // or null: the result's membership bits alone
    uint32_t *ph;           // or null: set to 1 when the phantom vertex was appended, else 0
};

__device__ __forceinline__ uint32_t comp_word(const CompDesc &d, uint32_t w) {
    uint32_t x = d.bits[w];
    for (uint32_t m = d.need; m && x; m &= m - 1) x &= d.bits[(uint64_t)__ffs(m) * d.words + w];
    return x;
}

__global__ void __launch_bounds__(kBlock) k3_count(const CompDesc *__restrict__ segs, const uint64_t *__restrict__ tile_first,
                                                   uint32_t nseg, uint32_t *__restrict__ tile_cnt) {
    const uint32_t t = blockIdx.x;
    const uint32_t sidx = find_segment(tile_first, nseg, t);
    const CompDesc d = segs[sidx];
    const uint32_t first = (uint32_t)(t - tile_first[sidx]) * kTile;
    uint32_t c = 0;
    for (uint32_t k = threadIdx.x; k < (uint32_t)kTile; k += kBlock) {
        const uint32_t w = first + k;
        if (w < d.words) c += __popc(comp_word(d, w));
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

// Segment sidx writes to out + tile_pos[tile_first[sidx]] + sidx (one spare
// slot per segment for the phantom vertex).
__global__ void __launch_bounds__(kBlock) k3_write(const CompDesc *__restrict__ segs, const uint64_t *__restrict__ tile_first,
                                                   uint32_t nseg, const uint64_t *__restrict__ tile_pos,
                                                   const uint32_t *__restrict__ vbl, uint32_t *__restrict__ out,
                                                   uint32_t *__restrict__ seg_count) {
    const uint32_t t = blockIdx.x;
    const uint32_t sidx = find_segment(tile_first, nseg, t);
    const CompDesc d = segs[sidx];
    const uint32_t first = (uint32_t)(t - tile_first[sidx]) * kTile;
    const uint32_t my = first + threadIdx.x * kItems;
    uint32_t x[kItems];
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        x[k] = (my + k < d.words) ? comp_word(d, my + k) : 0u;
        c += __popc(x[k]);
    }
    // block exclusive scan of c
    __shared__ uint32_t wsum[kBlock / 32];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t v = c;
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
    }
    if (lane == 31) wsum[warp] = v;
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
    const uint64_t seg_first = tile_pos[tile_first[sidx]];
    uint32_t *o = out ? out + seg_first + sidx : nullptr;  // null: sizes and bitsets only
    uint32_t pos = (uint32_t)(tile_pos[t] - seg_first) + (warp ? wsum[warp - 1] : 0) + v - c;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const uint32_t w = my + k;
        if (w >= d.words) break;
        if (d.cmem) d.cmem[w] = make_uint2(x[k], pos);
        if (d.sbits) d.sbits[w] = x[k];
        if (o)
            for (uint32_t y = x[k]; y; y &= y - 1) o[pos++] = vbl[d.lbase + 32 * w + (uint32_t)(__ffs(y) - 1)];
    }
    // the last tile of a segment records the segment size
    if (threadIdx.x == 0 && t + 1 == tile_first[sidx + 1]) {
        uint32_t size = (uint32_t)(tile_pos[t + 1] - seg_first);
        const bool ph = d.phantom && size < d.len;  // the reference's zero-filled storage tail
        if (ph) {
            if (o) o[size] = 0;
            ++size;
        }
        if (d.ph) *d.ph = ph ? 1u : 0u;
        seg_count[sidx] = size;
    }
}

// ---- K3b: candidate edges ---------------------------------------------------
struct EdgeDesc {
    const uint32_t *cand_u;   // C(u)
    const uint2 *cmem;        // per word of ranks in l(u2): {membership of C(u2), |C(u2)| before it}
    uint32_t ncand_u;
    uint32_t label_u2;
};

// Index in C(u2) of the vertex of rank r in l(u2), or kNone (one 8-byte
// load: the word's bits and prefix side by side).
__device__ __forceinline__ uint32_t cand_index(const uint2 *cm, uint32_t r) {
    const uint2 w = cm[r >> 5];
    const uint32_t bit = 1u << (r & 31u);
    return (w.x & bit) ? w.y + (uint32_t)__popc(w.x & (bit - 1u)) : kNone;
}

// rstart (optional): each item's label-run start, its length in cnt (read
// before cnt is overwritten with the count), both written by k3_bound.
template <bool kFill>
__global__ void __launch_bounds__(kBlock) k3_edges(DevGraph g, const EdgeDesc *__restrict__ edges,
                                                   const uint64_t *__restrict__ item_base, uint32_t nedges,
                                                   uint32_t *__restrict__ cnt, const uint64_t *__restrict__ wpos,
                                                   uint32_t *__restrict__ elist, unsigned long long *__restrict__ elems,
                                                   const uint32_t *__restrict__ rstart) {
    const uint64_t total = item_base[nedges];
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t scanned = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total; base += stride) {
        const uint64_t pos = base + lane;
        const uint64_t item = pos;
        uint32_t b = 0, e = 0;
        const uint2 *cm = nullptr;
        const uint32_t ei = warp_find_segment(item_base, nedges, base, item, pos < total, lane);
        if (pos < total) {
            const EdgeDesc d = edges[ei];
            if (rstart) {
                b = rstart[item];
                e = b + cnt[item];
            } else {
                const uint32_t i = (uint32_t)(item - item_base[ei]);
                if (i < d.ncand_u) label_run(g, d.cand_u[i], d.label_u2, b, e);
            }
            cm = d.cmem;
        }
        scanned += e - b;
        const bool coop = (e - b) > kLongRun;
        uint32_t mine = 0;
        uint64_t out = kFill && pos < total ? wpos[item] : 0;
        uint32_t todo = __ballot_sync(0xffffffffu, coop);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint32_t bb = __shfl_sync(0xffffffffu, b, src), ee = __shfl_sync(0xffffffffu, e, src);
            const uint2 *mm = (const uint2 *)__shfl_sync(0xffffffffu, (unsigned long long)cm, src);
            uint64_t o = __shfl_sync(0xffffffffu, out, src);
            uint32_t c = 0;
            for (uint32_t k0 = bb; k0 < ee; k0 += 32) {
                const uint32_t k = k0 + lane;
                const uint32_t idx = k < ee ? cand_index(mm, g.nbr_rank[k]) : kNone;
                const uint32_t hit = __ballot_sync(0xffffffffu, idx != kNone);
                if (kFill && idx != kNone) elist[o + __popc(hit & ((1u << lane) - 1))] = idx;
                o += __popc(hit);
                c += __popc(hit);
            }
            if ((int)lane == src) mine = c;
        }
        if (!coop) {
#pragma unroll 4
            for (uint32_t k = b; k < e; ++k) {
                const uint32_t idx = cand_index(cm, g.nbr_rank[k]);
                if (idx != kNone) {
                    if (kFill) elist[out++] = idx;
                    ++mine;
                }
            }
        }
        if (cnt && pos < total) cnt[item] = mine;
    }
    if (elems) {
        for (int o = 16; o; o >>= 1) scanned += __shfl_xor_sync(0xffffffffu, scanned, o);
        if (lane == 0 && scanned) atomicAdd(elems, (unsigned long long)scanned);
    }
}

// The padded fill with the neighbour scan spread over the lanes: a warp takes
// 32 consecutive items and walks the concatenation of their label runs 32
// entries at a time, a lane per entry, so every lane has a membership lookup
// in flight whatever the run lengths.  In: cnt = run lengths, rstart = run
// starts (k3_bound), upos = padded positions; out: each item's hits packed in
// order at the front of its padded region, cnt = their number.
__global__ void __launch_bounds__(kBlock, 6) k3_flat(DevGraph g, const EdgeDesc *__restrict__ edges,
                                                  const uint64_t *__restrict__ item_base, uint32_t nedges,
                                                  uint32_t *__restrict__ cnt, const uint64_t *__restrict__ upos,
                                                  const uint32_t *__restrict__ rstart, uint32_t *__restrict__ padded,
                                                  unsigned long long *__restrict__ elems) {
    constexpr uint32_t kWarps = kBlock / 32;
    __shared__ uint64_t s_pre[kWarps][33];   // exclusive prefix of the run lengths (s_pre[32] = total)
    __shared__ uint64_t s_out[kWarps][32];   // padded position of each item
    __shared__ const uint2 *s_cm[kWarps][32];
    __shared__ uint32_t s_rs[kWarps][32], s_hits[kWarps][32];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint64_t total = item_base[nedges];
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t scanned = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total; base += stride) {
        const uint64_t item = base + lane;
        uint64_t len = 0;
        const uint32_t ei = warp_find_segment(item_base, nedges, base, item, item < total, lane);
        if (item < total) {
            s_cm[wid][lane] = edges[ei].cmem;
            len = cnt[item];
            s_rs[wid][lane] = rstart[item];
            s_out[wid][lane] = upos[item];
        }
        uint64_t inc = len;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= (uint32_t)o) inc += y;
        }
        s_pre[wid][lane + 1] = inc;
        if (lane == 0) s_pre[wid][0] = 0;
        s_hits[wid][lane] = 0;
        __syncwarp();
        const uint64_t S = s_pre[wid][32];
        scanned += S;
        // owner of entry j: the last item whose run starts at or before j
        // (empty runs share their start with the next item and come first)
        auto owner = [&](uint64_t j) {
            uint32_t lo = 0, hi = 32;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (s_pre[wid][mid] <= j) lo = mid; else hi = mid;
            }
            return lo;
        };
        // one round's hits of the entries j0 .. j0+31 (idx = kNone for a miss)
        // packed behind their item's earlier hits
        auto emit = [&](uint64_t j0, uint32_t it, uint64_t first, uint32_t idx) {
            const uint64_t j = j0 + lane;
            const bool valid = j < S;
            const uint32_t mask = __ballot_sync(0xffffffffu, idx != kNone);
            // the item's lanes in this round are contiguous, from lane f
            const uint32_t f = first > j0 ? (uint32_t)(first - j0) : 0u;
            const uint32_t mine = mask & ~((1u << f) - 1u);
            const uint32_t done = s_hits[wid][it];
            if (idx != kNone) padded[s_out[wid][it] + done + __popc(mine & ((1u << lane) - 1u))] = idx;
            const uint32_t next_it = __shfl_down_sync(0xffffffffu, it, 1);
            const bool last = valid && (lane == 31 || j + 1 == S || next_it != it);
            __syncwarp();
            if (last) s_hits[wid][it] = done + __popc(mine & ((2u << lane) - 1u));
            __syncwarp();
        };
        // two rounds at a time: both rounds' rank and membership loads are in
        // flight together (the rounds' outputs are packed in order after)
        for (uint64_t j0 = 0; j0 < S; j0 += 64) {
            const uint64_t ja = j0 + lane, jb = ja + 32;
            const bool va = ja < S, vb = jb < S;
            const uint32_t ita = owner(ja), itb = owner(jb);
            const uint64_t fa = s_pre[wid][ita], fb = s_pre[wid][itb];
            const uint32_t ra = va ? g.nbr_rank[s_rs[wid][ita] + (uint32_t)(ja - fa)] : 0u;
            const uint32_t rb = vb ? g.nbr_rank[s_rs[wid][itb] + (uint32_t)(jb - fb)] : 0u;
            const uint32_t xa = va ? cand_index(s_cm[wid][ita], ra) : kNone;
            const uint32_t xb = vb ? cand_index(s_cm[wid][itb], rb) : kNone;
            emit(j0, ita, fa, xa);
            if (j0 + 32 < S) emit(j0 + 32, itb, fb, xb);
        }
        if (item < total) cnt[item] = s_hits[wid][lane];
        __syncwarp();
    }
    if (elems && lane == 0 && scanned) atomicAdd(elems, (unsigned long long)scanned);
}

// Upper bound of every item's list: the length of the candidate's label run.
__global__ void __launch_bounds__(kBlock) k3_bound(DevGraph g, const EdgeDesc *__restrict__ edges,
                                                   const uint64_t *__restrict__ item_base, uint32_t nedges,
                                                   uint32_t *__restrict__ ub,
                                                   uint32_t *__restrict__ rstart) {
    const uint64_t total = item_base[nedges];
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total;
         base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t item = base + lane;
        const uint32_t ei = warp_find_segment(item_base, nedges, base, item, item < total, lane);
        if (item >= total) continue;
        const EdgeDesc d = edges[ei];
        const uint32_t i = (uint32_t)(item - item_base[ei]);
        uint32_t b = 0, e = 0;
        if (i < d.ncand_u) label_run(g, d.cand_u[i], d.label_u2, b, e);
        ub[item] = e - b;
        if (rstart) rstart[item] = b;
    }
}

// Dense copy of the padded lists: a lane per item copies a short list, the
// warp together copies every list longer than 32 entries.
// The same pass turns the counts (cnt) into each item's offset within its
// edge's list, records each edge's first entry and flags a list offset past
// 2^32 (the work of k3_offsets).
__global__ void __launch_bounds__(kBlock) k3_pack(const uint64_t *__restrict__ upos, uint32_t *__restrict__ cnt,
                                                  const uint64_t *__restrict__ wpos, uint64_t nitems,
                                                  const uint32_t *__restrict__ padded, uint32_t *__restrict__ elist,
                                                  const uint64_t *__restrict__ item_base, uint32_t nedges,
                                                  uint64_t *__restrict__ edge_start, uint32_t *__restrict__ bad) {
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t nwarps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    for (uint64_t base = ((uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32; base < nitems;
         base += nwarps * 32) {
        const uint64_t my = base + lane;
        const uint32_t c = my < nitems ? cnt[my] : 0u;
        const uint64_t from = my < nitems ? upos[my] : 0, to = my < nitems ? wpos[my] : 0;
        const uint32_t ei = warp_find_segment(item_base, nedges, base, my, my < nitems, lane);
        if (my < nitems) {
            const uint64_t first = item_base[ei];
            const uint64_t rel = to - wpos[first];
            if (rel > 0xFFFFFFFFull) atomicExch(bad, 1u);
            cnt[my] = (uint32_t)rel;
            if (my == first) edge_start[ei] = to;
        }
        // the 32 items' dense lists are one contiguous range from lane 0's
        // position: the warp copies it a lane per entry (coalesced stores),
        // each entry read from its owner item's padded list
        uint64_t pre = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, pre, o);
            if (lane >= (uint32_t)o) pre += y;
        }
        const uint64_t total = __shfl_sync(0xffffffffu, pre, 31), to0 = __shfl_sync(0xffffffffu, to, 0);
        for (uint64_t t0 = 0; t0 < total; t0 += 32) {
            const uint64_t t = t0 + lane;
            // owner: the first lane whose inclusive prefix passes t
            uint32_t o = 0;
#pragma unroll
            for (uint32_t step = 16; step; step >>= 1) {
                const uint64_t v = __shfl_sync(0xffffffffu, pre, o + step - 1);
                if (v <= t) o += step;
            }
            const uint64_t f = __shfl_sync(0xffffffffu, from, o);
            const uint64_t ex = __shfl_sync(0xffffffffu, pre - c, o);
            if (t < total) elist[to0 + t] = padded[f + (t - ex)];
        }
    }
}

__global__ void k3_offsets(const uint64_t *__restrict__ item_base, uint32_t nedges, const uint64_t *__restrict__ wpos,
                           uint32_t *__restrict__ eoff, uint64_t *__restrict__ edge_start, uint32_t *__restrict__ bad) {
    const uint64_t total = item_base[nedges];
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total;
         base += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = base + lane;
        const uint32_t ei = warp_find_segment(item_base, nedges, base, i, i < total, lane);
        if (i >= total) continue;
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

// One compaction over the given segments into one new device buffer (*out,
// the caller frees it): segment i's vertices at *out + start[i], size[i] of
// them (plus, where asked, the phantom vertex).  With out null only the
// segments' device outputs (bitsets, phantom flags) are produced, with no
// wait for the device.
int compact(asdm_graph *G, const std::vector<CompDesc> &segs, uint32_t **out, std::vector<uint64_t> &start,
            std::vector<uint32_t> &sizes) {
    cudaStream_t s = G->stream;
    const uint32_t nseg = (uint32_t)segs.size();
    if (out) *out = nullptr;
    sizes.assign(nseg, 0);
    start.assign(nseg, 0);
    if (nseg == 0) return ASDM_OK;
    std::vector<uint64_t> tile_first(nseg + 1, 0);
    for (uint32_t i = 0; i < nseg; ++i) tile_first[i + 1] = tile_first[i] + (segs[i].words + kTile - 1) / kTile;
    const uint64_t ntiles = tile_first[nseg];
    CompDesc *d_segs = nullptr;
    uint64_t *d_tf = nullptr, *d_pos = nullptr;
    uint32_t *d_cnt = nullptr, *d_sc = nullptr;
    int rc = ASDM_OK;
    std::vector<uint64_t> pos(ntiles + 1, 0);
    do {
        if (ntiles == 0) {
            if (out && (rc = dalloc(out, nseg, s))) break;
            for (uint32_t i = 0; i < nseg; ++i) start[i] = i;
            break;
        }
        if ((rc = dalloc(&d_segs, nseg, s)) || (rc = dalloc(&d_tf, nseg + 1, s)) || (rc = dalloc(&d_cnt, ntiles, s)) ||
            (rc = dalloc(&d_pos, ntiles + 1, s)) || (rc = dalloc(&d_sc, nseg, s)))
            break;
        if (upload_async(G, d_segs, segs.data(), nseg * sizeof(CompDesc)) != cudaSuccess ||
            upload_async(G, d_tf, tile_first.data(), (nseg + 1) * sizeof(uint64_t)) !=
                cudaSuccess ||
            cudaMemsetAsync(d_sc, 0, nseg * sizeof(uint32_t), s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "compaction upload failed");
            break;
        }
        k3_count<<<(unsigned)ntiles, kBlock, 0, s>>>(d_segs, d_tf, nseg, d_cnt);
        ::asdm::count_launch();
        if (cudaGetLastError() != cudaSuccess) { rc = fail(ASDM_ERR_CUDA, "compaction count failed"); break; }
        if ((rc = scan_exclusive_u32(d_cnt, d_pos, ntiles, true, s))) break;
        if (!out) {
            // bitsets and flags only: nothing for the host to read back
            k3_write<<<(unsigned)ntiles, kBlock, 0, s>>>(d_segs, d_tf, nseg, d_pos, G->d.vbl, nullptr, d_sc);
            ::asdm::count_launch();
            if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "compaction write failed");
            break;
        }
        if (cudaMemcpyAsync(pos.data(), d_pos, (ntiles + 1) * sizeof(uint64_t), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "compaction readback failed");
            break;
        }
        if ((rc = dalloc(out, pos[ntiles] + nseg, s))) break;
        k3_write<<<(unsigned)ntiles, kBlock, 0, s>>>(d_segs, d_tf, nseg, d_pos, G->d.vbl, *out, d_sc);
        ::asdm::count_launch();
        if (cudaGetLastError() != cudaSuccess) { rc = fail(ASDM_ERR_CUDA, "compaction write failed"); break; }
        if (cudaMemcpyAsync(sizes.data(), d_sc, nseg * sizeof(uint32_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "compaction size readback failed");
            break;
        }
        for (uint32_t i = 0; i < nseg; ++i) start[i] = pos[tile_first[i]] + i;
    } while (false);
    dfree(d_segs, s); dfree(d_tf, s); dfree(d_cnt, s); dfree(d_pos, s); dfree(d_sc, s);
    if (rc != ASDM_OK && out) dfree(*out, s);
    return rc;
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
    ASDM_CUDA(upload_async(G, d_p, passes.data(), np * sizeof(PassDesc)));
    ASDM_CUDA(upload_async(G, d_prefix, prefix.data(), (np + 1) * sizeof(uint64_t)));
    int rc = ASDM_OK;
    k2_pass<<<grid_for(prefix[np], G->num_sms), kBlock, 0, s>>>(G->d, d_p, d_prefix, np, d_elems);
    ::asdm::count_launch();
    if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "marking pass failed");
    dfree(d_p, s);
    dfree(d_prefix, s);
    return rc;
}

// All pull passes of one phase in one launch.
int run_pulls(asdm_graph *G, const std::vector<PullDesc> &pulls, unsigned long long *d_elems) {
    cudaStream_t s = G->stream;
    const uint32_t np = (uint32_t)pulls.size();
    if (np == 0) return ASDM_OK;
    std::vector<uint64_t> gpre(np + 1, 0);
    for (uint32_t i = 0; i < np; ++i) gpre[i + 1] = gpre[i] + (pulls[i].words + 31) / 32;
    if (gpre[np] == 0) return ASDM_OK;
    PullDesc *d_p = nullptr;
    uint64_t *d_pre = nullptr;
    int rc = ASDM_OK;
    do {
        if ((rc = dalloc(&d_p, np, s)) || (rc = dalloc(&d_pre, np + 1, s))) break;
        if (upload_async(G, d_p, pulls.data(), np * sizeof(PullDesc)) != cudaSuccess ||
            upload_async(G, d_pre, gpre.data(), (np + 1) * sizeof(uint64_t)) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "pull-pass upload failed");
            break;
        }
        const uint64_t blocks = (gpre[np] + kBlock / 32 - 1) / (kBlock / 32);
        const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(blocks, (uint64_t)G->num_sms * 32));
        k2_pull<<<grid, kBlock, 0, s>>>(G->d, d_p, d_pre, np, d_elems);
        ::asdm::count_launch();
        if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "pull pass failed");
    } while (false);
    dfree(d_p, s);
    dfree(d_pre, s);
    return rc;
}

struct Scratch {
    cudaStream_t s;
    asdm_graph *G;
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
        if (!h.empty()) ASDM_CUDA(upload_async(G, *p, h.data(), h.size() * sizeof(T)));
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
    Scratch scr{s, G, {}};
    // descriptor uploads go through the graph's pinned stage, reused per build
    ASDM_CUDA(cudaStreamSynchronize(s));
    G->stage.reset();
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
    // bitset layout [F | slot 0 | slot 1 | ...] per query vertex; K1 filters
    // one query vertex per distinct (label, degree, neighbour-label counts)
    // and copies F to the others
    std::vector<uint64_t> fword(nseg + 1, 0);
    std::vector<uint32_t> words(nseg);
    std::vector<uint64_t> seg{0}, kfword;               // K1 segments (distinct signatures)
    std::vector<uint32_t> lbase, llen, qdeg, qnlc, qnlc_off{0};
    std::map<std::vector<uint32_t>, uint32_t> sig_k1;   // signature -> K1 segment
    std::vector<uint32_t> k1_of(nseg);
    for (const QPlan &qp : P) {
        const QueryGraph &q = qp.cs->q;
        for (uint32_t u = 0; u < q.n; ++u) {
            const uint32_t sg = qp.seg0 + u;
            words[sg] = (qp.lsize[u] + 31) / 32;
            fword[sg + 1] = fword[sg] + (uint64_t)(q.deg(u) + 1) * words[sg];
            std::vector<uint32_t> sig{q.lab[u], q.deg(u)};
            for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                const uint32_t l = q.lab[q.nbr[e]];
                if (sig.size() > 2 && sig[sig.size() - 2] == l) sig.back()++;
                else { sig.push_back(l); sig.push_back(1); }
            }
            auto it = sig_k1.find(sig);
            if (it != sig_k1.end()) {
                k1_of[sg] = it->second;
                continue;
            }
            const uint32_t k = (uint32_t)lbase.size();
            sig_k1.emplace(sig, k);
            k1_of[sg] = k;
            seg.push_back(seg.back() + 32ull * words[sg]);
            kfword.push_back(fword[sg]);
            lbase.push_back(qp.lbase[u]);
            llen.push_back(qp.lsize[u]);
            qdeg.push_back(q.deg(u));
            qnlc.insert(qnlc.end(), sig.begin() + 2, sig.end());
            qnlc_off.push_back((uint32_t)(qnlc.size() / 2));
        }
    }
    const uint32_t nk1 = (uint32_t)lbase.size();
    kfword.push_back(0);
    uint32_t *bits = nullptr, *d_fcount = nullptr, *d_lbase = nullptr, *d_llen = nullptr, *d_qdeg = nullptr,
             *d_qnlc = nullptr, *d_qnlc_off = nullptr;
    uint64_t *d_seg = nullptr, *d_fword = nullptr;
    unsigned long long *d_elems = nullptr;
    ASDM_TRY(scr.alloc(&bits, fword[nseg]));
    ASDM_CUDA(cudaMemsetAsync(bits, 0, std::max<uint64_t>(fword[nseg], 1) * sizeof(uint32_t), s));
    if (lbase.empty()) {
        lbase.push_back(0);
        llen.push_back(0);
        qdeg.push_back(0);
    }
    ASDM_TRY(scr.upload(&d_seg, seg));
    ASDM_TRY(scr.upload(&d_fword, kfword));
    ASDM_TRY(scr.upload(&d_lbase, lbase));
    ASDM_TRY(scr.upload(&d_llen, llen));
    ASDM_TRY(scr.upload(&d_qdeg, qdeg));
    if (qnlc.empty()) qnlc.push_back(0);
    ASDM_TRY(scr.upload(&d_qnlc, qnlc));
    ASDM_TRY(scr.upload(&d_qnlc_off, qnlc_off));
    ASDM_TRY(scr.alloc(&d_fcount, std::max<uint32_t>(nk1, 1)));
    ASDM_TRY(scr.alloc(&d_elems, 2));
    ASDM_CUDA(cudaMemsetAsync(d_fcount, 0, std::max<uint32_t>(nk1, 1) * sizeof(uint32_t), s));
    ASDM_CUDA(cudaMemsetAsync(d_elems, 0, 2 * sizeof(unsigned long long), s));
    if (seg[nk1]) {
        FilterArgs fa{g, bits, d_seg, d_fword, d_lbase, d_llen, d_qdeg, d_qnlc, d_qnlc_off, nk1, d_fcount};
        k1_filter<<<grid_for(seg[nk1] / kK1Words, G->num_sms), kBlock, 0, s>>>(fa);
        ::asdm::count_launch();
        ASDM_CUDA(cudaGetLastError());
    }
    uint64_t copied_words = 0;
    {
        // F of the repeated signatures
        std::vector<CopySeg> cps;
        std::vector<uint64_t> cpre{0};
        for (uint32_t sg = 0; sg < nseg; ++sg) {
            const uint32_t k = k1_of[sg];
            if (kfword[k] == fword[sg]) continue;  // the vertex K1 filtered
            cps.push_back(CopySeg{bits + kfword[k], bits + fword[sg]});
            cpre.push_back(cpre.back() + words[sg]);
        }
        copied_words = cpre.back();
        if (!cps.empty() && cpre.back()) {
            CopySeg *d_cps = nullptr;
            uint64_t *d_cpre = nullptr;
            ASDM_TRY(scr.upload(&d_cps, cps));
            ASDM_TRY(scr.upload(&d_cpre, cpre));
            copy_words<<<grid_for(cpre.back(), G->num_sms), kBlock, 0, s>>>(d_cps, d_cpre, (uint32_t)cps.size());
            ::asdm::count_launch();
            ASDM_CUDA(cudaGetLastError());
        }
    }
    std::vector<uint32_t> kcount(std::max<uint32_t>(nk1, 1), 0), fcount(nseg, 0);
    ASDM_CUDA(cudaMemcpyAsync(kcount.data(), d_fcount, kcount.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    ASDM_CUDA(cudaStreamSynchronize(s));
    for (uint32_t sg = 0; sg < nseg; ++sg) fcount[sg] = kcount[k1_of[sg]];

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
    // Ctd(u) as a membership bitset per query vertex (and whether the
    // storage S(u) scanned by the reference gets the phantom vertex 0)
    std::vector<uint64_t> mword(nseg + 1, 0);
    for (uint32_t i = 0; i < nseg; ++i) mword[i + 1] = mword[i] + words[i];
    uint32_t *sbits = nullptr, *d_zero = nullptr, *d_ph = nullptr;
    ASDM_TRY(scr.alloc(&sbits, std::max<uint64_t>(mword[nseg], 1)));
    ASDM_TRY(scr.alloc(&d_zero, 1));
    ASDM_TRY(scr.alloc(&d_ph, std::max<uint32_t>(nseg, 1)));
    ASDM_CUDA(cudaMemsetAsync(d_zero, 0, sizeof(uint32_t), s));
    ASDM_CUDA(cudaMemsetAsync(d_ph, 0, std::max<uint32_t>(nseg, 1) * sizeof(uint32_t), s));
    uint64_t bit_words_read = 0;
    // a pass p -> u: pulled over u's candidates, plus the push of the phantom
    // vertex, which runs where S(p) has it (a flag the compaction of Ctd(p)
    // sets on the device: the waves run without host reads)
    auto add_pass = [&](std::vector<PullDesc> &pulls, std::vector<PassDesc> &pushes, std::vector<uint64_t> &lens,
                        const QPlan &qp, uint32_t u, uint32_t e, const uint32_t *xbits) {
        const QueryGraph &q = qp.cs->q;
        const uint32_t p = q.nbr[e], su = qp.seg0 + u, sp = qp.seg0 + p, slot = e - q.off[u];
        uint32_t *mb = bits + fword[su] + (1ull + slot) * words[su];
        pulls.push_back(PullDesc{xbits, mb, sbits + mword[sp], qp.lbase[u], q.lab[p], words[su], 0});
        bit_words_read += words[su];
        pushes.push_back(PassDesc{d_zero, mb, q.lab[u], 0, d_ph + sp});
        lens.push_back(1);
    };
    for (uint32_t w = 0; w <= maxwave; ++w) {
        std::vector<PullDesc> pulls;
        std::vector<PassDesc> pushes;
        std::vector<uint64_t> lens;
        std::vector<CompDesc> segs;
        for (const QPlan &qp : P) {
            if (qp.empty) continue;
            const QueryGraph &q = qp.cs->q;
            for (uint32_t u : qp.order) {
                if (qp.wave[u] != w) continue;
                const uint32_t su = qp.seg0 + u;
                uint32_t need = 0;
                for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                    if (qp.rank[q.nbr[e]] >= qp.rank[u]) continue;
                    need |= 1u << (e - q.off[u]);
                    add_pass(pulls, pushes, lens, qp, u, e, bits + fword[su]);  // over F(u)
                }
                segs.push_back(CompDesc{bits + fword[su], words[su], need, qp.lsize[u], qp.lbase[u], 1, 0, nullptr,
                                        sbits + mword[su], d_ph + su});
                bit_words_read += (uint64_t)(1 + __builtin_popcount(need)) * words[su];
            }
        }
        ASDM_TRY(run_pulls(G, pulls, d_elems));
        ASDM_TRY(run_passes(G, pushes, lens, d_elems));
        std::vector<uint64_t> start;
        std::vector<uint32_t> sizes;
        ASDM_TRY(compact(G, segs, nullptr, start, sizes));  // Ctd(u) bitsets and phantom flags only
    }
    // remaining passes (neighbours later in the BFS order), all queries at
    // once, over Ctd(u)
    {
        std::vector<PullDesc> pulls;
        std::vector<PassDesc> pushes;
        std::vector<uint64_t> lens;
        for (const QPlan &qp : P) {
            if (qp.empty) continue;
            const QueryGraph &q = qp.cs->q;
            for (uint32_t u = 0; u < q.n; ++u)
                for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                    if (qp.rank[q.nbr[e]] < qp.rank[u]) continue;
                    add_pass(pulls, pushes, lens, qp, u, e, sbits + mword[qp.seg0 + u]);
                }
        }
        ASDM_TRY(run_pulls(G, pulls, d_elems));
        ASDM_TRY(run_passes(G, pushes, lens, d_elems));
    }
    // final candidate sets into the group's arena, with the membership
    // bitsets and per-word prefix counts that K3 looks indices up in
    auto arena = std::make_shared<CsArena>();
    arena->stream = s;
    uint2 *cmem = nullptr;
    ASDM_TRY(scr.alloc(&cmem, mword[nseg]));
    {
        std::vector<CompDesc> segs;
        std::vector<uint32_t> seg_ids;
        for (const QPlan &qp : P) {
            if (qp.empty) continue;
            const QueryGraph &q = qp.cs->q;
            for (uint32_t u = 0; u < q.n; ++u) {
                const uint32_t all = q.deg(u) ? ((q.deg(u) == 32 ? 0xFFFFFFFFu : (1u << q.deg(u)) - 1u)) : 0u;
                const uint32_t su = qp.seg0 + u;
                segs.push_back(CompDesc{bits + fword[su], words[su], all, qp.lsize[u], qp.lbase[u], 0, 0,
                                        cmem + mword[su]});
                seg_ids.push_back(su);
                bit_words_read += (uint64_t)(1 + q.deg(u)) * words[su];
            }
        }
        std::vector<uint64_t> start;
        std::vector<uint32_t> sizes;
        ASDM_TRY(compact(G, segs, &arena->d_cand, start, sizes));
        std::vector<uint32_t> ncand(nseg, 0);
        std::vector<uint64_t> cbase(nseg, 0);
        for (size_t i = 0; i < seg_ids.size(); ++i) {
            ncand[seg_ids[i]] = sizes[i];
            cbase[seg_ids[i]] = start[i];
        }
        if (!arena->d_cand) ASDM_TRY(dalloc(&arena->d_cand, 1, s));
        for (QPlan &qp : P) {
            if (qp.empty) continue;
            asdm_cs &cs = *qp.cs;
            bool ok = true;
            for (uint32_t u = 0; u < cs.q.n; ++u) {
                cs.ncand[u] = ncand[qp.seg0 + u];
                cs.cand_base[u] = cbase[qp.seg0 + u];
                ok &= cs.ncand[u] > 0;
            }
            cs.cand_base[cs.q.n] = cs.cand_base[cs.q.n - 1] + cs.ncand[cs.q.n - 1];
            qp.empty = !ok;
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
                const uint32_t s2 = qp.seg0 + u2;
                edges.push_back(EdgeDesc{arena->d_cand + cs.cand_base[u], cmem + mword[s2], cs.ncand[u], q.lab[u2]});
                item_base.push_back(item_base.back() + cs.ncand[u] + 1);
            }
    }
    const uint32_t ne = (uint32_t)edges.size();
    const uint64_t nitems = item_base.back();
    std::vector<uint64_t> estart(ne, 0);
    bool two_scan = false;
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
        // One scan of the neighbour runs: fill into lists padded to their
        // label-run lengths (counting on the way), then pack densely; the
        // exact two-scan form (count, then fill) where the padded lists would
        // be too large.
        uint64_t bound = 0;
        uint64_t *d_upos = nullptr;
        // K3 keeps edge-major order: a warp's lanes take consecutive candidates
        // of one edge, whose ascending ids put their adjacency runs side by
        // side in the CSR (grouping by vertex block across edges measured slower)
        ASDM_TRY(scr.alloc(&d_upos, nitems + 1));
        uint32_t *rstart = nullptr;
        ASDM_TRY(scr.alloc(&rstart, nitems));
        k3_bound<<<egrid, kBlock, 0, s>>>(g, d_edges, d_ib, ne, arena->d_eoff, rstart);
        ::asdm::count_launch();
        ASDM_CUDA(cudaGetLastError());
        ASDM_TRY(scan_exclusive_u32(arena->d_eoff, d_upos, nitems, true, s));
        ASDM_CUDA(cudaMemcpyAsync(&bound, d_upos + nitems, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        ASDM_CUDA(cudaStreamSynchronize(s));
        // padded lists up to 2^padded_cap_log2 entries in total (default 2^33:
        // 32 GiB), the exact two-scan form beyond
        const uint64_t padded_cap = 1ull << G->tuning.padded_cap_log2;
        two_scan = bound > padded_cap;
        if (bound <= padded_cap) {
            uint32_t *padded = nullptr;
            ASDM_TRY(scr.alloc(&padded, bound));
            k3_flat<<<egrid, kBlock, 0, s>>>(g, d_edges, d_ib, ne, arena->d_eoff, d_upos, rstart, padded, d_elems + 1);
            ::asdm::count_launch();
            ASDM_CUDA(cudaGetLastError());
            ASDM_TRY(scan_exclusive_u32(arena->d_eoff, d_wpos, nitems, true, s));
            ASDM_CUDA(cudaMemcpyAsync(&total, d_wpos + nitems, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
            ASDM_CUDA(cudaStreamSynchronize(s));
            ASDM_TRY(dalloc(&arena->d_elist, total, s));
            k3_pack<<<grid_for(nitems, G->num_sms), kBlock, 0, s>>>(d_upos, arena->d_eoff, d_wpos, nitems, padded,
                                                                   arena->d_elist, d_ib, ne, d_estart, d_bad);
            ::asdm::count_launch();
            ASDM_CUDA(cudaGetLastError());
        } else {
            k3_edges<false><<<egrid, kBlock, 0, s>>>(g, d_edges, d_ib, ne, arena->d_eoff, nullptr, nullptr,
                                                    d_elems + 1, nullptr);
            ::asdm::count_launch();
            ASDM_CUDA(cudaGetLastError());
            ASDM_TRY(scan_exclusive_u32(arena->d_eoff, d_wpos, nitems, true, s));
            ASDM_CUDA(cudaMemcpyAsync(&total, d_wpos + nitems, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
            ASDM_CUDA(cudaStreamSynchronize(s));
            ASDM_TRY(dalloc(&arena->d_elist, total, s));
            k3_edges<true><<<egrid, kBlock, 0, s>>>(g, d_edges, d_ib, ne, nullptr, d_wpos, arena->d_elist,
                                                    nullptr, nullptr);
            ::asdm::count_launch();
            ASDM_CUDA(cudaGetLastError());
            k3_offsets<<<grid_for(nitems, G->num_sms), kBlock, 0, s>>>(d_ib, ne, d_wpos, arena->d_eoff, d_estart,
                                                                      d_bad);
            ::asdm::count_launch();
            ASDM_CUDA(cudaGetLastError());
        }
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
    // K1 reads 8 bytes per vertex of the label of each distinct query-vertex
    // signature (and copies F words for the repeats); K2 and K3 read one rank
    // per scanned neighbour; compaction reads the bitsets it ANDs; K3 writes
    // the candidate-edge lists and their offsets (4 bytes per entry)
    const uint64_t bytes = 8ull * seg.back() + 8ull * copied_words + 4ull * (elems[0] + elems[1]) +
                           4ull * bit_words_read + 4ull * total + 4ull * nitems;
    for (uint32_t qi = 0; qi < Q; ++qi) {
        QPlan &qp = P[qi];
        asdm_cs &cs = *qp.cs;
        cs.build_ms = ms / Q;
        cs.build_bytes = bytes / Q;
        cs.build_flags = (two_scan ? ASDM_CS_TWO_SCAN : 0u) | (g.lab_pos ? ASDM_CS_LABEL_RUNS : 0u);
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
