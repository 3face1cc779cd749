// Exact counts of tree-shaped queries without enumeration.
//
// Within the candidate space, a map of the query vertices to candidates that
// sends every query edge to a candidate edge is a homomorphism; it is an
// embedding when, in addition, no two query vertices of one label that are
// not adjacent land on the same data vertex (the conflict pairs the
// enumeration checks; vertices of different labels have disjoint candidate
// sets, and adjacent ones differ because the data graph has no self loops).
// For a tree query the count of homomorphisms is a bottom-up dynamic program
// over the candidate-edge lists:
//     w_u(i) = prod over children c of u of  sum over j in list_{u->c}(i) of  w_c(j)
//     hom    = sum over i of w_root(i)
// and the count of embeddings follows by inclusion-exclusion over the
// partitions pi of each label's vertices into blocks of pairwise non-adjacent
// vertices:
//     count = sum over pi of  mu(pi) * hom(Q / pi),
//     mu(pi) = prod over blocks B of (-1)^(|B|-1) (|B|-1)!
// where Q / pi identifies the vertices of each block (one data vertex for the
// whole block: a candidate of every member).  Every candidate edge is a data
// edge between candidates and every data edge between candidates is a
// candidate edge (K3 keeps all of them), so parallel edges of Q / pi are one
// constraint; a query qualifies when every such quotient is again a tree.
// (The reference reaches the same number by enumeration: adaptiveShareJoin
// with ALL_LEVEL, matching/adaptive.cpp:1179-2279.)
//
// Arithmetic is modulo 2^64.  Each hom(Q / pi) is at most hom(Q) (a
// homomorphism of the quotient composed with the quotient map is one of Q), so
// when the identity partition's program does not overflow — checked — the
// signed sum is exact.  A query whose identity program overflows is left to
// the enumeration kernels, which report ASDM_ERR_OVERFLOW if its count itself
// exceeds 2^64 - 1.
#include <algorithm>
#include <functional>

#include "cs.cuh"

namespace asdm {
namespace {

// One (query, term, block) of a height level of the programs.  A block's
// candidates are indexed like those of its representative member r (the
// member its parent edge reaches); the other members' maps C(r) -> C(member)
// (kNone where the vertex is not their candidate) zero the weights of the
// candidates outside the intersection.
struct TreeSeg {
    unsigned long long *w;       // weights of the block's candidates (output)
    uint32_t ncand;              // |C(r)|
    uint32_t child_first;        // children in the TreeChild array
    uint32_t nchild;
    uint32_t query;              // index into counts / flags
    uint32_t root;               // 1: add the weights into the query's count
    uint32_t check;              // 1: the identity partition's program (overflow checked)
    uint32_t val_first, nval;    // the other members' maps, in the map array
    long long coef;              // mu(pi) of the term
    unsigned long long start;    // first item of this segment in the launch
};

struct TreeChild {
    const uint32_t *off;              // candidate-edge offsets of (u -> c), by candidate of u
    const uint32_t *list;             // entries: indices into C(c)
    const unsigned long long *w;      // weights of c's block (null for a one-vertex leaf: all 1)
    unsigned long long *s_out;        // local counts: the sum over the list, by candidate of u (or null)
    const uint32_t *src;              // map C(r) -> C(u) when u is not the representative (else null)
};

// Local counts, top down: up_c(j) = sum over i in list_{c->u}(j) of
// up_u(i) * prod over c's siblings c' of S_{u,c'}(i), with up = 1 at the root.
struct UpSeg {
    unsigned long long *up;             // up_c (output), by candidate of c
    const uint32_t *off, *list;         // candidate edges (c -> u): for j in C(c), indices into C(u)
    const unsigned long long *up_u;     // null when u is the root
    uint32_t sib_first, nsib;           // S arrays of u's other children
    uint32_t query, ncand;
    unsigned long long start;
};

// local[v][u] = w_u(i) * up_u(i) for v = C(u)[i]
struct LocSeg {
    const unsigned long long *w, *up;   // w null at a leaf, up null at the root
    const uint32_t *cand;
    unsigned long long *local;          // |Vg| x n block of the query
    uint32_t n, u, query, ncand;
    unsigned long long start;
};

// One thread per candidate of the level's blocks; a list longer than 32
// entries is summed by the whole warp.  Sums and products wrap modulo 2^64;
// the identity partition's program flags an overflow instead.
__global__ void tree_level(const TreeSeg *__restrict__ segs, uint32_t nseg, unsigned long long total,
                           const TreeChild *__restrict__ kids, const uint32_t *const *__restrict__ maps,
                           unsigned long long *__restrict__ counts, unsigned long long *__restrict__ homs,
                           unsigned int *__restrict__ overflow) {
    const uint32_t lane = threadIdx.x & 31;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total;
         base += stride) {
        const unsigned long long t = base + lane;
        const bool valid = t < total;
        TreeSeg sg{};
        uint32_t i = 0, seg = 0xFFFFFFFFu;
        bool alive = valid;
        if (valid) {
            uint32_t lo = 0, hi = nseg;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (segs[mid].start <= t) lo = mid; else hi = mid;
            }
            seg = lo;
            sg = segs[lo];
            i = (uint32_t)(t - sg.start);
            for (uint32_t k = 0; k < sg.nval && alive; ++k) alive = maps[sg.val_first + k][i] != kNone;
        }
        unsigned long long acc = alive ? 1ull : 0ull;
        bool over = false;
        // children are visited in lock step: k-th child of every lane's segment
        uint32_t maxk = alive ? sg.nchild : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) maxk = max(maxk, __shfl_xor_sync(0xffffffffu, maxk, o));
        for (uint32_t k = 0; k < maxk; ++k) {
            const bool mine = alive && k < sg.nchild;
            uint32_t b = 0, e = 0;
            const unsigned long long *w = nullptr;
            const uint32_t *list = nullptr;
            if (mine) {
                const TreeChild ch = kids[sg.child_first + k];
                const uint32_t iu = ch.src ? ch.src[i] : i;
                b = ch.off[iu];
                e = ch.off[iu + 1];
                w = ch.w;
                list = ch.list;
            }
            // a one-vertex leaf child contributes its list length
            unsigned long long sum = (mine && !w) ? (unsigned long long)(e - b) : 0ull;
            const bool coop = mine && w && (e - b) > 32;
            uint32_t todo = __ballot_sync(0xffffffffu, coop);
            while (todo) {
                const int src = __ffs(todo) - 1;
                todo &= todo - 1;
                const uint32_t bb = __shfl_sync(0xffffffffu, b, src), ee = __shfl_sync(0xffffffffu, e, src);
                const unsigned long long *ww =
                    (const unsigned long long *)__shfl_sync(0xffffffffu, (unsigned long long)w, src);
                const uint32_t *ll = (const uint32_t *)__shfl_sync(0xffffffffu, (unsigned long long)list, src);
                unsigned long long part = 0;
                bool pover = false;
#pragma unroll 4
                for (uint32_t x = bb + lane; x < ee; x += 32) {
                    const unsigned long long v = ww[ll[x]];
                    pover |= part + v < part;
                    part += v;
                }
#pragma unroll
                for (int o = 16; o; o >>= 1) {
                    const unsigned long long y = __shfl_xor_sync(0xffffffffu, part, o);
                    pover |= part + y < part;
                    part += y;
                }
                pover = __any_sync(0xffffffffu, pover);
                if ((int)lane == src) {
                    sum = part;
                    over |= pover;
                }
            }
            if (mine && w && !coop)
#pragma unroll 4
                for (uint32_t x = b; x < e; ++x) {
                    const unsigned long long v = w[list[x]];
                    over |= sum + v < sum;
                    sum += v;
                }
            if (mine) {
                unsigned long long *so = kids[sg.child_first + k].s_out;
                if (so) so[i] = sum;
                over |= __umul64hi(acc, sum) != 0;
                acc *= sum;
            }
        }
        if (valid) {
            if (over && sg.check) {
                atomicOr(&overflow[sg.query], 1u);
                acc = 0;
            }
            sg.w[i] = acc;
        }
        // root weights: summed over each segment's lanes (a segment's lanes
        // are contiguous), then one atomic per segment and warp
        const bool root = valid && sg.root;
        if (__any_sync(0xffffffffu, root)) {
            const uint32_t key = root ? seg : 0xFFFFFFFFu;
            unsigned long long v = root ? (unsigned long long)sg.coef * acc : 0ull;
            unsigned long long h = (root && sg.check) ? acc : 0ull;
            bool ov = false;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long yv = __shfl_down_sync(0xffffffffu, v, o);
                const unsigned long long yh = __shfl_down_sync(0xffffffffu, h, o);
                const bool yo = __shfl_down_sync(0xffffffffu, ov, o);
                const uint32_t yk = __shfl_down_sync(0xffffffffu, key, o);
                if (lane + o < 32 && yk == key) {
                    v += yv;
                    ov |= yo || h + yh < h;
                    h += yh;
                }
            }
            const uint32_t prev = __shfl_up_sync(0xffffffffu, key, 1);
            if (root && (lane == 0 || prev != key)) {
                if (v) atomicAdd(&counts[sg.query], v);
                if (sg.check) {
                    const unsigned long long old = h ? atomicAdd(&homs[sg.query], h) : 0ull;
                    if (ov || old + h < old) atomicOr(&overflow[sg.query], 1u);
                }
            }
        }
    }
}

__device__ __forceinline__ uint32_t seg_of(const unsigned long long *starts_base, size_t stride_bytes, uint32_t nseg,
                                           unsigned long long t) {
    uint32_t lo = 0, hi = nseg;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        const unsigned long long st =
            *reinterpret_cast<const unsigned long long *>(reinterpret_cast<const char *>(starts_base) + mid * stride_bytes);
        if (st <= t) lo = mid; else hi = mid;
    }
    return lo;
}

__global__ void tree_up(const UpSeg *__restrict__ segs, uint32_t nseg, unsigned long long total,
                        const unsigned long long *const *__restrict__ sibs, unsigned int *__restrict__ overflow) {
    for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        const UpSeg sg = segs[seg_of(&segs[0].start, sizeof(UpSeg), nseg, t)];
        const uint32_t j = (uint32_t)(t - sg.start);
        unsigned long long sum = 0;
        bool over = false;
        for (uint32_t e = sg.off[j]; e < sg.off[j + 1]; ++e) {
            const uint32_t i = sg.list[e];
            unsigned long long x = sg.up_u ? sg.up_u[i] : 1ull;
            for (uint32_t k = 0; k < sg.nsib && x; ++k) {
                const unsigned long long y = sibs[sg.sib_first + k][i];
                over |= __umul64hi(x, y) != 0;
                x *= y;
            }
            over |= sum + x < sum;
            sum += x;
        }
        if (over) {
            atomicOr(&overflow[sg.query], 1u);
            sum = 0;
        }
        sg.up[j] = sum;
    }
}

__global__ void tree_local(const LocSeg *__restrict__ segs, uint32_t nseg, unsigned long long total,
                           unsigned int *__restrict__ overflow) {
    for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        const LocSeg sg = segs[seg_of(&segs[0].start, sizeof(LocSeg), nseg, t)];
        const uint32_t i = (uint32_t)(t - sg.start);
        const unsigned long long a = sg.w ? sg.w[i] : 1ull, b = sg.up ? sg.up[i] : 1ull;
        if (__umul64hi(a, b) != 0) atomicOr(&overflow[sg.query], 1u);
        sg.local[(unsigned long long)sg.cand[i] * sg.n + sg.u] = a * b;
    }
}

// C(r) -> C(u) for the members u of merged blocks: index in C(u) of each
// candidate of r, or kNone.
struct MapSeg {
    const uint32_t *from, *to;
    uint32_t *out;
    uint32_t nto, pad;
    unsigned long long start;
};

__global__ void tree_maps(const MapSeg *__restrict__ segs, uint32_t nseg, unsigned long long total) {
    for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        const MapSeg sg = segs[seg_of(&segs[0].start, sizeof(MapSeg), nseg, t)];
        const uint32_t v = sg.from[t - sg.start];
        const uint32_t j = lower_bound_u32(sg.to, sg.nto, v);
        sg.out[t - sg.start] = (j < sg.nto && sg.to[j] == v) ? j : kNone;
    }
}

constexpr size_t kMaxPartitions = 4096;  // partitions generated for one query
constexpr size_t kMaxTerms = 64;         // terms counted for one query

// One term of the inclusion-exclusion: a partition of the query vertices
// into blocks, its quotient rooted at one block.
struct BlockTree {
    long long coef = 1;
    bool identity = true;                         // every block one vertex (block b = vertex b)
    uint32_t nb = 0;
    std::vector<uint32_t> block;                  // by vertex
    std::vector<std::vector<uint32_t>> members;   // by block, ascending
    std::vector<uint32_t> rep;                    // representative member
    std::vector<uint32_t> parent;                 // parent block (kNone at the root)
    std::vector<uint32_t> pedge;                  // query edge (pfrom -> rep) from the parent block
    std::vector<uint32_t> pfrom;                  // the parent block's member it leaves from
    std::vector<uint32_t> height, depth;
};

// Roots the quotient of t's partition at the block of vertex `root`
// (its representative); false when the quotient is not a tree.
bool root_quotient(const QueryGraph &q, BlockTree &t, uint32_t root = 0) {
    std::vector<std::pair<uint32_t, uint32_t>> qe;
    for (uint32_t u = 0; u < q.n; ++u)
        for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
            const uint32_t a = t.block[u], b = t.block[q.nbr[e]];
            if (a == b) return false;
            if (a < b) qe.emplace_back(a, b);
        }
    std::sort(qe.begin(), qe.end());
    qe.erase(std::unique(qe.begin(), qe.end()), qe.end());
    if (qe.size() + 1 != t.nb) return false;
    t.rep.assign(t.nb, kNone);
    t.parent.assign(t.nb, kNone);
    t.pedge.assign(t.nb, kNone);
    t.pfrom.assign(t.nb, kNone);
    t.height.assign(t.nb, 0);
    t.depth.assign(t.nb, 0);
    std::vector<uint32_t> order{t.block[root]};
    t.rep[t.block[root]] = root;
    for (size_t k = 0; k < order.size(); ++k) {
        const uint32_t B = order[k];
        for (uint32_t u : t.members[B])
            for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                const uint32_t w = q.nbr[e], C = t.block[w];
                if (C == B || t.rep[C] != kNone) continue;
                t.rep[C] = w;
                t.parent[C] = B;
                t.pedge[C] = e;
                t.pfrom[C] = u;
                t.depth[C] = t.depth[B] + 1;
                order.push_back(C);
            }
    }
    if (order.size() != t.nb) return false;
    for (size_t k = order.size(); k-- > 1;) {
        const uint32_t C = order[k], B = t.parent[C];
        t.height[B] = std::max(t.height[B], t.height[C] + 1);
    }
    return true;
}

// Device work of a rooted term: one item per candidate of every block that
// is not a one-vertex leaf, and one per entry of the lists summed into its
// parent (a one-vertex leaf's parent takes the list length).
uint64_t term_cost(const BlockTree &t, const asdm_cs &c) {
    uint64_t cost = 0;
    for (uint32_t b = 0; b < t.nb; ++b) {
        if (t.height[b] == 0 && t.members[b].size() == 1) continue;
        cost += c.ncand[t.rep[b]];
        if (t.parent[b] != kNone) cost += c.etotal[t.pedge[b]];
    }
    return cost;
}

// Every term of a tree query's count; false when the query does not qualify
// (not a tree, a quotient with a cycle, too many partitions).  With a built
// candidate space each term is rooted where its program reads the fewest
// list entries.
bool block_trees(const QueryGraph &q, std::vector<BlockTree> &out, const asdm_cs *cs = nullptr) {
    out.clear();
    if (q.n < 2 || q.off[q.n] != 2 * (q.n - 1)) return false;
    std::vector<uint32_t> block(q.n, kNone);
    std::vector<std::vector<uint32_t>> members;
    size_t generated = 0;
    bool ok = true;
    // vertex u joins a block of its label with no neighbour of u, or opens one
    std::function<void(uint32_t)> place = [&](uint32_t u) {
        if (!ok) return;
        if (u == q.n) {
            if (++generated > kMaxPartitions) { ok = false; return; }
            BlockTree t;
            t.nb = (uint32_t)members.size();
            t.block = block;
            t.members = members;
            for (const auto &m : members) {
                long long f = 1;
                for (size_t k = 2; k < m.size(); ++k) f *= (long long)k;
                t.coef *= (m.size() % 2 == 0) ? -f : f;
                t.identity = t.identity && m.size() == 1;
            }
            if (!root_quotient(q, t) || out.size() >= kMaxTerms) { ok = false; return; }
            if (cs) {
                BlockTree best = t;
                uint64_t best_cost = term_cost(t, *cs);
                for (uint32_t r = 1; r < q.n; ++r) {
                    if (t.members[t.block[r]][0] != r) continue;  // one root per block: its first member
                    BlockTree alt = t;
                    if (!root_quotient(q, alt, r)) continue;
                    const uint64_t cost = term_cost(alt, *cs);
                    if (cost < best_cost) { best_cost = cost; best = std::move(alt); }
                }
                t = std::move(best);
            }
            out.push_back(std::move(t));
            return;
        }
        for (uint32_t b = 0; b < members.size() && ok; ++b) {
            if (q.lab[members[b][0]] != q.lab[u]) continue;
            bool adj = false;
            for (uint32_t w : members[b]) adj = adj || q.slot(u, w) >= 0;
            if (adj) continue;
            members[b].push_back(u);
            block[u] = b;
            place(u + 1);
            members[b].pop_back();
        }
        if (!ok) return;
        block[u] = (uint32_t)members.size();
        members.push_back({u});
        place(u + 1);
        members.pop_back();
    };
    place(0);
    if (!ok) out.clear();
    return ok;
}

}  // namespace

// A query whose count (and local counts) the program gives with the identity
// partition alone: connected tree, no two non-adjacent vertices with one label.
bool tree_countable(const QueryGraph &q) {
    if (q.n < 2 || q.off[q.n] != 2 * (q.n - 1)) return false;
    for (uint32_t u = 0; u < q.n; ++u)
        for (uint32_t w = u + 1; w < q.n; ++w)
            if (q.lab[u] == q.lab[w] && q.slot(u, w) < 0) return false;
    return true;
}

// A tree query whose count the program gives by inclusion-exclusion: every
// quotient by same-label blocks is a tree (always so when the same-label
// vertices are at distance 2: siblings, or grandparent and grandchild).
bool tree_countable_conflicts(const QueryGraph &q) {
    std::vector<BlockTree> t;
    return block_trees(q, t);
}

// Counts every countable query of `cs` (non-empty candidate spaces on graph
// G); done[i] = 1 and counts[i] set for the queries it settled.  With local
// counts only queries without conflicts are taken.
int tree_counts(asdm_graph *G, const std::vector<asdm_cs *> &cs, std::vector<uint64_t> &counts,
                std::vector<char> &done, const std::vector<unsigned long long *> *local) {
    cudaStream_t s = G->stream;
    const uint32_t Q = (uint32_t)cs.size();
    counts.assign(Q, 0);
    done.assign(Q, 0);
    // (query, term, block) grouped by the block's height (and depth)
    struct Item { uint32_t q, t, b; };
    std::vector<std::vector<Item>> by_height, by_depth;
    std::vector<std::vector<BlockTree>> trees(Q);
    std::vector<std::vector<std::vector<uint64_t>>> woff(Q);  // first weight of (query, term, block)
    uint64_t wtotal = 0;
    std::vector<uint32_t> take;
    // maps C(rep) -> C(member) of merged blocks, one per (query, rep, member)
    std::vector<MapSeg> msegs;
    std::vector<std::vector<std::pair<uint64_t, uint32_t>>> mkey(Q);  // ((rep << 32) | member, seg)
    uint64_t mtotal = 0;
    for (uint32_t qi = 0; qi < Q; ++qi) {
        const asdm_cs &c = *cs[qi];
        if (!c.nonempty || !block_trees(c.q, trees[qi], &c)) continue;
        if (local && trees[qi].size() != 1) continue;
        woff[qi].resize(trees[qi].size());
        for (uint32_t ti = 0; ti < trees[qi].size(); ++ti) {
            const BlockTree &t = trees[qi][ti];
            woff[qi][ti].resize(t.nb);
            for (uint32_t b = 0; b < t.nb; ++b) {
                woff[qi][ti][b] = wtotal;
                wtotal += c.ncand[t.rep[b]];
                if (by_height.size() <= t.height[b]) by_height.resize(t.height[b] + 1);
                by_height[t.height[b]].push_back(Item{qi, ti, b});
                if (by_depth.size() <= t.depth[b]) by_depth.resize(t.depth[b] + 1);
                by_depth[t.depth[b]].push_back(Item{qi, ti, b});
                for (uint32_t u : t.members[b]) {
                    if (u == t.rep[b]) continue;
                    const uint64_t key = ((uint64_t)t.rep[b] << 32) | u;
                    bool have = false;
                    for (auto &kv : mkey[qi]) have = have || kv.first == key;
                    if (have) continue;
                    mkey[qi].emplace_back(key, (uint32_t)msegs.size());
                    msegs.push_back(MapSeg{c.d_cand + c.cand_base[t.rep[b]], c.d_cand + c.cand_base[u], nullptr,
                                           c.ncand[u], 0, mtotal});
                    mtotal += c.ncand[t.rep[b]];
                }
            }
        }
        take.push_back(qi);
    }
    if (take.empty()) return ASDM_OK;
    auto is_leaf1 = [&](uint32_t qi, uint32_t ti, uint32_t b) {
        const BlockTree &t = trees[qi][ti];
        return t.height[b] == 0 && t.members[b].size() == 1;
    };
    auto wptr_off = [&](uint32_t qi, uint32_t u) { return woff[qi][0][u]; };  // identity term: block = vertex
    // S_{parent(c), c} has |C(parent)| entries, at sslot[query][c]
    std::vector<std::vector<uint64_t>> sslot(Q);
    uint64_t stotal = 0;
    if (local) {
        for (uint32_t qi : take) sslot[qi].assign(cs[qi]->q.n, 0);
        for (const auto &lv : by_height)
            for (const Item &it : lv) {
                const uint32_t par = trees[it.q][it.t].parent[it.b];
                if (par != kNone) {
                    sslot[it.q][it.b] = stotal;
                    stotal += cs[it.q]->ncand[par];
                }
            }
    }
    unsigned long long *sbase = nullptr;
    auto s_of = [&](uint32_t qi, uint32_t ch) { return sbase + sslot[qi][ch]; };
    unsigned long long *w = nullptr, *d_counts = nullptr, *d_homs = nullptr, *sums = nullptr, *up = nullptr;
    unsigned int *d_over = nullptr;
    uint32_t *d_mapbuf = nullptr;
    TreeSeg *d_segs = nullptr;
    TreeChild *d_kids = nullptr;
    MapSeg *d_mseg = nullptr;
    const uint32_t **d_maps = nullptr;
    UpSeg *d_up = nullptr;
    LocSeg *d_loc = nullptr;
    const unsigned long long **d_sibs = nullptr;
    // local counts: the list sums S_{u,c} (one array per tree edge, by
    // candidate of the parent u) and up_u (laid out like the weights)
    int rc = ASDM_OK;
    do {
        if ((rc = dalloc(&w, wtotal, s)) || (rc = dalloc(&d_counts, 2ull * Q, s)) || (rc = dalloc(&d_over, Q, s)))
            break;
        d_homs = d_counts + Q;
        if (local && ((rc = dalloc(&sums, std::max<uint64_t>(stotal, 1), s)) || (rc = dalloc(&up, wtotal, s)))) break;
        sbase = sums;
        if (cudaMemsetAsync(d_counts, 0, 2ull * Q * sizeof(unsigned long long), s) != cudaSuccess ||
            cudaMemsetAsync(d_over, 0, Q * sizeof(unsigned int), s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "tree-count reset failed");
            break;
        }
        // member maps of merged blocks
        std::vector<const uint32_t *> maps;
        if (mtotal) {
            if ((rc = dalloc(&d_mapbuf, mtotal, s)) || (rc = dalloc(&d_mseg, msegs.size(), s))) break;
            for (auto &m : msegs) m.out = d_mapbuf + m.start;
            if (cudaMemcpyAsync(d_mseg, msegs.data(), msegs.size() * sizeof(MapSeg), cudaMemcpyHostToDevice, s) !=
                cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "tree-count map upload failed");
                break;
            }
            const unsigned grid =
                (unsigned)std::min<unsigned long long>((mtotal + 255) / 256, (unsigned long long)G->num_sms * 32);
            tree_maps<<<grid, 256, 0, s>>>(d_mseg, (uint32_t)msegs.size(), mtotal);
            ::asdm::count_launch();
            if (cudaGetLastError() != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "tree-count map kernel failed");
                break;
            }
        }
        auto map_of = [&](uint32_t qi, uint32_t r, uint32_t u) -> const uint32_t * {
            const uint64_t key = ((uint64_t)r << 32) | u;
            for (auto &kv : mkey[qi])
                if (kv.first == key) return msegs[kv.second].out;
            return nullptr;
        };
        // every level's segments and children, uploaded once
        std::vector<TreeSeg> segs;
        std::vector<TreeChild> kids;
        std::vector<size_t> lvl_first{0};
        std::vector<unsigned long long> lvl_total;
        for (size_t h = 0; h < by_height.size(); ++h) {
            unsigned long long total = 0;
            for (const Item &it : by_height[h]) {
                if (is_leaf1(it.q, it.t, it.b)) continue;  // weighs 1: its parent takes the list length
                const asdm_cs &c = *cs[it.q];
                const QueryGraph &q = c.q;
                const BlockTree &t = trees[it.q][it.t];
                const uint32_t r = t.rep[it.b];
                TreeSeg sg{};
                sg.w = w + woff[it.q][it.t][it.b];
                sg.ncand = c.ncand[r];
                sg.child_first = (uint32_t)kids.size();
                sg.query = it.q;
                sg.root = t.parent[it.b] == kNone ? 1u : 0u;
                sg.check = t.identity ? 1u : 0u;
                sg.coef = t.coef;
                sg.val_first = (uint32_t)maps.size();
                for (uint32_t u : t.members[it.b])
                    if (u != r) maps.push_back(map_of(it.q, r, u));
                sg.nval = (uint32_t)maps.size() - sg.val_first;
                sg.start = total;
                for (uint32_t C = 0; C < t.nb; ++C) {
                    if (t.parent[C] != it.b) continue;
                    const uint32_t e = t.pedge[C], u = t.pfrom[C];
                    kids.push_back(TreeChild{c.d_eoff + c.eoff_base[e], c.d_elist + c.elist_base[e],
                                             is_leaf1(it.q, it.t, C) ? nullptr : w + woff[it.q][it.t][C],
                                             local ? s_of(it.q, C) : nullptr, u == r ? nullptr : map_of(it.q, r, u)});
                }
                (void)q;
                sg.nchild = (uint32_t)kids.size() - sg.child_first;
                total += sg.ncand;
                segs.push_back(sg);
            }
            lvl_first.push_back(segs.size());
            lvl_total.push_back(total);
        }
        if (kids.empty()) kids.push_back(TreeChild{});
        if (maps.empty()) maps.push_back(nullptr);
        if (segs.empty()) segs.push_back(TreeSeg{});
        if ((rc = dalloc(&d_segs, segs.size(), s)) || (rc = dalloc(&d_kids, kids.size(), s)) ||
            (rc = dalloc(&d_maps, maps.size(), s)))
            break;
        if (cudaMemcpyAsync(d_segs, segs.data(), segs.size() * sizeof(TreeSeg), cudaMemcpyHostToDevice, s) !=
                cudaSuccess ||
            cudaMemcpyAsync(d_kids, kids.data(), kids.size() * sizeof(TreeChild), cudaMemcpyHostToDevice, s) !=
                cudaSuccess ||
            cudaMemcpyAsync(d_maps, maps.data(), maps.size() * sizeof(void *), cudaMemcpyHostToDevice, s) !=
                cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "tree-count upload failed");
            break;
        }
        for (size_t h = 0; h < by_height.size() && rc == ASDM_OK; ++h) {
            const unsigned long long total = lvl_total[h];
            if (total == 0) continue;
            const unsigned grid =
                (unsigned)std::min<unsigned long long>((total + 255) / 256, (unsigned long long)G->num_sms * 32);
            tree_level<<<grid, 256, 0, s>>>(d_segs + lvl_first[h], (uint32_t)(lvl_first[h + 1] - lvl_first[h]),
                                            total, d_kids, d_maps, d_counts, d_homs, d_over);
            ::asdm::count_launch();
            if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "tree-count kernel failed");
        }
        if (rc != ASDM_OK) break;
        std::vector<UpSeg> ups;
        std::vector<const unsigned long long *> sibs;
        std::vector<size_t> dfirst{0};
        std::vector<unsigned long long> dtotal;
        std::vector<LocSeg> locs;
        unsigned long long ltotal = 0;
        if (local) {
            // top down, one launch per depth
            for (size_t dpt = 1; dpt < by_depth.size(); ++dpt) {
                unsigned long long total = 0;
                for (const Item &it : by_depth[dpt]) {
                    // identity terms only: block b is vertex b
                    const asdm_cs &c = *cs[it.q];
                    const QueryGraph &q = c.q;
                    const std::vector<uint32_t> &par = trees[it.q][0].parent;
                    const uint32_t u = par[it.b];
                    const int k = q.slot(it.b, u);  // edge (c -> u)
                    const uint32_t e = q.off[it.b] + (uint32_t)k;
                    UpSeg sg{};
                    sg.up = up + wptr_off(it.q, it.b);
                    sg.off = c.d_eoff + c.eoff_base[e];
                    sg.list = c.d_elist + c.elist_base[e];
                    sg.up_u = par[u] == kNone ? nullptr : up + wptr_off(it.q, u);
                    sg.sib_first = (uint32_t)sibs.size();
                    for (uint32_t e2 = q.off[u]; e2 < q.off[u + 1]; ++e2) {
                        const uint32_t c2 = q.nbr[e2];
                        if (par[c2] == u && c2 != it.b) sibs.push_back(s_of(it.q, c2));
                    }
                    sg.nsib = (uint32_t)sibs.size() - sg.sib_first;
                    sg.query = it.q;
                    sg.ncand = c.ncand[it.b];
                    sg.start = total;
                    total += sg.ncand;
                    ups.push_back(sg);
                }
                dfirst.push_back(ups.size());
                dtotal.push_back(total);
            }
            for (uint32_t qi : take) {
                const asdm_cs &c = *cs[qi];
                for (uint32_t u = 0; u < c.q.n; ++u) {
                    const bool root = trees[qi][0].parent[u] == kNone;
                    LocSeg ls{is_leaf1(qi, 0, u) ? nullptr : w + wptr_off(qi, u), root ? nullptr : up + wptr_off(qi, u),
                              c.d_cand + c.cand_base[u], (*local)[qi], c.q.n, u, qi, c.ncand[u], ltotal};
                    ltotal += c.ncand[u];
                    locs.push_back(ls);
                }
            }
            if (sibs.empty()) sibs.push_back(nullptr);
            if (ups.empty()) ups.push_back(UpSeg{});
            if ((rc = dalloc(&d_up, ups.size(), s)) || (rc = dalloc(&d_sibs, sibs.size(), s)) ||
                (rc = dalloc(&d_loc, locs.size(), s)))
                break;
            if (cudaMemcpyAsync(d_up, ups.data(), ups.size() * sizeof(UpSeg), cudaMemcpyHostToDevice, s) !=
                    cudaSuccess ||
                cudaMemcpyAsync(d_sibs, sibs.data(), sibs.size() * sizeof(void *), cudaMemcpyHostToDevice, s) !=
                    cudaSuccess ||
                cudaMemcpyAsync(d_loc, locs.data(), locs.size() * sizeof(LocSeg), cudaMemcpyHostToDevice, s) !=
                    cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "tree local-count upload failed");
                break;
            }
            for (size_t k = 0; k < dtotal.size() && rc == ASDM_OK; ++k) {
                if (!dtotal[k]) continue;
                const unsigned grid = (unsigned)std::min<unsigned long long>((dtotal[k] + 255) / 256,
                                                                             (unsigned long long)G->num_sms * 32);
                tree_up<<<grid, 256, 0, s>>>(d_up + dfirst[k], (uint32_t)(dfirst[k + 1] - dfirst[k]), dtotal[k], d_sibs,
                                             d_over);
                ::asdm::count_launch();
                if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "tree local-count kernel failed");
            }
            if (rc == ASDM_OK && ltotal) {
                const unsigned grid = (unsigned)std::min<unsigned long long>((ltotal + 255) / 256,
                                                                             (unsigned long long)G->num_sms * 32);
                tree_local<<<grid, 256, 0, s>>>(d_loc, (uint32_t)locs.size(), ltotal, d_over);
                ::asdm::count_launch();
                if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "tree local-count kernel failed");
            }
            if (rc != ASDM_OK) break;
        }
        std::vector<unsigned long long> hc(Q);
        std::vector<unsigned int> ho(Q);
        if (cudaMemcpyAsync(hc.data(), d_counts, Q * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaMemcpyAsync(ho.data(), d_over, Q * sizeof(unsigned int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "tree-count readback failed");
            break;
        }
        for (uint32_t qi : take)
            if (!ho[qi]) {
                counts[qi] = hc[qi];
                done[qi] = 1;
            }
    } while (false);
    dfree(d_segs, s);
    dfree(d_kids, s);
    dfree(d_maps, s);
    dfree(d_mseg, s);
    dfree(d_mapbuf, s);
    dfree(d_up, s);
    dfree(d_sibs, s);
    dfree(d_loc, s);
    dfree(sums, s);
    dfree(up, s);
    dfree(w, s);
    dfree(d_counts, s);
    dfree(d_over, s);
    if (rc != ASDM_OK) {
        done.assign(Q, 0);
        cudaStreamSynchronize(s);
    }
    return rc;
}

}  // namespace asdm
