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
// list entries.  With classes (cls[u]: u's class, or kNone when u may take
// any candidate), vertices of different classes never share a block: they
// can never share a data vertex.
bool block_trees(const QueryGraph &q, std::vector<BlockTree> &out, const asdm_cs *cs = nullptr,
                 const std::vector<uint32_t> *cls = nullptr) {
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
            for (uint32_t w : members[b])
                adj = adj || q.slot(u, w) >= 0 ||
                      (cls && (*cls)[u] != kNone && (*cls)[w] != kNone && (*cls)[u] != (*cls)[w]);
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

namespace {

// tree_counts for one chunk of queries (all of whose device state is
// allocated at once).
int tree_counts_chunk(asdm_graph *G, const std::vector<asdm_cs *> &cs, std::vector<uint64_t> &counts,
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

// Device words (weights and member maps) a query's tree program needs, or 0
// when it does not qualify.
uint64_t tree_words(const asdm_cs &c) {
    std::vector<BlockTree> t;
    if (!c.nonempty || !block_trees(c.q, t)) return 0;
    uint64_t w = 0;
    for (const BlockTree &bt : t)
        for (uint32_t b = 0; b < bt.nb; ++b) w += c.ncand[bt.rep[b]] * (1 + bt.members[b].size());
    return w;
}

constexpr uint64_t kTreeChunkWords = 1ull << 28;  // 2 GiB of weights per launch group

// ---------------------------------------------------------------------------
// Overflow proofs.
//
// A count at or above 2^64 cannot be reported, only flagged (ASDM_ERR_OVERFLOW);
// enumerating that many matches to see the counter wrap is out of reach.  A
// lower bound settles it instead: for a query Q,
//   1. every label's query vertices get classes, a proper colouring of their
//      conflict graph (same label, not adjacent), and query vertex u may only
//      take candidates of its class (class = a hash of the vertex id modulo
//      the label's class count).  Conflicting vertices then have disjoint
//      candidate sets, so every homomorphism that respects the classes is an
//      embedding;
//   2. a feedback vertex set F of Q (greedy: peel leaves, take the vertex of
//      highest remaining degree, repeat) is fixed to one candidate each: the
//      candidate of its class with the largest data degree.  Each vertex f of
//      F becomes a leaf copy under each of its other neighbours, whose weight
//      is 1 at f's fixed candidate and 0 elsewhere; edges inside F are checked
//      between the fixed candidates;
//   3. Q minus F is a forest; each component's homomorphism count (with the
//      copies) is the tree program's bottom-up product of sums.
// The product over components counts a subset of Q's embeddings (those with
// the fixed images and the classes), so it is a lower bound of the count.  It
// is computed in doubles with every sum and product rounded toward zero
// (__dadd_rz, __dmul_rz): all operands are non-negative, so every stored value
// is at most the exact one, and a final bound of at least 2^64 proves
// count >= 2^64.
// (No counterpart in the reference, whose ALL_LEVEL count is a size_t that
// wraps silently: matching/join.cpp:1017-1097.)

constexpr uint32_t kMaxFixed = 6;  // largest feedback vertex set tried

// Feedback vertex set of q, greedily: peel vertices of degree <= 1, fix the
// one of highest remaining degree (the lowest id among equals), repeat.
void greedy_fvs(const QueryGraph &q, std::vector<char> &fixed, std::vector<uint32_t> &fvs) {
    const uint32_t n = q.n;
    fixed.assign(n, 0);
    fvs.clear();
    std::vector<char> gone(n, 0);
    std::vector<uint32_t> deg(n);
    for (uint32_t u = 0; u < n; ++u) deg[u] = q.deg(u);
    for (;;) {
        bool changed = true;
        while (changed) {
            changed = false;
            for (uint32_t u = 0; u < n; ++u)
                if (!gone[u] && deg[u] <= 1) {
                    gone[u] = 1;
                    changed = true;
                    for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e)
                        if (!gone[q.nbr[e]]) --deg[q.nbr[e]];
                }
        }
        uint32_t best = kNone;
        for (uint32_t u = 0; u < n; ++u)
            if (!gone[u] && (best == kNone || deg[u] > deg[best])) best = u;
        if (best == kNone) break;
        fixed[best] = 1;
        fvs.push_back(best);
        gone[best] = 1;
        for (uint32_t e = q.off[best]; e < q.off[best + 1]; ++e)
            if (!gone[q.nbr[e]]) --deg[q.nbr[e]];
    }
}

// Class of data vertex v among k classes (a multiplicative hash of its id).
__device__ __forceinline__ uint32_t vertex_class(uint32_t v, uint32_t k) {
    return (uint32_t)((((unsigned long long)v * 0x9E3779B97F4A7C15ull) >> 32) % k);
}

// A query vertex (or block of same-label vertices) of a lower-bound program:
// its weights over C(rep), rounded toward zero, or up (up = 1) where the
// program's result enters a bound with a negative sign.
struct BoundSeg {
    double *w;
    const uint32_t *cand;       // C(rep), for the class test
    uint32_t ncand, cls_k, cls_c;
    uint32_t child_first, nchild, up;
    uint32_t val_first, nval;   // maps C(rep) -> C(member) of the block's other members
    unsigned long long start;   // first item of this segment in the launch
    const uint32_t *pin;        // when set: only the data vertex pin_cand[*pin] (none when *pin is kNone)
    const uint32_t *pin_cand;
};

struct BoundChild {
    const uint32_t *off, *list;  // candidate edges u -> c
    const double *w;             // c's weights, or null (every candidate of c weighs 1)
    const uint32_t *src;         // map C(rep) -> C(u) when the edge leaves another member u (else null)
};

__device__ __forceinline__ double dadd(double a, double b, bool up) { return up ? __dadd_ru(a, b) : __dadd_rz(a, b); }
__device__ __forceinline__ double dmul(double a, double b, bool up) { return up ? __dmul_ru(a, b) : __dmul_rz(a, b); }

// One thread per candidate of the level's segments:
//   w_u(i) = [C(u)[i] has u's class, is the pinned vertex if u is pinned, and
//             is a candidate of every member] *
//            prod over children c of sum over j in list_{u->c}(i) of w_c(j),
// rounded toward zero (or up); lists longer than 32 entries are summed by the warp.
__global__ void bound_level(const BoundSeg *__restrict__ segs, uint32_t nseg, unsigned long long total,
                            const BoundChild *__restrict__ kids, const uint32_t *const *__restrict__ maps) {
    const uint32_t lane = threadIdx.x & 31;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total;
         base += stride) {
        const unsigned long long t = base + lane;
        const bool valid = t < total;
        BoundSeg sg{};
        uint32_t i = 0;
        bool alive = valid;
        // the segment of t (the last one starting at or before it): the warp's
        // first item is located once, 32 probes per round; a lane whose item
        // lies past that segment searches on from there
        uint32_t lo = 0, hi = nseg;
        while (hi - lo > 32) {
            const uint32_t step = (hi - lo + 31) / 32;
            const uint32_t p = lo + lane * step;
            const uint32_t m = __ballot_sync(0xffffffffu, p < hi && segs[p].start <= base);
            const uint32_t nlo = lo + (31 - __clz(m)) * step;
            hi = min(hi, nlo + step);
            lo = nlo;
        }
        lo += 31 - __clz(__ballot_sync(0xffffffffu, lo + lane < hi && segs[lo + lane].start <= base));
        if (valid && lo + 1 < nseg && segs[lo + 1].start <= t) {
            hi = nseg;
            ++lo;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (segs[mid].start <= t) lo = mid; else hi = mid;
            }
        }
        if (valid) {
            sg = segs[lo];
            i = (uint32_t)(t - sg.start);
            if (sg.cls_k > 1) alive = vertex_class(sg.cand[i], sg.cls_k) == sg.cls_c;
            if (sg.pin) {
                const uint32_t h = *sg.pin;
                alive = alive && h != kNone && sg.cand[i] == sg.pin_cand[h];
            }
            for (uint32_t k = 0; k < sg.nval && alive; ++k) alive = maps[sg.val_first + k][i] != kNone;
        }
        const bool up = sg.up != 0;
        double acc = alive ? 1.0 : 0.0;
        uint32_t maxk = alive ? sg.nchild : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) maxk = max(maxk, __shfl_xor_sync(0xffffffffu, maxk, o));
        for (uint32_t k = 0; k < maxk; ++k) {
            const bool mine = alive && k < sg.nchild;
            uint32_t b = 0, e = 0;
            const double *w = nullptr;
            const uint32_t *list = nullptr;
            if (mine) {
                const BoundChild ch = kids[sg.child_first + k];
                const uint32_t iu = ch.src ? ch.src[i] : i;
                b = ch.off[iu];
                e = ch.off[iu + 1];
                w = ch.w;
                list = ch.list;
            }
            double sum = (mine && !w) ? (double)(e - b) : 0.0;
            const bool coop = mine && w && (e - b) > 32;
            uint32_t todo = __ballot_sync(0xffffffffu, coop);
            while (todo) {
                const int src = __ffs(todo) - 1;
                todo &= todo - 1;
                const uint32_t bb = __shfl_sync(0xffffffffu, b, src), ee = __shfl_sync(0xffffffffu, e, src);
                const double *ww = (const double *)__shfl_sync(0xffffffffu, (unsigned long long)w, src);
                const uint32_t *ll = (const uint32_t *)__shfl_sync(0xffffffffu, (unsigned long long)list, src);
                const bool uu = __shfl_sync(0xffffffffu, (uint32_t)up, src) != 0;
                double part = 0.0;
                for (uint32_t x = bb + lane; x < ee; x += 32) part = dadd(part, ww[ll[x]], uu);
#pragma unroll
                for (int o = 16; o; o >>= 1) part = dadd(part, __shfl_xor_sync(0xffffffffu, part, o), uu);
                if ((int)lane == src) sum = part;
            }
            if (mine && w && !coop)
                for (uint32_t x = b; x < e; ++x) sum = dadd(sum, w[list[x]], up);
            if (mine) acc = dmul(acc, sum, up);
        }
        if (valid) sg.w[i] = acc;
    }
}

// A query's bound: for each component, the sum of its root's weights; the
// product over components; 0 when a fixed vertex has no candidate of its
// class or an edge between fixed vertices is missing.  The sums run in two
// steps: bound_parts sums kRootSlices slices of every root array (one block
// per slice), bound_queries adds a query's slices in order and multiplies.
constexpr uint32_t kRootSlices = 32;

struct BoundQuery {
    const double *const *roots;  // root weight arrays of the components
    const uint32_t *nroot;       // their lengths
    uint32_t ncomp, nhub, nedge, up;  // up = 1: sums and products rounded up (else toward zero)
    const uint32_t *hub;         // chosen hub indices of the fixed vertices
    const uint32_t *edge_ok;     // checks of the edges inside F
    double *part;                // ncomp * kRootSlices slice sums (set by attach_parts)
    double *out;
};

// Block (slice, query): the slice's share of every component's root sum.
__global__ void bound_parts(const BoundQuery *__restrict__ qs) {
    const BoundQuery bq = qs[blockIdx.y];
    const bool up = bq.up != 0;
    __shared__ double red[32];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) / 32;
    for (uint32_t c = 0; c < bq.ncomp; ++c) {
        const uint32_t n = bq.nroot[c];
        const uint32_t per = (n + kRootSlices - 1) / kRootSlices;
        const uint32_t lo = min(n, blockIdx.x * per), hi = min(n, lo + per);
        double part = 0.0;
        const double *w = bq.roots[c];
        for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) part = dadd(part, w[i], up);
#pragma unroll
        for (int o = 16; o; o >>= 1) part = dadd(part, __shfl_xor_sync(0xffffffffu, part, o), up);
        if (lane == 0) red[warp] = part;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (uint32_t k = 0; k < nw; ++k) tot = dadd(tot, red[k], up);
            bq.part[c * kRootSlices + blockIdx.x] = tot;
        }
        __syncthreads();
    }
}

// One thread per query.
__global__ void bound_queries(const BoundQuery *__restrict__ qs, uint32_t n) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const BoundQuery bq = qs[t];
    const bool up = bq.up != 0;
    double prod = 1.0;
    for (uint32_t k = 0; k < bq.nhub; ++k) prod = bq.hub[k] == kNone ? 0.0 : prod;
    for (uint32_t k = 0; k < bq.nedge; ++k) prod = bq.edge_ok[k] ? prod : 0.0;
    for (uint32_t c = 0; c < bq.ncomp; ++c) {
        double tot = 0.0;
        for (uint32_t k = 0; k < kRootSlices; ++k) tot = dadd(tot, bq.part[c * kRootSlices + k], up);
        prod = dmul(prod, tot, up);
    }
    *bq.out = prod;
}

// Slice-sum storage for the queries' components: one device buffer (*d_part,
// freed by the caller) that each BoundQuery's part points into.
int attach_parts(std::vector<BoundQuery> &bqs, double **d_part, cudaStream_t s) {
    uint64_t total = 0;
    for (const BoundQuery &bq : bqs) total += (uint64_t)bq.ncomp * kRootSlices;
    ASDM_TRY(dalloc(d_part, std::max<uint64_t>(total, 1), s));
    uint64_t at = 0;
    for (BoundQuery &bq : bqs) {
        bq.part = *d_part + at;
        at += (uint64_t)bq.ncomp * kRootSlices;
    }
    return ASDM_OK;
}

// The two launches of a set of queries' bounds (descriptors on the device).
void launch_bound_queries(const BoundQuery *d_bq, uint32_t n, cudaStream_t s) {
    if (!n) return;
    for (uint32_t at = 0; at < n; at += 65535u) {  // grid y is at most 65535
        bound_parts<<<dim3(kRootSlices, std::min(65535u, n - at)), 256, 0, s>>>(d_bq + at);
        ::asdm::count_launch();
    }
    bound_queries<<<(n + 127) / 128, 128, 0, s>>>(d_bq, n);
    ::asdm::count_launch();
}

// The inclusion-exclusion sum of a query's terms, rounded down: terms with a
// positive coefficient were computed rounding toward zero, the others
// rounding up, so the result is at most the exact sum.  One thread per query.
struct BoundSum {
    const double *terms;
    const double *coef;
    uint32_t nterm, pad;
    double *out;
};

__global__ void bound_sums(const BoundSum *__restrict__ sums, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const BoundSum b = sums[i];
    double acc = 0.0;
    for (uint32_t t = 0; t < b.nterm; ++t) {
        const double c = b.coef[t];
        acc = c > 0 ? __dadd_rd(acc, __dmul_rd(c, b.terms[t])) : __dadd_rd(acc, -__dmul_ru(-c, b.terms[t]));
    }
    *b.out = acc;
}

constexpr uint32_t kHubRounds = 8;  // candidates tried for the first fixed vertex

struct HubSeg {
    const uint32_t *cand;
    uint32_t ncand, cls_k, cls_c, nex;
    uint32_t *out;                 // index in C(f) of the chosen candidate, or kNone
    uint32_t ex[kHubRounds - 1];   // indices chosen in earlier rounds (skipped)
};

// The candidate of each segment's class with the largest data degree (ties:
// the smaller index), other than the excluded ones: block (slice, segment)
// takes the best key (set bit 63, degree, inverted index) of its slice of
// C(f) into keys[segment] (zeroed before), hub_decode turns it into an index.
constexpr uint32_t kHubSlices = 16;

__global__ void pick_hubs(const HubSeg *__restrict__ segs, const uint32_t *__restrict__ goff,
                          unsigned long long *__restrict__ keys) {
    const HubSeg sg = segs[blockIdx.y];
    const uint32_t per = (sg.ncand + kHubSlices - 1) / kHubSlices;
    const uint32_t lo = min(sg.ncand, blockIdx.x * per), hi = min(sg.ncand, lo + per);
    unsigned long long best = 0;
    for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        const uint32_t v = sg.cand[i];
        if (sg.cls_k > 1 && vertex_class(v, sg.cls_k) != sg.cls_c) continue;
        bool skip = false;
        for (uint32_t k = 0; k < sg.nex; ++k) skip |= sg.ex[k] == i;
        if (skip) continue;
        const unsigned long long key =
            (1ull << 63) | ((unsigned long long)(goff[v + 1] - goff[v]) << 32) | (0xFFFFFFFFu - i);
        best = max(best, key);
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
    __shared__ unsigned long long red[32];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = best;
    __syncthreads();
    if (warp == 0) {
        best = lane < (blockDim.x + 31) / 32 ? red[lane] : 0ull;
#pragma unroll
        for (int o = 16; o; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
        if (lane == 0 && best) atomicMax(keys + blockIdx.y, best);
    }
}

__global__ void hub_decode(const HubSeg *__restrict__ segs, const unsigned long long *__restrict__ keys, uint32_t n) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const unsigned long long k = keys[t];
    *segs[t].out = k ? 0xFFFFFFFFu - (uint32_t)(k & 0xFFFFFFFFull) : kNone;
}

// Both launches for n segments (descriptors on the device).
int launch_pick_hubs(asdm_graph *G, const HubSeg *d_segs, uint32_t n, cudaStream_t s) {
    if (!n) return ASDM_OK;
    unsigned long long *keys = nullptr;
    ASDM_TRY(dalloc(&keys, n, s));
    int rc = ASDM_OK;
    if (cudaMemsetAsync(keys, 0, n * sizeof(unsigned long long), s) != cudaSuccess) {
        rc = fail(ASDM_ERR_CUDA, "hub keys reset failed");
    } else {
        for (uint32_t at = 0; at < n; at += 65535u) {  // grid y is at most 65535
            pick_hubs<<<dim3(kHubSlices, std::min(65535u, n - at)), 256, 0, s>>>(d_segs + at, G->d.off, keys + at);
            ::asdm::count_launch();
        }
        hub_decode<<<(n + 127) / 128, 128, 0, s>>>(d_segs, keys, n);
        ::asdm::count_launch();
        if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "hub kernels failed");
    }
    dfree(keys, s);
    return rc;
}

// Indicator weights of the fixed vertices (w[hub] = 1; the arrays are zeroed
// before), and the checks of edges between fixed vertices: ok = 1 when fixed
// candidate b of the edge's head lies in the edge's list of fixed candidate a.
struct FixEdge {
    const uint32_t *off, *list;
    const uint32_t *ha, *hb;  // chosen indices of the two fixed vertices
    uint32_t *ok;
};

__global__ void fix_weights(double *const *__restrict__ w, const uint32_t *const *__restrict__ hub, uint32_t nw,
                            const FixEdge *__restrict__ edges, uint32_t ne) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < nw) {
        const uint32_t h = *hub[t];
        if (h != kNone) w[t][h] = 1.0;
    } else if (t < nw + ne) {
        const FixEdge e = edges[t - nw];
        const uint32_t a = *e.ha, b = *e.hb;
        uint32_t ok = 0;
        if (a != kNone && b != kNone) {
            const uint32_t lo = e.off[a], hi = e.off[a + 1];
            const uint32_t q = lo + lower_bound_u32(e.list + lo, hi - lo, b);
            ok = q < hi && e.list[q] == b;
        }
        *e.ok = ok;
    }
}

// Tighter bounds for tree queries: classes only where a same-label pair is
// three or more edges apart (a merge there would close a cycle), and the
// other same-label pairs, all two edges apart, handled exactly by the tree
// program's inclusion-exclusion over blocks (vertices of different classes
// never share a block).  That counts exactly the embeddings whose far-apart
// same-label vertices respect their classes, a subset of all embeddings.
// Terms with a positive coefficient are computed rounding toward zero, the
// others rounding up, and the signed sum rounding down (bound_sums), so the
// result is a lower bound.  lb[i] = the bound, formed[i] = 0 where the query
// is not a tree or has too many terms.
int tree_bounds(asdm_graph *G, const std::vector<asdm_cs *> &cs, std::vector<double> &lb, std::vector<char> &formed) {
    cudaStream_t s = G->stream;
    const size_t Q = cs.size();
    lb.assign(Q, 0.0);
    formed.assign(Q, 0);
    struct TPrep {
        std::vector<BlockTree> terms;
        std::vector<uint32_t> ck, cc;  // class count and class of each vertex (ck 1: unrestricted)
        uint64_t words = 0;
    };
    std::vector<TPrep> prep(Q);
    for (size_t i = 0; i < Q; ++i) {
        const asdm_cs &c = *cs[i];
        const QueryGraph &q = c.q;
        if (!c.nonempty || q.n < 2 || q.off[q.n] != 2 * (q.n - 1)) continue;
        const uint32_t n = q.n;
        // distances, then the classes of the far pairs' vertices
        std::vector<std::vector<uint32_t>> dist(n, std::vector<uint32_t>(n, kNone));
        for (uint32_t r = 0; r < n; ++r) {
            std::vector<uint32_t> fr{r};
            dist[r][r] = 0;
            for (size_t k = 0; k < fr.size(); ++k)
                for (uint32_t e = q.off[fr[k]]; e < q.off[fr[k] + 1]; ++e)
                    if (dist[r][q.nbr[e]] == kNone) {
                        dist[r][q.nbr[e]] = dist[r][fr[k]] + 1;
                        fr.push_back(q.nbr[e]);
                    }
        }
        auto far = [&](uint32_t u, uint32_t w) { return u != w && q.lab[u] == q.lab[w] && dist[u][w] >= 3; };
        TPrep &P = prep[i];
        std::vector<uint32_t> cls(n, kNone);
        for (uint32_t u = 0; u < n; ++u) {
            bool any = false;
            uint64_t used = 0;
            for (uint32_t w = 0; w < n; ++w)
                if (far(u, w)) {
                    any = true;
                    if (w < u) used |= 1ull << cls[w];
                }
            if (!any) continue;
            uint32_t c0 = 0;
            while (used >> c0 & 1ull) ++c0;
            cls[u] = c0;
        }
        P.ck.assign(n, 1);
        P.cc.assign(n, 0);
        for (uint32_t u = 0; u < n; ++u) {
            if (cls[u] == kNone) continue;
            uint32_t k = 0;
            for (uint32_t w = 0; w < n; ++w)
                if (q.lab[w] == q.lab[u] && cls[w] != kNone) k = std::max(k, cls[w] + 1);
            P.ck[u] = k;
            P.cc[u] = cls[u];
        }
        if (!block_trees(q, P.terms, &c, &cls)) continue;
        for (const BlockTree &t : P.terms)
            for (uint32_t b = 0; b < t.nb; ++b) P.words += c.ncand[t.rep[b]] * (1 + t.members[b].size());
        formed[i] = 1;
    }
    size_t at = 0;
    int rc = ASDM_OK;
    while (at < Q && rc == ASDM_OK) {
        std::vector<size_t> ids;
        uint64_t words = 0;
        for (; at < Q; ++at) {
            if (!formed[at]) continue;
            if (!ids.empty() && words + prep[at].words > kTreeChunkWords) break;
            words += prep[at].words;
            ids.push_back(at);
        }
        if (ids.empty()) break;
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "tree-bound sync failed");
            break;
        }
        G->stage.reset();
        double *wbuf = nullptr, *d_terms = nullptr, *d_coef = nullptr, *d_out = nullptr, *d_part = nullptr;
        uint32_t *d_mapbuf = nullptr, *d_nroot = nullptr;
        MapSeg *d_mseg = nullptr;
        BoundSeg *d_segs = nullptr;
        BoundChild *d_kids = nullptr;
        BoundQuery *d_bq = nullptr;
        BoundSum *d_sums = nullptr;
        const uint32_t **d_maps = nullptr;
        const double **d_roots = nullptr;
        do {
            // member maps C(rep) -> C(member) of merged blocks, one per (query, rep, member)
            std::vector<MapSeg> msegs;
            std::vector<std::vector<std::pair<uint64_t, uint32_t>>> mkey(ids.size());
            uint64_t mtotal = 0, wtotal = 0;
            std::vector<std::vector<std::vector<uint64_t>>> woff(ids.size());
            uint32_t nterms = 0;
            for (size_t k = 0; k < ids.size(); ++k) {
                const asdm_cs &c = *cs[ids[k]];
                const TPrep &P = prep[ids[k]];
                woff[k].resize(P.terms.size());
                nterms += (uint32_t)P.terms.size();
                for (size_t ti = 0; ti < P.terms.size(); ++ti) {
                    const BlockTree &t = P.terms[ti];
                    woff[k][ti].resize(t.nb);
                    for (uint32_t b = 0; b < t.nb; ++b) {
                        woff[k][ti][b] = wtotal;
                        wtotal += c.ncand[t.rep[b]];
                        for (uint32_t u : t.members[b]) {
                            if (u == t.rep[b]) continue;
                            const uint64_t key = ((uint64_t)t.rep[b] << 32) | u;
                            bool have = false;
                            for (auto &kv : mkey[k]) have = have || kv.first == key;
                            if (have) continue;
                            mkey[k].emplace_back(key, (uint32_t)msegs.size());
                            msegs.push_back(MapSeg{c.d_cand + c.cand_base[t.rep[b]], c.d_cand + c.cand_base[u],
                                                   nullptr, c.ncand[u], 0, mtotal});
                            mtotal += c.ncand[t.rep[b]];
                        }
                    }
                }
            }
            if ((rc = dalloc(&wbuf, std::max<uint64_t>(wtotal, 1), s)) || (rc = dalloc(&d_terms, nterms, s)) ||
                (rc = dalloc(&d_coef, nterms, s)) || (rc = dalloc(&d_out, ids.size(), s)))
                break;
            std::vector<const uint32_t *> maps;
            if (mtotal) {
                if ((rc = dalloc(&d_mapbuf, mtotal, s)) || (rc = dalloc(&d_mseg, msegs.size(), s))) break;
                for (auto &m : msegs) m.out = d_mapbuf + m.start;
                if (upload_async(G, d_mseg, msegs.data(), msegs.size() * sizeof(MapSeg)) != cudaSuccess) {
                    rc = fail(ASDM_ERR_CUDA, "tree-bound map upload failed");
                    break;
                }
                const unsigned grid =
                    (unsigned)std::min<unsigned long long>((mtotal + 255) / 256, (unsigned long long)G->num_sms * 32);
                tree_maps<<<grid, 256, 0, s>>>(d_mseg, (uint32_t)msegs.size(), mtotal);
                ::asdm::count_launch();
            }
            auto map_of = [&](size_t k, uint32_t r, uint32_t u) -> const uint32_t * {
                const uint64_t key = ((uint64_t)r << 32) | u;
                for (auto &kv : mkey[k])
                    if (kv.first == key) return msegs[kv.second].out;
                return nullptr;
            };
            // segments by height, children, the terms' root sums and the signed sums
            std::vector<std::vector<BoundSeg>> lv;
            std::vector<BoundChild> kids;
            std::vector<BoundQuery> bqs;
            std::vector<const double *> roots;
            std::vector<uint32_t> nroot;
            std::vector<double> coef;
            std::vector<BoundSum> sums;
            for (size_t k = 0; k < ids.size(); ++k) {
                const asdm_cs &c = *cs[ids[k]];
                const TPrep &P = prep[ids[k]];
                sums.push_back(BoundSum{d_terms + coef.size(), d_coef + coef.size(), (uint32_t)P.terms.size(), 0,
                                        d_out + k});
                for (size_t ti = 0; ti < P.terms.size(); ++ti) {
                    const BlockTree &t = P.terms[ti];
                    const uint32_t up = t.coef < 0 ? 1u : 0u;
                    auto restricted = [&](uint32_t b) {
                        for (uint32_t u : t.members[b])
                            if (P.ck[u] > 1) return u;
                        return kNone;
                    };
                    auto leaf1 = [&](uint32_t b) {
                        return t.height[b] == 0 && t.members[b].size() == 1 && restricted(b) == kNone;
                    };
                    uint32_t root = kNone;
                    for (uint32_t b = 0; b < t.nb; ++b) {
                        if (t.parent[b] == kNone) root = b;
                        if (leaf1(b) && t.parent[b] != kNone) continue;
                        const uint32_t r = t.rep[b], cu = restricted(b);
                        BoundSeg sg{};
                        sg.w = wbuf + woff[k][ti][b];
                        sg.cand = c.d_cand + c.cand_base[r];
                        sg.ncand = c.ncand[r];
                        sg.cls_k = cu == kNone ? 1u : P.ck[cu];
                        sg.cls_c = cu == kNone ? 0u : P.cc[cu];
                        sg.up = up;
                        sg.val_first = (uint32_t)maps.size();
                        for (uint32_t u : t.members[b])
                            if (u != r) maps.push_back(map_of(k, r, u));
                        sg.nval = (uint32_t)maps.size() - sg.val_first;
                        sg.child_first = (uint32_t)kids.size();
                        for (uint32_t C = 0; C < t.nb; ++C) {
                            if (t.parent[C] != b) continue;
                            const uint32_t e = t.pedge[C], u = t.pfrom[C];
                            kids.push_back(BoundChild{c.d_eoff + c.eoff_base[e], c.d_elist + c.elist_base[e],
                                                      leaf1(C) ? nullptr : wbuf + woff[k][ti][C],
                                                      u == r ? nullptr : map_of(k, r, u)});
                        }
                        sg.nchild = (uint32_t)kids.size() - sg.child_first;
                        if (lv.size() <= t.height[b]) lv.resize(t.height[b] + 1);
                        lv[t.height[b]].push_back(sg);
                    }
                    BoundQuery bq{};
                    bq.ncomp = 1;
                    bq.up = up;
                    bq.out = d_terms + coef.size();
                    roots.push_back(wbuf + woff[k][ti][root]);
                    nroot.push_back(c.ncand[t.rep[root]]);
                    bqs.push_back(bq);
                    coef.push_back((double)t.coef);
                }
            }
            std::vector<BoundSeg> segs;
            std::vector<size_t> first{0};
            std::vector<unsigned long long> totals;
            for (auto &l : lv) {
                unsigned long long tt = 0;
                for (BoundSeg &sg : l) {
                    sg.start = tt;
                    tt += sg.ncand;
                    segs.push_back(sg);
                }
                first.push_back(segs.size());
                totals.push_back(tt);
            }
            if (kids.empty()) kids.push_back(BoundChild{});
            if (segs.empty()) segs.push_back(BoundSeg{});
            if (maps.empty()) maps.push_back(nullptr);
            if ((rc = dalloc(&d_segs, segs.size(), s)) || (rc = dalloc(&d_kids, kids.size(), s)) ||
                (rc = dalloc(&d_maps, maps.size(), s)) || (rc = dalloc(&d_roots, roots.size(), s)) ||
                (rc = dalloc(&d_nroot, nroot.size(), s)) || (rc = dalloc(&d_bq, bqs.size(), s)) ||
                (rc = dalloc(&d_sums, sums.size(), s)))
                break;
            for (size_t j = 0; j < bqs.size(); ++j) {
                bqs[j].roots = d_roots + j;
                bqs[j].nroot = d_nroot + j;
            }
            if ((rc = attach_parts(bqs, &d_part, s))) break;
            if (upload_async(G, d_segs, segs.data(), segs.size() * sizeof(BoundSeg)) != cudaSuccess ||
                upload_async(G, d_kids, kids.data(), kids.size() * sizeof(BoundChild)) != cudaSuccess ||
                upload_async(G, d_maps, maps.data(), maps.size() * sizeof(void *)) != cudaSuccess ||
                upload_async(G, d_roots, roots.data(), roots.size() * sizeof(void *)) != cudaSuccess ||
                upload_async(G, d_nroot, nroot.data(), nroot.size() * sizeof(uint32_t)) != cudaSuccess ||
                upload_async(G, d_coef, coef.data(), coef.size() * sizeof(double)) != cudaSuccess ||
                upload_async(G, d_bq, bqs.data(), bqs.size() * sizeof(BoundQuery)) != cudaSuccess ||
                upload_async(G, d_sums, sums.data(), sums.size() * sizeof(BoundSum)) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "tree-bound upload failed");
                break;
            }
            for (size_t h = 0; h < totals.size() && rc == ASDM_OK; ++h) {
                if (!totals[h]) continue;
                const unsigned grid =
                    (unsigned)std::min<unsigned long long>((totals[h] + 255) / 256, (unsigned long long)G->num_sms * 32);
                bound_level<<<grid, 256, 0, s>>>(d_segs + first[h], (uint32_t)(first[h + 1] - first[h]), totals[h],
                                                 d_kids, d_maps);
                ::asdm::count_launch();
                if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "tree-bound kernel failed");
            }
            if (rc != ASDM_OK) break;
            launch_bound_queries(d_bq, (uint32_t)bqs.size(), s);
            bound_sums<<<(unsigned)((sums.size() + 127) / 128), 128, 0, s>>>(d_sums, (uint32_t)sums.size());
            ::asdm::count_launch();
            std::vector<double> out(ids.size());
            if (cudaGetLastError() != cudaSuccess ||
                cudaMemcpyAsync(out.data(), d_out, out.size() * sizeof(double), cudaMemcpyDeviceToHost, s) !=
                    cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "tree-bound readback failed");
                break;
            }
            for (size_t k = 0; k < ids.size(); ++k) lb[ids[k]] = std::max(0.0, out[k]);
        } while (false);
        dfree(wbuf, s);
        dfree(d_terms, s);
        dfree(d_coef, s);
        dfree(d_out, s);
        dfree(d_mapbuf, s);
        dfree(d_mseg, s);
        dfree(d_nroot, s);
        dfree(d_segs, s);
        dfree(d_kids, s);
        dfree(d_bq, s);
        dfree(d_sums, s);
        dfree(d_maps, s);
        dfree(d_roots, s);
        dfree(d_part, s);
        cudaStreamSynchronize(s);
    }
    if (rc != ASDM_OK) {
        lb.assign(Q, 0.0);
        formed.assign(Q, 0);
    }
    return rc;
}

// First-order (Bonferroni) bounds, without classes.  With F (greedy_fvs)
// fixed to hubs, H is the number of homomorphisms of Q into the candidate
// space: every vertex outside F on its candidates, F on its hubs, every edge
// kept (the forest program with indicator copies, without classes).  A
// homomorphism that is not an embedding maps two query vertices to one data
// vertex; the two have one label (a candidate carries its query vertex's
// label) and are not adjacent (data graphs have no self loops).  Those that
// map the pair {a, b} together number at most T_ab:
//   * a in F, b not: the program with b pinned to a's hub (exact);
//   * neither in F: the program with b merged into a (one block on the
//     candidates of both); where the merge closes a cycle, the edge that
//     would close it is left out of the forest (fewer constraints, so more
//     homomorphisms: an upper bound);
//   * both in F: none (same-label vertices of F take hubs of different
//     classes, never one vertex).
// So count >= H - sum of T_ab.  H is rounded toward zero, every T_ab up, and
// the difference down (on the host: sums stepped one ulp up, the difference
// one ulp down).  As with the class bounds, later rounds move F's first
// vertex to its next hubs and the rounds' positive bounds add up.  Where only
// the proof matters (no bound value asked for), a round counts its T terms
// only for queries whose H could still carry the sum to 2^64.

// Weight words of one launch group of pair programs (8 GiB): many small
// programs per launch keep the level launches full.
constexpr uint64_t kPairChunkWords = 1ull << 30;

// One program of a pair bound: the forest over the vertices outside F, with
// b in a's block when merged, or vertex `pin` pinned to the hub of F's
// vertex fvs[pin_f].
struct PairTerm {
    uint32_t ma = kNone, mb = kNone;
    uint32_t pin = kNone, pin_f = kNone;
    uint32_t nb = 0;
    std::vector<uint32_t> block;                  // by vertex (kNone in F)
    std::vector<std::vector<uint32_t>> members;   // by block, ascending
    std::vector<uint32_t> rep, parent, pedge, pfrom, height;
    std::vector<char> fnbr;                       // a member has an edge into F
    uint64_t words = 0;                           // weight words of the blocks that need them
};

// Whether block b of term t needs a weight array: all but one-vertex leaves
// with a parent, no edge into F and no pin (the parent takes their list length).
bool pair_needs_weights(const PairTerm &t, uint32_t b) {
    return !(t.height[b] == 0 && t.members[b].size() == 1 && !t.fnbr[b] && t.parent[b] != kNone &&
             t.members[b][0] != t.pin);
}

// The forest of a term: blocks in order of their lowest member; breadth-first
// from the lowest unvisited block, each block's members in id order and
// their neighbours in adjacency order; an edge into a visited block is left
// out.
void pair_forest(const QueryGraph &q, const std::vector<char> &fixed, const asdm_cs &c, PairTerm &t) {
    const uint32_t n = q.n;
    t.block.assign(n, kNone);
    t.members.clear();
    for (uint32_t u = 0; u < n; ++u) {
        if (fixed[u] || u == t.mb) continue;
        t.block[u] = (uint32_t)t.members.size();
        t.members.push_back({u});
    }
    if (t.mb != kNone) {
        auto &m = t.members[t.block[t.ma]];
        t.block[t.mb] = t.block[t.ma];
        m.push_back(t.mb);
        std::sort(m.begin(), m.end());
    }
    t.nb = (uint32_t)t.members.size();
    t.rep.assign(t.nb, kNone);
    t.parent.assign(t.nb, kNone);
    t.pedge.assign(t.nb, kNone);
    t.pfrom.assign(t.nb, kNone);
    t.height.assign(t.nb, 0);
    t.fnbr.assign(t.nb, 0);
    std::vector<uint32_t> order;
    for (uint32_t r = 0; r < t.nb; ++r) {
        if (t.rep[r] != kNone) continue;
        t.rep[r] = t.members[r][0];
        const size_t first = order.size();
        order.push_back(r);
        for (size_t k = first; k < order.size(); ++k) {
            const uint32_t B = order[k];
            for (uint32_t u : t.members[B])
                for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                    const uint32_t w = q.nbr[e];
                    if (fixed[w]) {
                        t.fnbr[B] = 1;
                        continue;
                    }
                    const uint32_t C = t.block[w];
                    if (C == B || t.rep[C] != kNone) continue;
                    t.rep[C] = w;
                    t.parent[C] = B;
                    t.pedge[C] = e;
                    t.pfrom[C] = u;
                    order.push_back(C);
                }
        }
    }
    for (size_t k = order.size(); k-- > 0;) {
        const uint32_t C = order[k];
        if (t.parent[C] != kNone) t.height[t.parent[C]] = std::max(t.height[t.parent[C]], t.height[C] + 1);
    }
    t.words = 0;
    for (uint32_t b = 0; b < t.nb; ++b)
        if (pair_needs_weights(t, b)) t.words += c.ncand[t.rep[b]];
}

struct PairPrep {
    std::vector<char> fixed;
    std::vector<uint32_t> fvs, fk, fc;  // F; class counts and classes among F's same-label vertices
    std::vector<PairTerm> terms;        // terms[0]: H; then one per pair
    uint64_t fwords = 0;                // indicator words of F
};

// Values of the programs `jobs` (query, term) of one round, one double each:
// rounded toward zero for terms[0], up for the others.  d_hub holds the
// round's hub indices (query i's F from hub0[i]), d_eok the checks of the
// edges inside F (query i's from fe0[i], nfe[i] of them).  A query's jobs
// are consecutive.
int pair_values(asdm_graph *G, const std::vector<asdm_cs *> &cs, const std::vector<PairPrep> &prep,
                const std::vector<std::pair<size_t, uint32_t>> &jobs, const uint32_t *d_hub,
                const std::vector<uint32_t> &hub0, const uint32_t *d_eok, const std::vector<uint32_t> &fe0,
                const std::vector<uint32_t> &nfe, std::vector<double> &vals) {
    cudaStream_t s = G->stream;
    vals.assign(jobs.size(), 0.0);
    size_t at = 0;
    int rc = ASDM_OK;
    while (at < jobs.size() && rc == ASDM_OK) {
        // a chunk: consecutive jobs whose weights and indicators fit kPairChunkWords (one job at least)
        const size_t j0 = at;
        uint64_t words = 0;
        std::vector<size_t> qs;
        for (; at < jobs.size(); ++at) {
            const size_t i = jobs[at].first;
            uint64_t add = prep[i].terms[jobs[at].second].words;
            const bool new_q = qs.empty() || qs.back() != i;
            if (new_q) add += prep[i].fwords;
            if (at > j0 && words + add > kPairChunkWords) break;
            words += add;
            if (new_q) qs.push_back(i);
        }
        const size_t j1 = at;
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "pair-bound sync failed");
            break;
        }
        G->stage.reset();
        double *wbuf = nullptr, *d_out = nullptr, *d_part = nullptr;
        uint32_t *d_mapbuf = nullptr, *d_nroot = nullptr;
        MapSeg *d_mseg = nullptr;
        BoundSeg *d_segs = nullptr;
        BoundChild *d_kids = nullptr;
        BoundQuery *d_bq = nullptr;
        double **d_fw = nullptr;
        const uint32_t **d_fh = nullptr, **d_maps = nullptr;
        const double **d_roots = nullptr;
        do {
            if ((rc = dalloc(&wbuf, std::max<uint64_t>(words, 1), s)) || (rc = dalloc(&d_out, j1 - j0, s))) break;
            if (cudaMemsetAsync(wbuf, 0, std::max<uint64_t>(words, 1) * sizeof(double), s) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "pair-bound reset failed");
                break;
            }
            // indicators of F, one set per query of the chunk
            uint64_t wo = 0;
            std::vector<std::vector<double *>> find(cs.size());
            std::vector<double *> fw;
            std::vector<const uint32_t *> fh;
            for (size_t i : qs) {
                const asdm_cs &c = *cs[i];
                const PairPrep &P = prep[i];
                find[i].assign(c.q.n, nullptr);
                for (size_t j = 0; j < P.fvs.size(); ++j) {
                    const uint32_t f = P.fvs[j];
                    find[i][f] = wbuf + wo;
                    wo += c.ncand[f];
                    fw.push_back(find[i][f]);
                    fh.push_back(d_hub + hub0[i] + j);
                }
            }
            // maps C(rep) -> C(other member) of merged blocks
            std::vector<MapSeg> msegs;
            std::vector<std::pair<std::pair<size_t, uint64_t>, uint32_t>> mkey;
            uint64_t mtotal = 0;
            auto map_slot = [&](size_t i, uint32_t r, uint32_t u) -> uint32_t {
                const auto key = std::make_pair(i, ((uint64_t)r << 32) | u);
                for (auto &kv : mkey)
                    if (kv.first == key) return kv.second;
                const asdm_cs &c = *cs[i];
                mkey.emplace_back(key, (uint32_t)msegs.size());
                msegs.push_back(MapSeg{c.d_cand + c.cand_base[r], c.d_cand + c.cand_base[u], nullptr, c.ncand[u], 0,
                                       mtotal});
                mtotal += c.ncand[r];
                return (uint32_t)msegs.size() - 1;
            };
            for (size_t j = j0; j < j1; ++j) {
                const PairTerm &t = prep[jobs[j].first].terms[jobs[j].second];
                if (t.mb == kNone) continue;
                const uint32_t b = t.block[t.ma];
                for (uint32_t u : t.members[b])
                    if (u != t.rep[b]) map_slot(jobs[j].first, t.rep[b], u);
            }
            if (mtotal) {
                if ((rc = dalloc(&d_mapbuf, mtotal, s)) || (rc = dalloc(&d_mseg, msegs.size(), s))) break;
                for (auto &m : msegs) m.out = d_mapbuf + m.start;
                if (upload_async(G, d_mseg, msegs.data(), msegs.size() * sizeof(MapSeg)) != cudaSuccess) {
                    rc = fail(ASDM_ERR_CUDA, "pair-bound map upload failed");
                    break;
                }
                const unsigned grid =
                    (unsigned)std::min<unsigned long long>((mtotal + 255) / 256, (unsigned long long)G->num_sms * 32);
                tree_maps<<<grid, 256, 0, s>>>(d_mseg, (uint32_t)msegs.size(), mtotal);
                ::asdm::count_launch();
            }
            if (!fw.empty()) {
                if ((rc = dalloc(&d_fw, fw.size(), s)) || (rc = dalloc(&d_fh, fh.size(), s))) break;
                if (upload_async(G, d_fw, fw.data(), fw.size() * sizeof(void *)) != cudaSuccess ||
                    upload_async(G, d_fh, fh.data(), fh.size() * sizeof(void *)) != cudaSuccess) {
                    rc = fail(ASDM_ERR_CUDA, "pair-bound indicator upload failed");
                    break;
                }
                fix_weights<<<(unsigned)((fw.size() + 255) / 256), 256, 0, s>>>(d_fw, d_fh, (uint32_t)fw.size(),
                                                                                  nullptr, 0);
                ::asdm::count_launch();
            }
            // segments by height, children (forest children, then edges into F), roots, one query per term
            std::vector<std::vector<BoundSeg>> lv;
            std::vector<BoundChild> kids;
            std::vector<const uint32_t *> maps;
            std::vector<const double *> roots;
            std::vector<uint32_t> nroot;
            std::vector<BoundQuery> bqs;
            std::vector<size_t> root0;
            for (size_t j = j0; j < j1; ++j) {
                const size_t i = jobs[j].first;
                const asdm_cs &c = *cs[i];
                const QueryGraph &q = c.q;
                const PairPrep &P = prep[i];
                const PairTerm &t = P.terms[jobs[j].second];
                const uint32_t up = jobs[j].second > 0 ? 1u : 0u;
                std::vector<double *> wb(t.nb, nullptr);
                for (uint32_t b = 0; b < t.nb; ++b)
                    if (pair_needs_weights(t, b)) {
                        wb[b] = wbuf + wo;
                        wo += c.ncand[t.rep[b]];
                    }
                auto src_map = [&](uint32_t b, uint32_t u) -> const uint32_t * {
                    return u == t.rep[b] ? nullptr : d_mapbuf + msegs[map_slot(i, t.rep[b], u)].start;
                };
                root0.push_back(roots.size());
                for (uint32_t b = 0; b < t.nb; ++b) {
                    if (t.parent[b] == kNone) {
                        roots.push_back(wb[b]);
                        nroot.push_back(c.ncand[t.rep[b]]);
                    }
                    if (!wb[b]) continue;
                    const uint32_t r = t.rep[b];
                    BoundSeg sg{};
                    sg.w = wb[b];
                    sg.cand = c.d_cand + c.cand_base[r];
                    sg.ncand = c.ncand[r];
                    sg.cls_k = 1;
                    sg.up = up;
                    if (t.pin != kNone && t.block[t.pin] == b) {
                        sg.pin = d_hub + hub0[i] + t.pin_f;
                        sg.pin_cand = c.d_cand + c.cand_base[P.fvs[t.pin_f]];
                    }
                    sg.val_first = (uint32_t)maps.size();
                    for (uint32_t u : t.members[b])
                        if (u != r) maps.push_back(src_map(b, u));
                    sg.nval = (uint32_t)maps.size() - sg.val_first;
                    sg.child_first = (uint32_t)kids.size();
                    for (uint32_t C = 0; C < t.nb; ++C) {
                        if (t.parent[C] != b) continue;
                        const uint32_t e = t.pedge[C];
                        kids.push_back(BoundChild{c.d_eoff + c.eoff_base[e], c.d_elist + c.elist_base[e], wb[C],
                                                  src_map(b, t.pfrom[C])});
                    }
                    for (uint32_t u : t.members[b])
                        for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                            const uint32_t f = q.nbr[e];
                            if (!P.fixed[f]) continue;
                            kids.push_back(BoundChild{c.d_eoff + c.eoff_base[e], c.d_elist + c.elist_base[e],
                                                      find[i][f], src_map(b, u)});
                        }
                    sg.nchild = (uint32_t)kids.size() - sg.child_first;
                    if (lv.size() <= t.height[b]) lv.resize(t.height[b] + 1);
                    lv[t.height[b]].push_back(sg);
                }
                BoundQuery bq{};
                bq.ncomp = (uint32_t)(roots.size() - root0.back());
                bq.nhub = (uint32_t)P.fvs.size();
                bq.nedge = nfe[i];
                bq.up = up;
                bq.out = d_out + (j - j0);
                bqs.push_back(bq);
            }
            std::vector<BoundSeg> segs;
            std::vector<size_t> first{0};
            std::vector<unsigned long long> totals;
            for (auto &l : lv) {
                unsigned long long tt = 0;
                for (BoundSeg &sg : l) {
                    sg.start = tt;
                    tt += sg.ncand;
                    segs.push_back(sg);
                }
                first.push_back(segs.size());
                totals.push_back(tt);
            }
            if (kids.empty()) kids.push_back(BoundChild{});
            if (segs.empty()) segs.push_back(BoundSeg{});
            if (maps.empty()) maps.push_back(nullptr);
            if ((rc = dalloc(&d_segs, segs.size(), s)) || (rc = dalloc(&d_kids, kids.size(), s)) ||
                (rc = dalloc(&d_maps, maps.size(), s)) || (rc = dalloc(&d_roots, roots.size(), s)) ||
                (rc = dalloc(&d_nroot, nroot.size(), s)) || (rc = dalloc(&d_bq, bqs.size(), s)))
                break;
            for (size_t k = 0; k < bqs.size(); ++k) {
                const size_t i = jobs[j0 + k].first;
                bqs[k].roots = d_roots + root0[k];
                bqs[k].nroot = d_nroot + root0[k];
                bqs[k].hub = d_hub + hub0[i];
                bqs[k].edge_ok = d_eok + fe0[i];
            }
            if ((rc = attach_parts(bqs, &d_part, s))) break;
            if (upload_async(G, d_segs, segs.data(), segs.size() * sizeof(BoundSeg)) != cudaSuccess ||
                upload_async(G, d_kids, kids.data(), kids.size() * sizeof(BoundChild)) != cudaSuccess ||
                upload_async(G, d_maps, maps.data(), maps.size() * sizeof(void *)) != cudaSuccess ||
                upload_async(G, d_roots, roots.data(), roots.size() * sizeof(void *)) != cudaSuccess ||
                upload_async(G, d_nroot, nroot.data(), nroot.size() * sizeof(uint32_t)) != cudaSuccess ||
                upload_async(G, d_bq, bqs.data(), bqs.size() * sizeof(BoundQuery)) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "pair-bound upload failed");
                break;
            }
            for (size_t h = 0; h < totals.size() && rc == ASDM_OK; ++h) {
                if (!totals[h]) continue;
                const unsigned grid =
                    (unsigned)std::min<unsigned long long>((totals[h] + 255) / 256, (unsigned long long)G->num_sms * 32);
                bound_level<<<grid, 256, 0, s>>>(d_segs + first[h], (uint32_t)(first[h + 1] - first[h]), totals[h],
                                                 d_kids, d_maps);
                ::asdm::count_launch();
                if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "pair-bound kernel failed");
            }
            if (rc != ASDM_OK) break;
            launch_bound_queries(d_bq, (uint32_t)bqs.size(), s);
            if (cudaGetLastError() != cudaSuccess ||
                cudaMemcpyAsync(vals.data() + j0, d_out, (j1 - j0) * sizeof(double), cudaMemcpyDeviceToHost, s) !=
                    cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "pair-bound readback failed");
                break;
            }
        } while (false);
        dfree(wbuf, s);
        dfree(d_out, s);
        dfree(d_mapbuf, s);
        dfree(d_mseg, s);
        dfree(d_segs, s);
        dfree(d_kids, s);
        dfree(d_maps, s);
        dfree(d_roots, s);
        dfree(d_nroot, s);
        dfree(d_bq, s);
        dfree(d_fw, s);
        dfree(d_fh, s);
        dfree(d_part, s);
        cudaStreamSynchronize(s);
    }
    return rc;
}

// lb[i] = the pair bound of each query with want[i] (0 where none is formed;
// without all_terms, also where H alone shows that it stays below 2^64).
int pair_bounds(asdm_graph *G, const std::vector<asdm_cs *> &cs, const std::vector<char> &want,
                std::vector<double> &lb, bool all_terms) {
    cudaStream_t s = G->stream;
    const size_t Q = cs.size();
    const double two64 = 18446744073709551616.0;
    lb.assign(Q, 0.0);
    std::vector<PairPrep> prep(Q);
    std::vector<char> ok(Q, 0);
    for (size_t i = 0; i < Q; ++i) {
        const asdm_cs &c = *cs[i];
        const QueryGraph &q = c.q;
        if (!want[i] || !c.nonempty || q.n < 2) continue;
        PairPrep &P = prep[i];
        const uint32_t n = q.n;
        greedy_fvs(q, P.fixed, P.fvs);
        if (P.fvs.size() > kMaxFixed || P.fvs.size() == n) continue;
        // classes among F: the r-th of F's k vertices with one label (in F's order) takes class r
        P.fk.assign(P.fvs.size(), 0);
        P.fc.assign(P.fvs.size(), 0);
        for (size_t j = 0; j < P.fvs.size(); ++j)
            for (size_t j2 = 0; j2 < P.fvs.size(); ++j2)
                if (q.lab[P.fvs[j2]] == q.lab[P.fvs[j]]) {
                    P.fc[j] += j2 < j;
                    ++P.fk[j];
                }
        for (uint32_t f : P.fvs) P.fwords += c.ncand[f];
        std::vector<uint32_t> fpos(n, kNone);
        for (size_t j = 0; j < P.fvs.size(); ++j) fpos[P.fvs[j]] = (uint32_t)j;
        P.terms.emplace_back();
        for (uint32_t a = 0; a < n; ++a)
            for (uint32_t b = a + 1; b < n; ++b) {
                if (q.lab[a] != q.lab[b] || q.slot(a, b) >= 0 || (P.fixed[a] && P.fixed[b])) continue;
                PairTerm t;
                if (P.fixed[a]) {
                    t.pin = b;
                    t.pin_f = fpos[a];
                } else if (P.fixed[b]) {
                    t.pin = a;
                    t.pin_f = fpos[b];
                } else {
                    t.ma = a;
                    t.mb = b;
                }
                P.terms.push_back(std::move(t));
            }
        if (P.terms.size() == 1) continue;  // no pairs: the plain forest program counts embeddings
        for (PairTerm &t : P.terms) pair_forest(q, P.fixed, c, t);
        ok[i] = 1;
    }
    std::vector<std::vector<uint32_t>> excl(Q);
    int rc = ASDM_OK;
    for (uint32_t round = 0; round < kHubRounds && rc == ASDM_OK; ++round) {
        std::vector<size_t> ids;
        for (size_t i = 0; i < Q; ++i)
            if (ok[i] && lb[i] < two64 && (round == 0 || (!prep[i].fvs.empty() && excl[i].size() == round)))
                ids.push_back(i);
        if (ids.empty()) break;
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "pair-bound sync failed");
            break;
        }
        G->stage.reset();
        // the round's hubs and the checks of the edges inside F
        std::vector<uint32_t> hub0(Q, 0), fe0(Q, 0), nfe(Q, 0);
        std::vector<HubSeg> hsegs;
        std::vector<FixEdge> fedges;
        uint32_t nhub = 0;
        for (size_t i : ids) {
            hub0[i] = nhub;
            nhub += (uint32_t)prep[i].fvs.size();
        }
        uint32_t *d_hub = nullptr, *d_eok = nullptr;
        HubSeg *d_hsegs = nullptr;
        FixEdge *d_fe = nullptr;
        do {
            if ((rc = dalloc(&d_hub, std::max<uint32_t>(nhub, 1), s))) break;
            for (size_t i : ids) {
                const asdm_cs &c = *cs[i];
                const PairPrep &P = prep[i];
                for (size_t j = 0; j < P.fvs.size(); ++j) {
                    const uint32_t f = P.fvs[j];
                    HubSeg hs{c.d_cand + c.cand_base[f], c.ncand[f], P.fk[j], P.fc[j], 0, d_hub + hub0[i] + j, {}};
                    if (j == 0)
                        for (uint32_t x : excl[i]) hs.ex[hs.nex++] = x;
                    hsegs.push_back(hs);
                }
                fe0[i] = (uint32_t)fedges.size();
                for (size_t j = 0; j < P.fvs.size(); ++j)
                    for (size_t j2 = j + 1; j2 < P.fvs.size(); ++j2) {
                        const int sl = c.q.slot(P.fvs[j], P.fvs[j2]);
                        if (sl < 0) continue;
                        const uint32_t e = c.q.off[P.fvs[j]] + (uint32_t)sl;
                        fedges.push_back(FixEdge{c.d_eoff + c.eoff_base[e], c.d_elist + c.elist_base[e],
                                                 d_hub + hub0[i] + j, d_hub + hub0[i] + j2, nullptr});
                    }
                nfe[i] = (uint32_t)fedges.size() - fe0[i];
            }
            const uint32_t ne = (uint32_t)fedges.size();
            if ((rc = dalloc(&d_eok, std::max<uint32_t>(ne, 1), s))) break;
            for (uint32_t e = 0; e < ne; ++e) fedges[e].ok = d_eok + e;
            if (!hsegs.empty()) {
                if ((rc = dalloc(&d_hsegs, hsegs.size(), s))) break;
                if (upload_async(G, d_hsegs, hsegs.data(), hsegs.size() * sizeof(HubSeg)) != cudaSuccess) {
                    rc = fail(ASDM_ERR_CUDA, "pair-bound hub upload failed");
                    break;
                }
                if ((rc = launch_pick_hubs(G, d_hsegs, (uint32_t)hsegs.size(), s))) break;
            }
            if (ne) {
                if ((rc = dalloc(&d_fe, ne, s))) break;
                if (upload_async(G, d_fe, fedges.data(), ne * sizeof(FixEdge)) != cudaSuccess) {
                    rc = fail(ASDM_ERR_CUDA, "pair-bound edge upload failed");
                    break;
                }
                fix_weights<<<(ne + 255) / 256, 256, 0, s>>>(nullptr, nullptr, 0, d_fe, ne);
                ::asdm::count_launch();
            }
            std::vector<uint32_t> hubs(std::max<uint32_t>(nhub, 1));
            if (cudaGetLastError() != cudaSuccess ||
                cudaMemcpyAsync(hubs.data(), d_hub, hubs.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s) !=
                    cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "pair-bound hub readback failed");
                break;
            }
            // H of every query of the round, then the T terms where H could settle it
            std::vector<std::pair<size_t, uint32_t>> jobs;
            for (size_t i : ids) jobs.emplace_back(i, 0u);
            std::vector<double> hv;
            if ((rc = pair_values(G, cs, prep, jobs, d_hub, hub0, d_eok, fe0, nfe, hv))) break;
            std::vector<double> H(Q, 0.0);
            jobs.clear();
            for (size_t k = 0; k < ids.size(); ++k) {
                const size_t i = ids[k];
                H[i] = hv[k];
                if (!prep[i].fvs.empty() && hubs[hub0[i]] != kNone) excl[i].push_back(hubs[hub0[i]]);
                if (H[i] > 0 && (all_terms || lb[i] + H[i] >= two64))
                    for (uint32_t t = 1; t < prep[i].terms.size(); ++t) jobs.emplace_back(i, t);
            }
            std::vector<double> tv;
            if ((rc = pair_values(G, cs, prep, jobs, d_hub, hub0, d_eok, fe0, nfe, tv))) break;
            std::vector<double> S(Q, 0.0);
            for (size_t k = 0; k < jobs.size(); ++k) S[jobs[k].first] = std::nextafter(S[jobs[k].first] + tv[k], HUGE_VAL);
            for (size_t k = 0; k < jobs.size(); ++k) {
                const size_t i = jobs[k].first;
                if (k + 1 < jobs.size() && jobs[k + 1].first == i) continue;  // once per query, at its last term
                const double b = std::nextafter(H[i] - S[i], -HUGE_VAL);
                if (b > 0) lb[i] = lb[i] == 0.0 ? b : std::nextafter(lb[i] + b, 0.0);
            }

        } while (false);
        dfree(d_hub, s);
        dfree(d_eok, s);
        dfree(d_hsegs, s);
        dfree(d_fe, s);
        cudaStreamSynchronize(s);
    }
    if (rc != ASDM_OK) lb.assign(Q, 0.0);
    return rc;
}

}  // namespace

// proven[i] = 1 when query i's count is shown to be at least 2^64 (see the
// overflow proofs above); lower (optional) receives each lower bound, capped
// at 2^64 - 1 (0 where no bound was formed).  Queries are processed in chunks
// of at most kTreeChunkWords weight words.
int overflow_bounds(asdm_graph *G, const std::vector<asdm_cs *> &cs, std::vector<char> &proven,
                    std::vector<uint64_t> *lower) {
    cudaStream_t s = G->stream;
    const size_t Q = cs.size();
    proven.assign(Q, 0);
    if (lower) lower->assign(Q, 0);
    const double two64 = 18446744073709551616.0;  // exactly 2^64
    // tree queries first: their far-class bounds are the tighter ones
    std::vector<double> tlb;
    std::vector<char> tformed;
    ASDM_TRY(tree_bounds(G, cs, tlb, tformed));
    for (size_t i = 0; i < Q; ++i) {
        if (!tformed[i]) continue;
        proven[i] = tlb[i] >= two64;
        if (lower) (*lower)[i] = proven[i] ? ~0ull : (uint64_t)tlb[i];
    }
    struct Prep {
        std::vector<char> fixed;                // u in F
        std::vector<uint32_t> fvs;              // F
        std::vector<uint32_t> cls_k, cls_c;     // classes
        std::vector<uint32_t> parent, height;   // forest over Q - F (kNone: component root)
        std::vector<uint32_t> comp;             // component of each vertex outside F
        std::vector<uint32_t> croot;            // root of each component
        std::vector<char> seg;                  // u needs a weight array
        uint64_t words = 0;
    };
    std::vector<Prep> prep(Q);
    std::vector<char> ok(Q, 0);
    for (size_t i = 0; i < Q; ++i) {
        const asdm_cs &c = *cs[i];
        const QueryGraph &q = c.q;
        if (!c.nonempty || q.n < 2 || proven[i]) continue;
        Prep &P = prep[i];
        const uint32_t n = q.n;
        greedy_fvs(q, P.fixed, P.fvs);
        if (P.fvs.size() > kMaxFixed || P.fvs.size() == n) continue;
        // classes: greedy colouring of each label's conflict graph
        P.cls_k.assign(n, 1);
        P.cls_c.assign(n, 0);
        for (uint32_t u = 0; u < n; ++u) {
            uint64_t used = 0;
            for (uint32_t w = 0; w < u; ++w)
                if (q.lab[w] == q.lab[u] && q.slot(u, w) < 0) used |= 1ull << P.cls_c[w];
            uint32_t c0 = 0;
            while (used >> c0 & 1ull) ++c0;
            P.cls_c[u] = c0;
        }
        for (uint32_t u = 0; u < n; ++u) {
            uint32_t k = 0;
            for (uint32_t w = 0; w < n; ++w)
                if (q.lab[w] == q.lab[u]) k = std::max(k, P.cls_c[w] + 1);
            P.cls_k[u] = k;
        }
        // forest over Q - F: components, parents, heights
        P.parent.assign(n, kNone);
        P.height.assign(n, 0);
        P.comp.assign(n, kNone);
        std::vector<uint32_t> order;
        for (uint32_t r = 0; r < n; ++r) {
            if (P.fixed[r] || P.comp[r] != kNone) continue;
            const size_t first = order.size();
            P.comp[r] = (uint32_t)P.croot.size();
            P.croot.push_back(r);
            order.push_back(r);
            for (size_t k = first; k < order.size(); ++k) {
                const uint32_t u = order[k];
                for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                    const uint32_t w = q.nbr[e];
                    if (P.fixed[w] || P.comp[w] != kNone) continue;
                    P.comp[w] = P.comp[r];
                    P.parent[w] = u;
                    order.push_back(w);
                }
            }
        }
        for (size_t k = order.size(); k-- > 0;) {
            const uint32_t u = order[k];
            if (P.parent[u] != kNone) P.height[P.parent[u]] = std::max(P.height[P.parent[u]], P.height[u] + 1);
        }
        // a vertex needs its own weights unless it is an unrestricted leaf
        // with no fixed neighbour (its parent then takes the list length)
        P.seg.assign(n, 0);
        for (uint32_t u = 0; u < n; ++u) {
            if (P.fixed[u]) continue;
            bool fixed_nbr = false, child = false;
            for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                fixed_nbr |= P.fixed[q.nbr[e]] != 0;
                child |= P.parent[q.nbr[e]] == u;
            }
            P.seg[u] = child || fixed_nbr || P.cls_k[u] > 1 || P.parent[u] == kNone;
            if (P.seg[u]) P.words += c.ncand[u];
        }
        for (uint32_t f : P.fvs) P.words += c.ncand[f];  // the indicator arrays
        ok[i] = 1;
    }
    // Round 0 fixes every vertex of F to its best candidate.  Later rounds
    // (queries with a cycle that are not settled yet) move F's first vertex
    // to its next-best candidates: different images of one vertex count
    // disjoint sets of embeddings, so the rounds' bounds add up (each sum
    // stepped down one ulp to stay a lower bound).
    std::vector<double> acc(Q, 0.0);
    std::vector<std::vector<uint32_t>> excl(Q);
    int rc = ASDM_OK;
    for (uint32_t round = 0; round < kHubRounds && rc == ASDM_OK; ++round) {
    if (round > 0)
        for (size_t i = 0; i < Q; ++i)
            ok[i] = ok[i] && !proven[i] && !prep[i].fvs.empty() && excl[i].size() == round;
    size_t at = 0;
    while (at < Q && rc == ASDM_OK) {
        std::vector<size_t> ids;
        uint64_t words = 0;
        for (; at < Q; ++at) {
            if (!ok[at]) continue;
            if (!ids.empty() && words + prep[at].words > kTreeChunkWords) break;
            words += prep[at].words;
            ids.push_back(at);
        }
        if (ids.empty()) break;
        // descriptor uploads go through the graph's pinned stage: nothing is in flight after this sync
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "overflow-bound sync failed");
            break;
        }
        G->stage.reset();
        std::vector<uint32_t> hub0(ids.size());
        uint32_t nhub = 0;
        for (size_t k = 0; k < ids.size(); ++k) {
            hub0[k] = nhub;
            nhub += (uint32_t)prep[ids[k]].fvs.size();
        }
        double *wbuf = nullptr, *d_out = nullptr, *d_part = nullptr;
        uint32_t *d_hub = nullptr, *d_eok = nullptr, *d_nroot = nullptr;
        BoundSeg *d_segs = nullptr;
        BoundChild *d_kids = nullptr;
        HubSeg *d_hsegs = nullptr;
        FixEdge *d_fe = nullptr;
        BoundQuery *d_bq = nullptr;
        double **d_fw = nullptr;
        const uint32_t **d_fh = nullptr;
        const double **d_roots = nullptr;
        do {
            if ((rc = dalloc(&wbuf, std::max<uint64_t>(words, 1), s)) || (rc = dalloc(&d_out, ids.size(), s)) ||
                (rc = dalloc(&d_hub, std::max<uint32_t>(nhub, 1), s)))
                break;
            if (cudaMemsetAsync(wbuf, 0, std::max<uint64_t>(words, 1) * sizeof(double), s) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "overflow-bound reset failed");
                break;
            }
            // weight arrays: vertices with segments and the fixed vertices' indicators
            std::vector<std::vector<double *>> wptr(ids.size());
            std::vector<HubSeg> hsegs;
            std::vector<double *> fw;
            std::vector<const uint32_t *> fh;
            std::vector<FixEdge> fedges;
            std::vector<uint32_t> fe0(ids.size() + 1, 0);
            uint64_t wo = 0;
            for (size_t k = 0; k < ids.size(); ++k) {
                const asdm_cs &c = *cs[ids[k]];
                const Prep &P = prep[ids[k]];
                wptr[k].assign(c.q.n, nullptr);
                for (uint32_t u = 0; u < c.q.n; ++u)
                    if (P.seg[u] || P.fixed[u]) {
                        wptr[k][u] = wbuf + wo;
                        wo += c.ncand[u];
                    }
                for (size_t j = 0; j < P.fvs.size(); ++j) {
                    const uint32_t f = P.fvs[j];
                    HubSeg hs{c.d_cand + c.cand_base[f], c.ncand[f], P.cls_k[f], P.cls_c[f], 0,
                              d_hub + hub0[k] + j, {}};
                    if (j == 0)
                        for (uint32_t x : excl[ids[k]]) hs.ex[hs.nex++] = x;
                    hsegs.push_back(hs);
                    fw.push_back(wptr[k][f]);
                    fh.push_back(d_hub + hub0[k] + j);
                }
                fe0[k] = (uint32_t)fedges.size();
                for (size_t j = 0; j < P.fvs.size(); ++j)
                    for (size_t j2 = j + 1; j2 < P.fvs.size(); ++j2) {
                        const uint32_t f = P.fvs[j], f2 = P.fvs[j2];
                        const int sl = c.q.slot(f, f2);
                        if (sl < 0) continue;
                        const uint32_t e = c.q.off[f] + (uint32_t)sl;
                        fedges.push_back(FixEdge{c.d_eoff + c.eoff_base[e], c.d_elist + c.elist_base[e],
                                                 d_hub + hub0[k] + j, d_hub + hub0[k] + j2, nullptr});
                    }
            }
            fe0[ids.size()] = (uint32_t)fedges.size();
            const uint32_t ne = (uint32_t)fedges.size();
            if ((rc = dalloc(&d_eok, std::max<uint32_t>(ne, 1), s))) break;
            for (uint32_t e = 0; e < ne; ++e) fedges[e].ok = d_eok + e;
            if (!hsegs.empty()) {
                if ((rc = dalloc(&d_hsegs, hsegs.size(), s)) || (rc = dalloc(&d_fw, fw.size(), s)) ||
                    (rc = dalloc(&d_fh, fh.size(), s)) || (rc = dalloc(&d_fe, std::max<uint32_t>(ne, 1), s)))
                    break;
                if (upload_async(G, d_hsegs, hsegs.data(), hsegs.size() * sizeof(HubSeg)) != cudaSuccess ||
                    upload_async(G, d_fw, fw.data(), fw.size() * sizeof(void *)) != cudaSuccess ||
                    upload_async(G, d_fh, fh.data(), fh.size() * sizeof(void *)) != cudaSuccess ||
                    (ne && upload_async(G, d_fe, fedges.data(), ne * sizeof(FixEdge)) != cudaSuccess)) {
                    rc = fail(ASDM_ERR_CUDA, "overflow-bound upload failed");
                    break;
                }
                if ((rc = launch_pick_hubs(G, d_hsegs, (uint32_t)hsegs.size(), s))) break;
                const uint32_t nfix = (uint32_t)fw.size() + ne;
                fix_weights<<<(nfix + 255) / 256, 256, 0, s>>>(d_fw, d_fh, (uint32_t)fw.size(), d_fe, ne);
                ::asdm::count_launch();
                if (cudaGetLastError() != cudaSuccess) {
                    rc = fail(ASDM_ERR_CUDA, "overflow-bound hub kernels failed");
                    break;
                }
            }
            // segments by height; children: forest children, then fixed copies
            std::vector<std::vector<BoundSeg>> lv;
            std::vector<BoundChild> kids;
            std::vector<const double *> roots;
            std::vector<uint32_t> nroot;
            std::vector<BoundQuery> bqs(ids.size());
            for (size_t k = 0; k < ids.size(); ++k) {
                const asdm_cs &c = *cs[ids[k]];
                const QueryGraph &q = c.q;
                const Prep &P = prep[ids[k]];
                for (uint32_t u = 0; u < q.n; ++u) {
                    if (!P.seg[u]) continue;
                    BoundSeg sg{};
                    sg.w = wptr[k][u];
                    sg.cand = c.d_cand + c.cand_base[u];
                    sg.ncand = c.ncand[u];
                    sg.cls_k = P.cls_k[u];
                    sg.cls_c = P.cls_c[u];
                    sg.child_first = (uint32_t)kids.size();
                    for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                        const uint32_t w = q.nbr[e];
                        if (P.parent[w] == u || P.fixed[w])
                            kids.push_back(BoundChild{c.d_eoff + c.eoff_base[e], c.d_elist + c.elist_base[e],
                                                      wptr[k][w], nullptr});
                    }
                    sg.nchild = (uint32_t)kids.size() - sg.child_first;
                    if (lv.size() <= P.height[u]) lv.resize(P.height[u] + 1);
                    lv[P.height[u]].push_back(sg);
                }
                BoundQuery &bq = bqs[k];
                bq.ncomp = (uint32_t)P.croot.size();
                bq.nhub = (uint32_t)P.fvs.size();
                bq.nedge = fe0[k + 1] - fe0[k];
                bq.out = d_out + k;
                // pointer fields are set once the device arrays exist
                for (uint32_t r : P.croot) {
                    roots.push_back(wptr[k][r]);
                    nroot.push_back(c.ncand[r]);
                }
            }
            std::vector<BoundSeg> segs;
            std::vector<size_t> first{0};
            std::vector<unsigned long long> totals;
            for (auto &l : lv) {
                unsigned long long t = 0;
                for (BoundSeg &sg : l) {
                    sg.start = t;
                    t += sg.ncand;
                    segs.push_back(sg);
                }
                first.push_back(segs.size());
                totals.push_back(t);
            }
            if (kids.empty()) kids.push_back(BoundChild{});
            if (segs.empty()) segs.push_back(BoundSeg{});
            if ((rc = dalloc(&d_segs, segs.size(), s)) || (rc = dalloc(&d_kids, kids.size(), s)) ||
                (rc = dalloc(&d_roots, std::max<size_t>(roots.size(), 1), s)) ||
                (rc = dalloc(&d_nroot, std::max<size_t>(nroot.size(), 1), s)) || (rc = dalloc(&d_bq, ids.size(), s)))
                break;
            uint32_t r0 = 0;
            for (size_t k = 0; k < ids.size(); ++k) {
                bqs[k].roots = d_roots + r0;
                bqs[k].nroot = d_nroot + r0;
                bqs[k].hub = d_hub + hub0[k];
                bqs[k].edge_ok = d_eok + fe0[k];
                r0 += bqs[k].ncomp;
            }
            if ((rc = attach_parts(bqs, &d_part, s))) break;
            if (upload_async(G, d_segs, segs.data(), segs.size() * sizeof(BoundSeg)) != cudaSuccess ||
                upload_async(G, d_kids, kids.data(), kids.size() * sizeof(BoundChild)) != cudaSuccess ||
                upload_async(G, d_roots, roots.data(), roots.size() * sizeof(void *)) != cudaSuccess ||
                upload_async(G, d_nroot, nroot.data(), nroot.size() * sizeof(uint32_t)) != cudaSuccess ||
                upload_async(G, d_bq, bqs.data(), bqs.size() * sizeof(BoundQuery)) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "overflow-bound upload failed");
                break;
            }
            for (size_t h = 0; h < totals.size() && rc == ASDM_OK; ++h) {
                if (!totals[h]) continue;
                const unsigned grid =
                    (unsigned)std::min<unsigned long long>((totals[h] + 255) / 256, (unsigned long long)G->num_sms * 32);
                bound_level<<<grid, 256, 0, s>>>(d_segs + first[h], (uint32_t)(first[h + 1] - first[h]), totals[h],
                                                 d_kids, nullptr);
                ::asdm::count_launch();
                if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "overflow-bound kernel failed");
            }
            if (rc != ASDM_OK) break;
            launch_bound_queries(d_bq, (uint32_t)ids.size(), s);
            std::vector<double> out(ids.size());
            std::vector<uint32_t> hubs(std::max<uint32_t>(nhub, 1));
            if (cudaGetLastError() != cudaSuccess ||
                cudaMemcpyAsync(out.data(), d_out, out.size() * sizeof(double), cudaMemcpyDeviceToHost, s) !=
                    cudaSuccess ||
                cudaMemcpyAsync(hubs.data(), d_hub, hubs.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s) !=
                    cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "overflow-bound readback failed");
                break;
            }
            for (size_t k = 0; k < ids.size(); ++k) {
                const size_t i = ids[k];
                acc[i] = round == 0 ? out[k] : std::nextafter(acc[i] + out[k], 0.0);
                if (!prep[i].fvs.empty() && hubs[hub0[k]] != kNone) excl[i].push_back(hubs[hub0[k]]);
                // the larger of this bound and the tree bound (both count subsets of the embeddings)
                proven[i] = acc[i] >= two64;
                if (lower) (*lower)[i] = std::max<uint64_t>((*lower)[i], proven[i] ? ~0ull : (uint64_t)acc[i]);
            }
        } while (false);
        dfree(wbuf, s);
        dfree(d_out, s);
        dfree(d_hub, s);
        dfree(d_eok, s);
        dfree(d_nroot, s);
        dfree(d_segs, s);
        dfree(d_kids, s);
        dfree(d_hsegs, s);
        dfree(d_fe, s);
        dfree(d_bq, s);
        dfree(d_fw, s);
        dfree(d_fh, s);
        dfree(d_roots, s);
        dfree(d_part, s);
        cudaStreamSynchronize(s);
    }
    }
    // the pair bounds for what is still open
    if (rc == ASDM_OK) {
        std::vector<char> want(Q, 0);
        for (size_t i = 0; i < Q; ++i) want[i] = !proven[i];
        std::vector<double> plb;
        rc = pair_bounds(G, cs, want, plb, lower != nullptr);
        if (rc == ASDM_OK)
            for (size_t i = 0; i < Q; ++i) {
                if (!want[i] || plb[i] <= 0) continue;
                proven[i] = plb[i] >= two64;
                if (lower) (*lower)[i] = std::max<uint64_t>((*lower)[i], proven[i] ? ~0ull : (uint64_t)plb[i]);
            }
    }
    if (rc != ASDM_OK) {
        proven.assign(Q, 0);
        if (lower) lower->assign(Q, 0);
    }
    return rc;
}

// Counts every countable query of `cs` (non-empty candidate spaces on graph
// G); done[i] = 1 and counts[i] set for the queries it settled.  With local
// counts only queries without conflicts are taken.  Queries run in chunks of
// at most kTreeChunkWords device words (one query alone may exceed it).
int tree_counts(asdm_graph *G, const std::vector<asdm_cs *> &cs, std::vector<uint64_t> &counts,
                std::vector<char> &done, const std::vector<unsigned long long *> *local) {
    const size_t Q = cs.size();
    counts.assign(Q, 0);
    done.assign(Q, 0);
    size_t at = 0;
    while (at < Q) {
        std::vector<asdm_cs *> part;
        std::vector<unsigned long long *> lpart;
        std::vector<size_t> ids;
        uint64_t words = 0;
        for (; at < Q; ++at) {
            const uint64_t w = tree_words(*cs[at]);
            if (!ids.empty() && words + w > kTreeChunkWords) break;
            words += w;
            part.push_back(cs[at]);
            if (local) lpart.push_back((*local)[at]);
            ids.push_back(at);
        }
        std::vector<uint64_t> pc;
        std::vector<char> pd;
        const int rc = tree_counts_chunk(G, part, pc, pd, local ? &lpart : nullptr);
        if (rc != ASDM_OK) {
            done.assign(Q, 0);
            return rc;
        }
        for (size_t k = 0; k < ids.size(); ++k) {
            counts[ids[k]] = pc[k];
            done[ids[k]] = pd[k];
        }
    }
    return ASDM_OK;
}

}  // namespace asdm
