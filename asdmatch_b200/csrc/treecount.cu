// Exact counts of tree-shaped queries without enumeration.
//
// Within the candidate space, a map of the query vertices to candidates that
// sends every query edge to a candidate edge is an embedding unless two
// distinct query vertices land on the same data vertex.  Two vertices of
// different labels never do (their candidate sets are disjoint), nor do two
// adjacent vertices (the data graph has no self loops).  So when no two
// non-adjacent query vertices share a label, the count of embeddings equals
// the count of such maps, and for a tree query that count is a bottom-up
// dynamic program over the candidate-edge lists:
//     w_u(i) = prod over children c of u of  sum over j in list_{u->c}(i) of  w_c(j)
//     count  = sum over i of w_root(i)
// (the reference reaches the same number by enumeration: adaptiveShareJoin
// with ALL_LEVEL, matching/adaptive.cpp:1179-2279).  Arithmetic is uint64
// with overflow detection; a query whose program overflows anywhere is left
// to the enumeration kernels, which report ASDM_ERR_OVERFLOW if its count
// itself exceeds 2^64 - 1.
#include <algorithm>

#include "cs.cuh"

namespace asdm {
namespace {

// One (query, query vertex) of a height level of the programs.
struct TreeSeg {
    unsigned long long *w;       // weights of u's candidates (output)
    uint32_t ncand;              // |C(u)|
    uint32_t child_first;        // children in the TreeChild array
    uint32_t nchild;
    uint32_t query;              // index into counts / flags
    uint32_t root;               // 1: add the weights into the query's count
    uint32_t pad;
    unsigned long long start;    // first item of this segment in the launch
};

struct TreeChild {
    const uint32_t *off;              // candidate-edge offsets of (u -> c), by candidate of u
    const uint32_t *list;             // entries: indices into C(c)
    const unsigned long long *w;      // weights of c's candidates (null for a leaf: all 1)
    unsigned long long *s_out;        // local counts: the sum over the list, by candidate of u (or null)
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

// One thread per candidate of the level's query vertices; a list longer than
// 32 entries is summed by the whole warp.
__global__ void tree_level(const TreeSeg *__restrict__ segs, uint32_t nseg, unsigned long long total,
                           const TreeChild *__restrict__ kids, unsigned long long *__restrict__ counts,
                           unsigned int *__restrict__ overflow) {
    const uint32_t lane = threadIdx.x & 31;
    const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < total;
         base += stride) {
        const unsigned long long t = base + lane;
        const bool valid = t < total;
        TreeSeg sg{};
        uint32_t i = 0;
        if (valid) {
            uint32_t lo = 0, hi = nseg;
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (segs[mid].start <= t) lo = mid; else hi = mid;
            }
            sg = segs[lo];
            i = (uint32_t)(t - sg.start);
        }
        unsigned long long acc = 1;
        bool over = false;
        // children are visited in lock step: k-th child of every lane's segment
        uint32_t maxk = valid ? sg.nchild : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) maxk = max(maxk, __shfl_xor_sync(0xffffffffu, maxk, o));
        for (uint32_t k = 0; k < maxk; ++k) {
            const bool mine = valid && k < sg.nchild;
            uint32_t b = 0, e = 0;
            const unsigned long long *w = nullptr;
            const uint32_t *list = nullptr;
            if (mine) {
                const TreeChild ch = kids[sg.child_first + k];
                b = ch.off[i];
                e = ch.off[i + 1];
                w = ch.w;
                list = ch.list;
            }
            // a leaf child contributes its list length
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
        if (!valid) continue;
        if (over) {
            atomicOr(&overflow[sg.query], 1u);
            acc = 0;
        }
        sg.w[i] = acc;
        if (sg.root && acc) {
            const unsigned long long old = atomicAdd(&counts[sg.query], acc);
            if (old + acc < old) atomicOr(&overflow[sg.query], 1u);
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

}  // namespace

// A query the program counts exactly: connected tree, no two non-adjacent
// vertices with one label.
bool tree_countable(const QueryGraph &q) {
    if (q.n < 2 || q.off[q.n] != 2 * (q.n - 1)) return false;
    for (uint32_t u = 0; u < q.n; ++u)
        for (uint32_t w = u + 1; w < q.n; ++w)
            if (q.lab[u] == q.lab[w] && q.slot(u, w) < 0) return false;
    return true;
}

// Counts every countable query of `cs` (non-empty candidate spaces on graph
// G); done[i] = 1 and counts[i] set for the queries it settled.
int tree_counts(asdm_graph *G, const std::vector<asdm_cs *> &cs, std::vector<uint64_t> &counts,
                std::vector<char> &done, const std::vector<unsigned long long *> *local) {
    cudaStream_t s = G->stream;
    const uint32_t Q = (uint32_t)cs.size();
    counts.assign(Q, 0);
    done.assign(Q, 0);
    // rooted trees, vertices grouped by height
    struct Item { uint32_t q, u, parent; };
    std::vector<std::vector<Item>> by_height, by_depth;
    std::vector<uint64_t> qwb(Q, 0);  // per query: first weight
    std::vector<std::vector<uint32_t>> parent(Q);
    uint64_t wtotal = 0;
    std::vector<uint32_t> take;
    for (uint32_t qi = 0; qi < Q; ++qi) {
        const asdm_cs &c = *cs[qi];
        if (!c.nonempty || !tree_countable(c.q)) continue;
        const QueryGraph &q = c.q;
        // root at vertex 0; BFS gives parents, heights from the leaves up
        std::vector<uint32_t> order{0}, par(q.n, kNone), height(q.n, 0);
        std::vector<char> seen(q.n, 0);
        seen[0] = 1;
        for (size_t k = 0; k < order.size(); ++k)
            for (uint32_t e = q.off[order[k]]; e < q.off[order[k] + 1]; ++e) {
                const uint32_t w = q.nbr[e];
                if (!seen[w]) { seen[w] = 1; par[w] = order[k]; order.push_back(w); }
            }
        if (order.size() != q.n) continue;
        for (size_t k = order.size(); k-- > 1;) height[par[order[k]]] = std::max(height[par[order[k]]], height[order[k]] + 1);
        qwb[qi] = wtotal;
        for (uint32_t u = 0; u < q.n; ++u) wtotal += c.ncand[u];
        for (uint32_t u = 0; u < q.n; ++u) {
            if (by_height.size() <= height[u]) by_height.resize(height[u] + 1);
            by_height[height[u]].push_back(Item{qi, u, par[u]});
        }
        {
            std::vector<uint32_t> depth(q.n, 0);
            for (size_t k = 1; k < order.size(); ++k) depth[order[k]] = depth[par[order[k]]] + 1;
            for (uint32_t u = 0; u < q.n; ++u) {
                if (by_depth.size() <= depth[u]) by_depth.resize(depth[u] + 1);
                by_depth[depth[u]].push_back(Item{qi, u, par[u]});
            }
        }
        parent[qi] = par;
        take.push_back(qi);
    }
    if (take.empty()) return ASDM_OK;
    auto wptr_off = [&](uint32_t qi, uint32_t u) {
        uint64_t o = qwb[qi];
        for (uint32_t v = 0; v < u; ++v) o += cs[qi]->ncand[v];
        return o;
    };
    // S_{parent(c), c} has |C(parent)| entries, at sslot[query][c]
    std::vector<std::vector<uint64_t>> sslot(Q);
    uint64_t stotal = 0;
    if (local) {
        for (uint32_t qi : take) {
            const asdm_cs &c = *cs[qi];
            sslot[qi].assign(c.q.n, 0);
        }
        for (const auto &lv : by_height)
            for (const Item &it : lv)
                if (it.parent != kNone) {
                    sslot[it.q][it.u] = stotal;
                    stotal += cs[it.q]->ncand[it.parent];
                }
    }
    unsigned long long *sbase = nullptr;
    auto s_of = [&](uint32_t qi, uint32_t ch) { return sbase + sslot[qi][ch]; };
    unsigned long long *w = nullptr, *d_counts = nullptr, *sums = nullptr, *up = nullptr;
    unsigned int *d_over = nullptr;
    TreeSeg *d_segs = nullptr;
    TreeChild *d_kids = nullptr;
    UpSeg *d_up = nullptr;
    LocSeg *d_loc = nullptr;
    const unsigned long long **d_sibs = nullptr;
    // local counts: the list sums S_{u,c} (one array per tree edge, by
    // candidate of the parent u) and up_u (laid out like the weights)
    int rc = ASDM_OK;
    do {
        if ((rc = dalloc(&w, wtotal, s)) || (rc = dalloc(&d_counts, Q, s)) || (rc = dalloc(&d_over, Q, s))) break;
        if (local && ((rc = dalloc(&sums, std::max<uint64_t>(stotal, 1), s)) || (rc = dalloc(&up, wtotal, s)))) break;
        sbase = sums;
        if (cudaMemsetAsync(d_counts, 0, Q * sizeof(unsigned long long), s) != cudaSuccess ||
            cudaMemsetAsync(d_over, 0, Q * sizeof(unsigned int), s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "tree-count reset failed");
            break;
        }
        // every level's segments and children, uploaded once
        std::vector<TreeSeg> segs;
        std::vector<TreeChild> kids;
        std::vector<size_t> lvl_first{0};
        std::vector<unsigned long long> lvl_total;
        for (size_t h = 0; h < by_height.size(); ++h) {
            unsigned long long total = 0;
            for (const Item &it : by_height[h]) {
                const asdm_cs &c = *cs[it.q];
                const QueryGraph &q = c.q;
                TreeSeg sg{};
                sg.w = w + wptr_off(it.q, it.u);
                sg.ncand = c.ncand[it.u];
                sg.child_first = (uint32_t)kids.size();
                sg.query = it.q;
                sg.root = it.parent == kNone ? 1u : 0u;
                sg.start = total;
                for (uint32_t e = q.off[it.u]; e < q.off[it.u + 1]; ++e) {
                    const uint32_t ch = q.nbr[e];
                    if (ch == it.parent) continue;
                    const bool leaf = q.deg(ch) == 1;
                    kids.push_back(TreeChild{c.d_eoff + c.eoff_base[e], c.d_elist + c.elist_base[e],
                                             leaf ? nullptr : w + wptr_off(it.q, ch), local ? s_of(it.q, ch) : nullptr});
                }
                sg.nchild = (uint32_t)kids.size() - sg.child_first;
                total += sg.ncand;
                segs.push_back(sg);
            }
            lvl_first.push_back(segs.size());
            lvl_total.push_back(total);
        }
        if (kids.empty()) kids.push_back(TreeChild{nullptr, nullptr, nullptr});
        if ((rc = dalloc(&d_segs, segs.size(), s)) || (rc = dalloc(&d_kids, kids.size(), s))) break;
        if (cudaMemcpyAsync(d_segs, segs.data(), segs.size() * sizeof(TreeSeg), cudaMemcpyHostToDevice, s) !=
                cudaSuccess ||
            cudaMemcpyAsync(d_kids, kids.data(), kids.size() * sizeof(TreeChild), cudaMemcpyHostToDevice, s) !=
                cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "tree-count upload failed");
            break;
        }
        for (size_t h = 1; h < by_height.size() && rc == ASDM_OK; ++h) {  // leaves (height 0) weigh 1
            const unsigned long long total = lvl_total[h];
            if (total == 0) continue;
            const unsigned grid =
                (unsigned)std::min<unsigned long long>((total + 255) / 256, (unsigned long long)G->num_sms * 32);
            tree_level<<<grid, 256, 0, s>>>(d_segs + lvl_first[h], (uint32_t)(lvl_first[h + 1] - lvl_first[h]),
                                            total, d_kids, d_counts, d_over);
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
                    const asdm_cs &c = *cs[it.q];
                    const QueryGraph &q = c.q;
                    const uint32_t u = it.parent;
                    const int k = q.slot(it.u, u);  // edge (c -> u)
                    const uint32_t e = q.off[it.u] + (uint32_t)k;
                    UpSeg sg{};
                    sg.up = up + wptr_off(it.q, it.u);
                    sg.off = c.d_eoff + c.eoff_base[e];
                    sg.list = c.d_elist + c.elist_base[e];
                    const std::vector<uint32_t> &par = parent[it.q];
                    sg.up_u = par[u] == kNone ? nullptr : up + wptr_off(it.q, u);
                    sg.sib_first = (uint32_t)sibs.size();
                    for (uint32_t e2 = q.off[u]; e2 < q.off[u + 1]; ++e2) {
                        const uint32_t c2 = q.nbr[e2];
                        if (par[c2] == u && c2 != it.u) sibs.push_back(s_of(it.q, c2));
                    }
                    sg.nsib = (uint32_t)sibs.size() - sg.sib_first;
                    sg.query = it.q;
                    sg.ncand = c.ncand[it.u];
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
                    const bool root = parent[qi][u] == kNone;
                    LocSeg ls{(c.q.deg(u) == 1 && !root) ? nullptr : w + wptr_off(qi, u), root ? nullptr : up + wptr_off(qi, u),
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
