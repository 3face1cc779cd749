// ORACLE — test infrastructure only.
//
// A plain CPU restatement of the reference's matching and counting path, used
// by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg as the
// checker.  The product (asdmatch_b200/, the CLI, the C-ABI library) never
// links, loads or calls it.
//
// Parity is pinned against the reference itself: oracle/ref.mk compiles the
// reference sources into oracle/_ref/{ref_count,ref_local,ref_embed}, and
// tests/golden/ holds counts, local-count CSV digests, embedding digests and
// candidate-space digests produced by those binaries (tests/golden/make_golden.py).
//
// What is restated (reference file:line):
//  * Graph::loadGraphFromTextFile (relation/graph.cpp:68-148): 't N M' header,
//    'v id label degree' lines whose degree sets the CSR offsets, 'e a b'
//    lines appended to both endpoints, other tokens skipped; neighbours sorted
//    by (label, id); vertices grouped by label in id order; numLabels =
//    max label + 1.
//  * nlcValid (utility/utils.cpp:30-40): for every label, the query vertex's
//    neighbour-label count is <= the data vertex's.
//  * CandidateSpace::selectCFLRoot (relation/candidate_space.cpp:723-763),
//    buildCFLBFSTree (:765-816) and buildCandCFL (:550-721).  buildCandCFL is
//    restated as the set formula it computes:
//       F(u)    = { v in V_l(u) : deg v >= deg u, nlc(u) <= nlc(v) }
//       Ctd(r)  = F(r) for the root r
//       Ctd(u)  = F(u) ∩ ⋂_{p in before(u)} N_l(u)(S(p))    (BFS order)
//       C(u)    = Ctd(u) ∩ ⋂_{p in N_q(u) \ before(u)} N_l(u)(S(p))
//    where S(p) is the *storage* the reference scans for p's candidates: the
//    top-down candidates Ctd(p) plus data vertex 0 whenever Ctd(p) is smaller
//    than |V_l(p)| (candidateSet[p] is resized to |V_l(p)| up front and its
//    unused zero-initialised tail is iterated by the range-for loops at
//    :588,:623,:661; pruned entries stay in that storage until the final
//    compaction at :692-703).
//  * CandidateSpace::buildCandidateEdge(false) (:458-487): for query edge
//    (u,u2) and v in C(u), the label-l(u2) neighbours of v that are in C(u2),
//    in adjacency order; CandidateSpace::writeToStream (:489-505) format.
//  * The ALL_LEVEL / LOCAL_COUNT / COLLECT_RESULT results of
//    adaptiveShareJoin (matching/adaptive.cpp:1179-2279 with
//    matching/join.cpp:819-907,1017-1097): the number of injective,
//    label-preserving, edge-preserving maps V_q -> V_g; the |V_g|x|V_q|
//    matrix of how many of them send u to v; the sorted list of the maps in
//    storeMatches format (matching/join.cpp:1099-1107).  Counted here by plain
//    backtracking over the candidate space, which is exact because the CFL
//    filter only removes vertices that cannot be in any embedding.
//  * For tree queries whose counts are too large to enumerate: the same count
//    by inclusion-exclusion over same-label blocks (tree_count below), a
//    restatement of the identity count = sum over partitions pi of mu(pi) *
//    hom(Q/pi) that the product's tree program evaluates on the device
//    (the identity itself is checked against brute-force embedding counts in
//    tests/test_cpu_inclusion_exclusion.py).  Written independently of the
//    device code: set partitions by recursion, quotient homomorphisms by a
//    bottom-up product of sums over data adjacency, in 128-bit integers.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <iostream>
#include <queue>
#include <sstream>
#include <string>
#include <vector>

namespace {

struct OGraph {
    uint32_t n = 0;
    uint64_t m2 = 0;
    uint32_t nlabels = 0;
    std::vector<uint64_t> off;
    std::vector<uint32_t> nbr;
    std::vector<uint32_t> lab;
    std::vector<uint32_t> vbl_off;  // vertices by label: [vbl_off[l], vbl_off[l+1])
    std::vector<uint32_t> vbl;

    uint32_t deg(uint32_t v) const { return (uint32_t)(off[v + 1] - off[v]); }
    // label-l neighbour run of v (neighbours are sorted by (label, id))
    void run(uint32_t v, uint32_t l, uint64_t &b, uint64_t &e) const {
        const uint32_t *base = nbr.data();
        uint64_t lo = off[v], hi = off[v + 1];
        auto cmp_lo = [&](uint32_t x, uint32_t lbl) { return lab[x] < lbl; };
        b = std::lower_bound(base + lo, base + hi, l, cmp_lo) - base;
        uint64_t p = b;
        while (p < hi && lab[base[p]] == l) ++p;
        e = p;
    }
    bool adjacent(uint32_t a, uint32_t b) const {
        uint64_t s, e;
        run(a, lab[b], s, e);
        return std::binary_search(nbr.begin() + s, nbr.begin() + e, b);
    }
    // neighbour-label counts, sorted by label
    std::vector<std::pair<uint32_t, uint32_t>> nlc(uint32_t v) const {
        std::vector<std::pair<uint32_t, uint32_t>> r;
        for (uint64_t i = off[v]; i < off[v + 1]; ++i) {
            uint32_t l = lab[nbr[i]];
            if (!r.empty() && r.back().first == l) ++r.back().second;
            else r.emplace_back(l, 1);
        }
        return r;
    }
};

bool load_graph(const std::string &path, OGraph &g) {
    std::ifstream in(path);
    if (!in.is_open()) return false;
    std::string tok;
    uint64_t m = 0;
    in >> tok >> g.n >> m;
    g.m2 = 2 * m;
    g.off.assign(g.n + 1, 0);
    g.lab.assign(g.n, 0);
    g.nbr.assign(g.m2, 0);
    std::vector<uint64_t> fill(g.n, 0);
    uint32_t maxl = 0;
    while (in >> tok) {
        if (tok == "v") {
            uint64_t id, l, d;
            in >> id >> l >> d;
            g.lab[id] = (uint32_t)l;
            g.off[id + 1] = g.off[id] + d;
            maxl = std::max<uint32_t>(maxl, (uint32_t)l);
        } else if (tok == "e") {
            uint64_t a, b;
            in >> a >> b;
            g.nbr[g.off[a] + fill[a]++] = (uint32_t)b;
            g.nbr[g.off[b] + fill[b]++] = (uint32_t)a;
        }
    }
    g.nlabels = maxl + 1;
    for (uint32_t v = 0; v < g.n; ++v)
        std::sort(g.nbr.begin() + g.off[v], g.nbr.begin() + g.off[v + 1], [&](uint32_t a, uint32_t b) {
            return g.lab[a] != g.lab[b] ? g.lab[a] < g.lab[b] : a < b;
        });
    g.vbl_off.assign(g.nlabels + 1, 0);
    for (uint32_t v = 0; v < g.n; ++v) g.vbl_off[g.lab[v] + 1]++;
    for (uint32_t l = 0; l < g.nlabels; ++l) g.vbl_off[l + 1] += g.vbl_off[l];
    g.vbl.resize(g.n);
    std::vector<uint32_t> pos(g.vbl_off.begin(), g.vbl_off.end() - 1);
    for (uint32_t v = 0; v < g.n; ++v) g.vbl[pos[g.lab[v]]++] = v;
    return true;
}

bool nlc_contained(const std::vector<std::pair<uint32_t, uint32_t>> &qn,
                   const std::vector<std::pair<uint32_t, uint32_t>> &dn) {
    size_t j = 0;
    for (auto &e : qn) {
        while (j < dn.size() && dn[j].first < e.first) ++j;
        if (j == dn.size() || dn[j].first != e.first || dn[j].second < e.second) return false;
    }
    return true;
}

struct CandSpace {
    bool ok = false;
    std::vector<std::vector<uint32_t>> C;  // sorted candidate vertex ids per query vertex
    // edges[u][k] = candidate edge lists for the k-th query neighbour of u:
    // lists[i] = neighbours of C[u][i] (vertex ids) in C[u2]
    std::vector<std::vector<std::vector<std::vector<uint32_t>>>> edges;
    uint32_t root = 0;
    std::vector<uint32_t> bfs_order;
};

void label_vertices(const OGraph &g, uint32_t l, const uint32_t *&p, uint32_t &cnt) {
    if (l >= g.nlabels) { p = nullptr; cnt = 0; return; }
    p = g.vbl.data() + g.vbl_off[l];
    cnt = g.vbl_off[l + 1] - g.vbl_off[l];
}

CandSpace build_cfl(const OGraph &q, const OGraph &g) {
    CandSpace cs;
    const uint32_t nq = q.n;
    std::vector<std::vector<char>> F(nq);
    std::vector<uint32_t> fsize(nq, 0);
    for (uint32_t u = 0; u < nq; ++u) {
        F[u].assign(g.n, 0);
        const uint32_t *vs; uint32_t cnt;
        label_vertices(g, q.lab[u], vs, cnt);
        auto qn = q.nlc(u);
        for (uint32_t i = 0; i < cnt; ++i) {
            uint32_t v = vs[i];
            if (g.deg(v) < q.deg(u)) continue;
            if (!nlc_contained(qn, g.nlc(v))) continue;
            F[u][v] = 1;
            ++fsize[u];
        }
    }
    // Root: keep the three smallest |V_l(u)|/deg(u) in a max-heap (same
    // container and comparator semantics as candidate_space.cpp:724-733), then
    // pop them largest-first and keep the first strict minimum of
    // |F(u)|/deg(u).
    auto cmp = [](const std::pair<uint32_t, double> &a, const std::pair<uint32_t, double> &b) {
        return a.second < b.second;
    };
    std::priority_queue<std::pair<uint32_t, double>, std::vector<std::pair<uint32_t, double>>, decltype(cmp)> pq(cmp);
    for (uint32_t u = 0; u < nq; ++u) {
        const uint32_t *vs; uint32_t cnt;
        label_vertices(g, q.lab[u], vs, cnt);
        pq.emplace(u, cnt / (double)q.deg(u));
    }
    while (pq.size() > 3) pq.pop();
    uint32_t root = 0;
    double best = g.n;
    while (!pq.empty()) {
        uint32_t u = pq.top().first;
        pq.pop();
        double score = fsize[u] / (double)q.deg(u);
        if (score < best) { best = score; root = u; }
    }
    cs.root = root;
    // BFS levels; within a level, discovery order over each vertex's
    // (label, id)-sorted query neighbours.
    std::vector<uint32_t> order;
    std::vector<char> seen(nq, 0);
    std::vector<uint32_t> frontier{root};
    seen[root] = 1;
    while (!frontier.empty()) {
        std::vector<uint32_t> next;
        for (uint32_t u : frontier) {
            order.push_back(u);
            for (uint64_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                uint32_t w = q.nbr[e];
                if (!seen[w]) { seen[w] = 1; next.push_back(w); }
            }
        }
        frontier.swap(next);
    }
    cs.bfs_order = order;
    std::vector<uint32_t> rank(nq, 0);
    for (uint32_t i = 0; i < order.size(); ++i) rank[order[i]] = i;
    // Unreached query vertices (disconnected query) never get candidates in
    // the reference's pass loop; they keep an empty set.
    std::vector<char> reached(nq, 0);
    for (uint32_t u : order) reached[u] = 1;

    auto mark_neighbours = [&](const std::vector<uint32_t> &support, uint32_t l, std::vector<char> &mark) {
        mark.assign(g.n, 0);
        for (uint32_t w : support) {
            uint64_t b, e;
            g.run(w, l, b, e);
            for (uint64_t i = b; i < e; ++i) mark[g.nbr[i]] = 1;
        }
    };
    std::vector<std::vector<uint32_t>> Ctd(nq), S(nq);
    std::vector<char> mark;
    for (uint32_t u : order) {
        std::vector<char> cur = F[u];
        if (u != root) {
            for (uint64_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                uint32_t p = q.nbr[e];
                if (rank[p] >= rank[u]) continue;
                mark_neighbours(S[p], q.lab[u], mark);
                for (uint32_t v = 0; v < g.n; ++v) cur[v] &= mark[v];
            }
        }
        for (uint32_t v = 0; v < g.n; ++v) if (cur[v]) Ctd[u].push_back(v);
        const uint32_t *vs; uint32_t cnt;
        label_vertices(g, q.lab[u], vs, cnt);
        S[u] = Ctd[u];
        if (Ctd[u].size() < cnt) S[u].push_back(0);
    }
    cs.C.assign(nq, {});
    for (uint32_t u = 0; u < nq; ++u) {
        if (!reached[u]) continue;
        std::vector<char> cur(g.n, 0);
        for (uint32_t v : Ctd[u]) cur[v] = 1;
        for (uint64_t e = q.off[u]; e < q.off[u + 1]; ++e) {
            uint32_t p = q.nbr[e];
            if (rank[p] < rank[u]) continue;
            mark_neighbours(S[p], q.lab[u], mark);
            for (uint32_t v = 0; v < g.n; ++v) cur[v] &= mark[v];
        }
        for (uint32_t v = 0; v < g.n; ++v) if (cur[v]) cs.C[u].push_back(v);
    }
    for (uint32_t u = 0; u < nq; ++u)
        if (cs.C[u].empty()) { cs.ok = false; return cs; }
    cs.ok = true;
    cs.edges.assign(nq, {});
    std::vector<std::vector<char>> inC(nq, std::vector<char>(g.n, 0));
    for (uint32_t u = 0; u < nq; ++u) for (uint32_t v : cs.C[u]) inC[u][v] = 1;
    for (uint32_t u = 0; u < nq; ++u) {
        for (uint64_t e = q.off[u]; e < q.off[u + 1]; ++e) {
            uint32_t u2 = q.nbr[e];
            std::vector<std::vector<uint32_t>> lists(cs.C[u].size());
            for (size_t i = 0; i < cs.C[u].size(); ++i) {
                uint64_t b, en;
                g.run(cs.C[u][i], q.lab[u2], b, en);
                for (uint64_t k = b; k < en; ++k)
                    if (inC[u2][g.nbr[k]]) lists[i].push_back(g.nbr[k]);
            }
            cs.edges[u].push_back(std::move(lists));
        }
    }
    return cs;
}

void write_cs(const OGraph &q, const CandSpace &cs, std::ostream &os) {
    for (uint32_t u = 0; u < q.n; ++u) {
        os << "C " << u << " " << cs.C[u].size();
        for (uint32_t v : cs.C[u]) os << " " << v;
        os << "\n";
    }
    for (uint32_t u = 0; u < q.n; ++u) {
        for (uint64_t e = q.off[u], k = 0; e < q.off[u + 1]; ++e, ++k) {
            os << "# " << u << " " << q.nbr[e] << "\n";
            for (size_t i = 0; i < cs.C[u].size(); ++i)
                for (uint32_t v2 : cs.edges[u][k][i]) os << cs.C[u][i] << " " << v2 << "\n";
        }
    }
}

enum { MODE_COUNT = 0, MODE_LOCAL = 1, MODE_EMBED = 2 };

struct Enumerator {
    const OGraph &q, &g;
    const CandSpace &cs;
    int mode;
    std::vector<uint32_t> order;                 // level -> query vertex
    std::vector<uint32_t> first_parent_level;    // level -> level of the parent whose list drives it
    std::vector<uint32_t> first_parent_slot;     // index of u_k in that parent's neighbour list
    std::vector<std::vector<uint32_t>> checks;   // level -> other backward levels (adjacency checks)
    std::vector<uint32_t> phi, phi_idx;          // per level: vertex id, index in C(u)
    std::vector<char> used;
    uint64_t count = 0;
    bool overflow = false;
    std::vector<uint64_t> *local = nullptr;      // |Vg| x |Vq|, row-major
    std::vector<std::vector<uint32_t>> *emb = nullptr;

    Enumerator(const OGraph &q_, const OGraph &g_, const CandSpace &cs_, int mode_)
        : q(q_), g(g_), cs(cs_), mode(mode_) {
        // Connected order: start at the smallest candidate set, then always
        // take the frontier vertex with the most already-ordered neighbours
        // (ties: smaller candidate set, then smaller id).
        const uint32_t nq = q.n;
        std::vector<char> in(nq, 0);
        uint32_t start = 0;
        for (uint32_t u = 1; u < nq; ++u)
            if (cs.C[u].size() < cs.C[start].size()) start = u;
        order.push_back(start);
        in[start] = 1;
        while (order.size() < nq) {
            int best = -1; uint32_t bestConn = 0;
            for (uint32_t u = 0; u < nq; ++u) {
                if (in[u]) continue;
                uint32_t conn = 0;
                for (uint64_t e = q.off[u]; e < q.off[u + 1]; ++e) conn += in[q.nbr[e]];
                if (conn == 0) continue;
                if (best < 0 || conn > bestConn ||
                    (conn == bestConn && cs.C[u].size() < cs.C[best].size())) {
                    best = (int)u; bestConn = conn;
                }
            }
            if (best < 0) break;  // disconnected query: handled by the caller
            order.push_back((uint32_t)best);
            in[best] = 1;
        }
        std::vector<uint32_t> lvl(nq, 0);
        for (uint32_t i = 0; i < order.size(); ++i) lvl[order[i]] = i;
        first_parent_level.assign(nq, 0);
        first_parent_slot.assign(nq, 0);
        checks.assign(nq, {});
        for (uint32_t k = 1; k < order.size(); ++k) {
            uint32_t u = order[k];
            bool have = false;
            for (uint64_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                uint32_t p = q.nbr[e];
                if (lvl[p] >= k) continue;
                if (!have) {
                    have = true;
                    first_parent_level[k] = lvl[p];
                    uint32_t slot = 0;
                    for (uint64_t e2 = q.off[p]; e2 < q.off[p + 1]; ++e2, ++slot)
                        if (q.nbr[e2] == u) break;
                    first_parent_slot[k] = slot;
                } else {
                    checks[k].push_back(lvl[p]);
                }
            }
        }
        phi.assign(nq, 0);
        phi_idx.assign(nq, 0);
        used.assign(g.n, 0);
    }

    void add(uint64_t c) {
        if (__builtin_add_overflow(count, c, &count)) overflow = true;
    }

    void record_full() {
        if (mode == MODE_LOCAL || mode == MODE_EMBED)
            for (uint32_t k = 0; k < q.n; ++k) (*local)[(uint64_t)phi[k] * q.n + order[k]] += 1;
        if (mode == MODE_EMBED) {
            std::vector<uint32_t> row(q.n);
            for (uint32_t k = 0; k < q.n; ++k) row[order[k]] = phi[k];
            emb->push_back(std::move(row));
        }
    }

    void extend(uint32_t k) {
        const uint32_t u = order[k];
        const uint32_t pl = first_parent_level[k];
        const uint32_t pu = order[pl];
        const std::vector<uint32_t> &list = cs.edges[pu][first_parent_slot[k]][phi_idx[pl]];
        for (uint32_t v : list) {
            if (used[v]) continue;
            bool ok = true;
            for (uint32_t j : checks[k])
                if (!g.adjacent(phi[j], v)) { ok = false; break; }
            if (!ok) continue;
            phi[k] = v;
            phi_idx[k] = (uint32_t)(std::lower_bound(cs.C[u].begin(), cs.C[u].end(), v) - cs.C[u].begin());
            if (k + 1 == q.n) {
                add(1);
                record_full();
            } else {
                used[v] = 1;
                extend(k + 1);
                used[v] = 0;
            }
        }
    }

    void run() {
        const uint32_t u0 = order[0];
        for (uint32_t i = 0; i < cs.C[u0].size(); ++i) {
            uint32_t v = cs.C[u0][i];
            phi[0] = v;
            phi_idx[0] = i;
            if (q.n == 1) { add(1); record_full(); continue; }
            used[v] = 1;
            extend(1);
            used[v] = 0;
        }
    }
};

uint32_t vertex_class(uint32_t v, uint32_t k);

// Classes of query vertices for restricted counts: vertex u may only take data
// vertices v with vertex_class(v, k[u]) == c[u] (k[u] <= 1: no restriction).
struct Classes {
    std::vector<uint32_t> k, c;
};

// hom(Q/pi) for the quotient of tree query q by the blocks `block` (block of
// each vertex): a block's candidates are the data vertices that are candidates
// of all its members (and of the members' classes, when given); an edge
// between two blocks needs data adjacency.  Returns false when the quotient is
// not a tree.
bool quotient_hom(const OGraph &q, const OGraph &g, const CandSpace &cs, const std::vector<uint32_t> &block,
                  uint32_t nb, unsigned __int128 &out, const Classes *cls = nullptr) {
    std::vector<std::vector<uint32_t>> adj(nb), members(nb);
    for (uint32_t u = 0; u < q.n; ++u) members[block[u]].push_back(u);
    uint64_t nedges = 0;
    for (uint32_t u = 0; u < q.n; ++u)
        for (uint64_t e = q.off[u]; e < q.off[u + 1]; ++e) {
            const uint32_t a = block[u], b = block[q.nbr[e]];
            if (a == b) return false;
            if (std::find(adj[a].begin(), adj[a].end(), b) == adj[a].end()) {
                adj[a].push_back(b);
                ++nedges;
            }
        }
    if (nedges != 2ull * (nb - 1)) return false;
    // candidates of each block: intersection of its members' candidate sets
    std::vector<std::vector<uint32_t>> cand(nb);
    for (uint32_t b = 0; b < nb; ++b) {
        cand[b] = cs.C[members[b][0]];
        for (size_t k = 1; k < members[b].size(); ++k) {
            std::vector<uint32_t> t;
            const auto &o = cs.C[members[b][k]];
            std::set_intersection(cand[b].begin(), cand[b].end(), o.begin(), o.end(), std::back_inserter(t));
            cand[b].swap(t);
        }
        if (cls)
            for (uint32_t u : members[b]) {
                if (cls->k[u] <= 1) continue;
                std::vector<uint32_t> t;
                for (uint32_t v : cand[b])
                    if (vertex_class(v, cls->k[u]) == cls->c[u]) t.push_back(v);
                cand[b].swap(t);
            }
    }
    // rooted at block 0: BFS order, then weights bottom-up
    std::vector<uint32_t> order{0}, parent(nb, UINT32_MAX);
    std::vector<char> seen(nb, 0);
    seen[0] = 1;
    for (size_t k = 0; k < order.size(); ++k)
        for (uint32_t c : adj[order[k]])
            if (!seen[c]) {
                seen[c] = 1;
                parent[c] = order[k];
                order.push_back(c);
            }
    if (order.size() != nb) return false;
    std::vector<std::vector<unsigned __int128>> w(nb);
    for (size_t k = order.size(); k-- > 0;) {
        const uint32_t b = order[k];
        const uint32_t lb = q.lab[members[b][0]];
        w[b].assign(cand[b].size(), 1);
        for (uint32_t c : adj[b]) {
            if (parent[c] != b) continue;
            const uint32_t lc = q.lab[members[c][0]];
            for (size_t i = 0; i < cand[b].size(); ++i) {
                if (w[b][i] == 0) continue;
                uint64_t s0, s1;
                g.run(cand[b][i], lc, s0, s1);
                unsigned __int128 sum = 0;
                for (uint64_t j = s0; j < s1; ++j) {
                    const auto it = std::lower_bound(cand[c].begin(), cand[c].end(), g.nbr[j]);
                    if (it != cand[c].end() && *it == g.nbr[j]) sum += w[c][it - cand[c].begin()];
                }
                w[b][i] *= sum;
            }
        }
        (void)lb;
    }
    out = 0;
    for (auto x : w[0]) out += x;
    return true;
}

// Exact count of tree query q: sum over the partitions pi of the query
// vertices into blocks of one label whose members are pairwise non-adjacent
// of mu(pi) * hom(Q/pi), mu(pi) = prod over blocks of (-1)^(|B|-1) (|B|-1)!.
// status: 0 exact (count set), 1 the count is >= 2^64, 2 not countable this
// way (a quotient with a cycle, too many partitions, or a term too large).
int tree_count(const OGraph &q, const OGraph &g, const CandSpace &cs, uint64_t &count,
               const Classes *cls = nullptr, unsigned __int128 *wide = nullptr) {
    count = 0;
    if (q.n < 2 || q.m2 != 2ull * (q.n - 1)) return 2;
    std::vector<uint32_t> block(q.n, 0);
    std::vector<std::vector<uint32_t>> members;
    __int128 total = 0;
    size_t partitions = 0;
    bool ok = true;
    const __int128 limit = (__int128)1 << 120;
    std::function<void(uint32_t)> place = [&](uint32_t u) {
        if (!ok) return;
        if (u == q.n) {
            if (++partitions > (1u << 14)) { ok = false; return; }
            __int128 mu = 1;
            for (auto &m : members) {
                __int128 f = 1;
                for (size_t k = 2; k < m.size(); ++k) f *= (__int128)k;
                mu *= (m.size() % 2 == 0) ? -f : f;
            }
            unsigned __int128 h = 0;
            if (!quotient_hom(q, g, cs, block, (uint32_t)members.size(), h, cls) || h >= (unsigned __int128)limit) {
                ok = false;
                return;
            }
            total += mu * (__int128)h;
            return;
        }
        for (size_t b = 0; b < members.size() && ok; ++b) {
            if (q.lab[members[b][0]] != q.lab[u]) continue;
            bool adj = false;
            for (uint32_t w : members[b])
                adj = adj || q.adjacent(u, w) ||
                      (cls && cls->k[u] > 1 && cls->k[w] > 1 && cls->c[u] != cls->c[w]);
            if (adj) continue;
            members[b].push_back(u);
            block[u] = (uint32_t)b;
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
    if (!ok || total < 0) return 2;
    if (wide) *wide = (unsigned __int128)total;
    if (total >= ((__int128)1 << 64)) return 1;
    count = (uint64_t)total;
    return 0;
}

// The device's tighter bound for tree queries, restated: classes (greedy in
// vertex order) only for same-label pairs three or more edges apart, the
// other pairs by inclusion-exclusion; the exact number of embeddings that
// respect those classes.  false when the query is not a tree or the count
// cannot be formed this way.
bool tree_class_bound(const OGraph &q, const OGraph &g, const CandSpace &cs, unsigned __int128 &out) {
    const uint32_t n = q.n;
    if (n < 2 || q.m2 != 2ull * (n - 1)) return false;
    std::vector<std::vector<uint32_t>> dist(n, std::vector<uint32_t>(n, UINT32_MAX));
    for (uint32_t r = 0; r < n; ++r) {
        std::vector<uint32_t> fr{r};
        dist[r][r] = 0;
        for (size_t k = 0; k < fr.size(); ++k)
            for (uint64_t e = q.off[fr[k]]; e < q.off[fr[k] + 1]; ++e)
                if (dist[r][q.nbr[e]] == UINT32_MAX) {
                    dist[r][q.nbr[e]] = dist[r][fr[k]] + 1;
                    fr.push_back(q.nbr[e]);
                }
    }
    std::vector<uint32_t> col(n, UINT32_MAX);
    for (uint32_t u = 0; u < n; ++u) {
        std::vector<char> used(n + 1, 0);
        bool any = false;
        for (uint32_t w = 0; w < n; ++w)
            if (w != u && q.lab[w] == q.lab[u] && dist[u][w] >= 3) {
                any = true;
                if (w < u) used[col[w]] = 1;
            }
        if (!any) continue;
        uint32_t c = 0;
        while (used[c]) ++c;
        col[u] = c;
    }
    Classes cls;
    cls.k.assign(n, 1);
    cls.c.assign(n, 0);
    for (uint32_t u = 0; u < n; ++u) {
        if (col[u] == UINT32_MAX) continue;
        uint32_t k = 0;
        for (uint32_t w = 0; w < n; ++w)
            if (q.lab[w] == q.lab[u] && col[w] != UINT32_MAX) k = std::max(k, col[w] + 1);
        cls.k[u] = k;
        cls.c[u] = col[u];
    }
    uint64_t c64 = 0;
    return tree_count(q, g, cs, c64, &cls, &out) != 2;
}

// The device's overflow lower bound, restated from its definition (the set
// of embeddings it counts), not from the kernels: same-label query vertices
// that are not adjacent get distinct classes (greedy colouring in vertex
// order), a query vertex may only take candidates whose hashed class is its
// own; a feedback vertex set (peel vertices of degree <= 1, then take the
// vertex of highest remaining degree, lowest id first) is fixed to the
// highest-degree candidate of its class (lowest id on ties); the forest left
// is counted exactly.  Returns 0 and lb (saturated at 2^127) when a bound is
// formed, 1 when the rules form none (more than 6 fixed vertices).
uint32_t vertex_class(uint32_t v, uint32_t k) {
    return (uint32_t)((((unsigned __int128)v * 0x9E3779B97F4A7C15ull) >> 32) % k);
}

int lower_bound(const OGraph &q, const OGraph &g, const CandSpace &cs, unsigned __int128 &lb) {
    const uint32_t n = q.n;
    const unsigned __int128 kSat = (unsigned __int128)1 << 127;
    auto sat_mul = [&](unsigned __int128 a, unsigned __int128 b) -> unsigned __int128 {
        if (a == 0 || b == 0) return 0;
        if (a >= kSat || b >= kSat || a > kSat / b) return kSat;
        return a * b;
    };
    auto sat_add = [&](unsigned __int128 a, unsigned __int128 b) -> unsigned __int128 {
        return (a >= kSat || b >= kSat || a + b >= kSat) ? kSat : a + b;
    };
    lb = 0;
    std::vector<char> fixed(n, 0), gone(n, 0);
    std::vector<uint32_t> fvs, deg(n);
    for (uint32_t u = 0; u < n; ++u) deg[u] = q.deg(u);
    auto drop = [&](uint32_t u) {
        gone[u] = 1;
        for (uint64_t e = q.off[u]; e < q.off[u + 1]; ++e)
            if (!gone[q.nbr[e]]) --deg[q.nbr[e]];
    };
    for (;;) {
        for (bool changed = true; changed;) {
            changed = false;
            for (uint32_t u = 0; u < n; ++u)
                if (!gone[u] && deg[u] <= 1) { drop(u); changed = true; }
        }
        int best = -1;
        for (uint32_t u = 0; u < n; ++u)
            if (!gone[u] && (best < 0 || deg[u] > deg[best])) best = (int)u;
        if (best < 0) break;
        fixed[best] = 1;
        fvs.push_back((uint32_t)best);
        drop((uint32_t)best);
    }
    if (fvs.size() > 6 || fvs.size() == n) return 1;
    std::vector<uint32_t> cls(n, 0), ncls(n, 1);
    for (uint32_t u = 0; u < n; ++u) {
        std::vector<char> used(n + 1, 0);
        for (uint32_t w = 0; w < u; ++w)
            if (q.lab[w] == q.lab[u] && !q.adjacent(u, w)) used[cls[w]] = 1;
        while (used[cls[u]]) ++cls[u];
    }
    for (uint32_t u = 0; u < n; ++u)
        for (uint32_t w = 0; w < n; ++w)
            if (q.lab[w] == q.lab[u]) ncls[u] = std::max(ncls[u], cls[w] + 1);
    auto allowed = [&](uint32_t u, uint32_t v) { return ncls[u] <= 1 || vertex_class(v, ncls[u]) == cls[u]; };
    std::vector<uint32_t> hub(n, UINT32_MAX);
    for (uint32_t f : fvs) {
        for (uint32_t v : cs.C[f])
            if (allowed(f, v) && (hub[f] == UINT32_MAX || g.deg(v) > g.deg(hub[f]))) hub[f] = v;
        if (hub[f] == UINT32_MAX) return 0;  // lb = 0
    }
    for (uint32_t f : fvs)
        for (uint32_t f2 : fvs)
            if (f < f2 && q.adjacent(f, f2) && !g.adjacent(hub[f], hub[f2])) return 0;
    // forest components, rooted at their lowest vertex; weights bottom-up
    std::vector<uint32_t> comp(n, UINT32_MAX), parent(n, UINT32_MAX), order;
    unsigned __int128 prod = 1;
    for (uint32_t r = 0; r < n; ++r) {
        if (fixed[r] || comp[r] != UINT32_MAX) continue;
        const size_t first = order.size();
        comp[r] = r;
        order.push_back(r);
        for (size_t k = first; k < order.size(); ++k)
            for (uint64_t e = q.off[order[k]]; e < q.off[order[k] + 1]; ++e) {
                const uint32_t w = q.nbr[e];
                if (fixed[w] || comp[w] != UINT32_MAX) continue;
                comp[w] = r;
                parent[w] = order[k];
                order.push_back(w);
            }
        std::vector<std::vector<unsigned __int128>> wt(n);
        for (size_t k = order.size(); k-- > first;) {
            const uint32_t u = order[k];
            const auto &C = cs.C[u];
            wt[u].assign(C.size(), 0);
            for (size_t i = 0; i < C.size(); ++i) {
                if (!allowed(u, C[i])) continue;
                unsigned __int128 acc = 1;
                for (uint64_t e = q.off[u]; e < q.off[u + 1] && acc; ++e) {
                    const uint32_t c = q.nbr[e];
                    if (fixed[c]) {
                        acc = g.adjacent(C[i], hub[c]) ? acc : 0;
                    } else if (parent[c] == u) {
                        uint64_t s0, s1;
                        g.run(C[i], q.lab[c], s0, s1);
                        unsigned __int128 sum = 0;
                        for (uint64_t j = s0; j < s1; ++j) {
                            const auto it = std::lower_bound(cs.C[c].begin(), cs.C[c].end(), g.nbr[j]);
                            if (it != cs.C[c].end() && *it == g.nbr[j]) sum = sat_add(sum, wt[c][it - cs.C[c].begin()]);
                        }
                        acc = sat_mul(acc, sum);
                    }
                }
                wt[u][i] = acc;
            }
        }
        unsigned __int128 tot = 0;
        for (auto x : wt[r]) tot = sat_add(tot, x);
        prod = sat_mul(prod, tot);
    }
    lb = prod;
    return 0;
}

// The device's pair bound, restated for its first round of hubs: F as in
// lower_bound, each vertex of F on the largest-degree candidate of its class,
// classes now only among F's same-label vertices (the r-th of k in F's order
// takes class r); H = the homomorphisms with F on its hubs; for every
// same-label, non-adjacent pair not both in F, T = the homomorphisms with one
// of them pinned to the other's hub (one in F) or with the two merged into one
// block on the candidates of both, the forest of the merged query built
// breadth-first (blocks in order of their lowest member, from the lowest
// unvisited one, members in id order, neighbours in adjacency order, an edge
// into a visited block left out).  bound = H - sum T when positive.  Exact
// 128-bit integers (a saturated T sum gives no bound).  Returns false when no
// bound is formed.
bool pair_bound(const OGraph &q, const OGraph &g, const CandSpace &cs, unsigned __int128 &out) {
    const uint32_t n = q.n;
    const unsigned __int128 kSat = (unsigned __int128)1 << 127;
    auto sat_mul = [&](unsigned __int128 a, unsigned __int128 b) -> unsigned __int128 {
        if (a == 0 || b == 0) return 0;
        if (a >= kSat || b >= kSat || a > kSat / b) return kSat;
        return a * b;
    };
    auto sat_add = [&](unsigned __int128 a, unsigned __int128 b) -> unsigned __int128 {
        return (a >= kSat || b >= kSat || a + b >= kSat) ? kSat : a + b;
    };
    out = 0;
    // F: peel leaves, fix the vertex of highest remaining degree
    std::vector<char> fixed(n, 0), gone(n, 0);
    std::vector<uint32_t> fvs, deg(n);
    for (uint32_t u = 0; u < n; ++u) deg[u] = q.deg(u);
    auto drop = [&](uint32_t u) {
        gone[u] = 1;
        for (uint64_t e = q.off[u]; e < q.off[u + 1]; ++e)
            if (!gone[q.nbr[e]]) --deg[q.nbr[e]];
    };
    for (;;) {
        for (bool changed = true; changed;) {
            changed = false;
            for (uint32_t u = 0; u < n; ++u)
                if (!gone[u] && deg[u] <= 1) { drop(u); changed = true; }
        }
        int best = -1;
        for (uint32_t u = 0; u < n; ++u)
            if (!gone[u] && (best < 0 || deg[u] > deg[best])) best = (int)u;
        if (best < 0) break;
        fixed[best] = 1;
        fvs.push_back((uint32_t)best);
        drop((uint32_t)best);
    }
    if (fvs.size() > 6 || fvs.size() == n) return false;
    std::vector<uint32_t> hub(n, UINT32_MAX);
    for (size_t j = 0; j < fvs.size(); ++j) {
        uint32_t c = 0, k = 0;
        for (size_t j2 = 0; j2 < fvs.size(); ++j2)
            if (q.lab[fvs[j2]] == q.lab[fvs[j]]) {
                if (j2 < j) ++c;
                ++k;
            }
        const uint32_t f = fvs[j];
        for (uint32_t v : cs.C[f])
            if ((k <= 1 || vertex_class(v, k) == c) && (hub[f] == UINT32_MAX || g.deg(v) > g.deg(hub[f]))) hub[f] = v;
        if (hub[f] == UINT32_MAX) return false;
    }
    for (uint32_t f : fvs)
        for (uint32_t f2 : fvs)
            if (f < f2 && q.adjacent(f, f2) && !g.adjacent(hub[f], hub[f2])) return false;
    // the homomorphisms of one program
    auto count = [&](uint32_t ma, uint32_t mb, uint32_t pin, uint32_t pinv) -> unsigned __int128 {
        std::vector<uint32_t> block(n, UINT32_MAX);
        std::vector<std::vector<uint32_t>> members;
        for (uint32_t u = 0; u < n; ++u) {
            if (fixed[u] || u == mb) continue;
            block[u] = (uint32_t)members.size();
            members.push_back({u});
        }
        if (mb != UINT32_MAX) {
            block[mb] = block[ma];
            members[block[ma]].push_back(mb);
            std::sort(members[block[ma]].begin(), members[block[ma]].end());
        }
        const uint32_t nb = (uint32_t)members.size();
        std::vector<std::vector<uint32_t>> cand(nb);
        for (uint32_t b = 0; b < nb; ++b) {
            cand[b] = cs.C[members[b][0]];
            for (size_t k = 1; k < members[b].size(); ++k) {
                std::vector<uint32_t> t;
                const auto &o = cs.C[members[b][k]];
                std::set_intersection(cand[b].begin(), cand[b].end(), o.begin(), o.end(), std::back_inserter(t));
                cand[b].swap(t);
            }
            if (pin != UINT32_MAX && block[pin] == b) {
                const bool has = std::binary_search(cand[b].begin(), cand[b].end(), pinv);
                cand[b].clear();
                if (has) cand[b].push_back(pinv);
            }
        }
        // breadth-first forest; the tree edge into block C leaves member pfrom[C] for vertex crep[C]
        std::vector<uint32_t> parent(nb, UINT32_MAX), pfrom(nb, UINT32_MAX), crep(nb, UINT32_MAX), order;
        std::vector<char> seen(nb, 0);
        for (uint32_t r = 0; r < nb; ++r) {
            if (seen[r]) continue;
            seen[r] = 1;
            const size_t first = order.size();
            order.push_back(r);
            for (size_t k = first; k < order.size(); ++k) {
                const uint32_t B = order[k];
                for (uint32_t u : members[B])
                    for (uint64_t e = q.off[u]; e < q.off[u + 1]; ++e) {
                        const uint32_t w = q.nbr[e];
                        if (fixed[w]) continue;
                        const uint32_t C = block[w];
                        if (C == B || seen[C]) continue;
                        seen[C] = 1;
                        parent[C] = B;
                        pfrom[C] = u;
                        crep[C] = w;
                        order.push_back(C);
                    }
            }
        }
        std::vector<std::vector<unsigned __int128>> wt(nb);
        for (size_t k = order.size(); k-- > 0;) {
            const uint32_t B = order[k];
            wt[B].assign(cand[B].size(), 0);
            for (size_t i = 0; i < cand[B].size(); ++i) {
                const uint32_t v = cand[B][i];
                unsigned __int128 acc = 1;
                for (uint32_t u : members[B])
                    for (uint64_t e = q.off[u]; e < q.off[u + 1] && acc; ++e) {
                        const uint32_t w = q.nbr[e];
                        if (fixed[w]) {
                            if (!g.adjacent(v, hub[w])) acc = 0;
                            continue;
                        }
                        const uint32_t C = block[w];
                        if (parent[C] != B || pfrom[C] != u || crep[C] != w) continue;
                        uint64_t s0, s1;
                        g.run(v, q.lab[w], s0, s1);
                        unsigned __int128 sum = 0;
                        for (uint64_t j = s0; j < s1; ++j) {
                            const auto it = std::lower_bound(cand[C].begin(), cand[C].end(), g.nbr[j]);
                            if (it != cand[C].end() && *it == g.nbr[j]) sum = sat_add(sum, wt[C][it - cand[C].begin()]);
                        }
                        acc = sat_mul(acc, sum);
                    }
                wt[B][i] = acc;
            }
        }
        unsigned __int128 prod = 1;
        for (uint32_t b = 0; b < nb; ++b) {
            if (parent[b] != UINT32_MAX) continue;
            unsigned __int128 tot = 0;
            for (auto x : wt[b]) tot = sat_add(tot, x);
            prod = sat_mul(prod, tot);
        }
        return prod;
    };
    const unsigned __int128 H = count(UINT32_MAX, UINT32_MAX, UINT32_MAX, 0);
    unsigned __int128 S = 0;
    bool pairs = false;
    for (uint32_t a = 0; a < n; ++a)
        for (uint32_t b = a + 1; b < n; ++b) {
            if (q.lab[a] != q.lab[b] || q.adjacent(a, b) || (fixed[a] && fixed[b])) continue;
            pairs = true;
            if (fixed[a]) S = sat_add(S, count(UINT32_MAX, UINT32_MAX, b, hub[a]));
            else if (fixed[b]) S = sat_add(S, count(UINT32_MAX, UINT32_MAX, a, hub[b]));
            else S = sat_add(S, count(a, b, UINT32_MAX, 0));
        }
    if (!pairs || S >= kSat) return false;
    out = H > S ? H - S : 0;
    return true;
}

struct RunResult {
    uint64_t count = 0;
    bool overflow = false;
    bool empty_cs = false;
};

int run_files(const char *qpath, const char *dpath, int mode, RunResult &res, const char *csv,
              const char *embp, const char *csp) {
    OGraph q, g;
    if (!load_graph(qpath, q) || !load_graph(dpath, g)) return 2;
    CandSpace cs = build_cfl(q, g);
    std::vector<uint64_t> local;
    std::vector<std::vector<uint32_t>> emb;
    if (!cs.ok) {
        res.empty_cs = true;
        res.count = 0;
        local.assign((uint64_t)g.n * q.n, 0);
    } else {
        if (csp && *csp) {
            std::ofstream os(csp);
            write_cs(q, cs, os);
        }
        Enumerator en(q, g, cs, mode);
        if (en.order.size() != q.n) return 3;  // disconnected query
        if (mode != MODE_COUNT) local.assign((uint64_t)g.n * q.n, 0);
        en.local = &local;
        en.emb = &emb;
        en.run();
        res.count = en.count;
        res.overflow = en.overflow;
    }
    if (csv && *csv && mode != MODE_COUNT) {
        std::ofstream os(csv);
        for (uint32_t v = 0; v < g.n; ++v) {
            for (uint32_t u = 0; u < q.n; ++u) {
                os << local[(uint64_t)v * q.n + u];
                if (u + 1 != q.n) os << ",";
            }
            os << "\n";
        }
    }
    if (embp && *embp && mode == MODE_EMBED) {
        std::sort(emb.begin(), emb.end());
        std::ofstream os(embp);
        os << emb.size() << "\n";
        for (auto &r : emb) {
            for (uint32_t v : r) os << v << " ";
            os << "\n";
        }
    }
    return 0;
}

}  // namespace

extern "C" {

// mode: 0 count, 1 local counts (csv), 2 local counts + embeddings.
// Returns 0 on success, 2 unreadable file, 3 disconnected query.
// *flags: bit0 = uint64 overflow of the count, bit1 = empty candidate set.
int orc_run(const char *qpath, const char *dpath, int mode, uint64_t *count, uint32_t *flags,
            const char *csv_path, const char *emb_path, const char *cs_path) {
    RunResult r;
    int rc = run_files(qpath, dpath, mode, r, csv_path, emb_path, cs_path);
    if (count) *count = r.count;
    if (flags) *flags = (r.overflow ? 1u : 0u) | (r.empty_cs ? 2u : 0u);
    return rc;
}

// Tree queries of a list file (one path per line) against one data graph,
// loaded once: one line per query on stdout, "T <k> ok <count>",
// "T <k> overflow", "T <k> empty" (a candidate set is empty: count 0) or
// "T <k> skip" (not a tree countable this way).
int orc_tree_list(const char *dpath, const char *list) {
    OGraph g;
    if (!load_graph(dpath, g)) return 2;
    std::ifstream in(list);
    std::string qp;
    for (uint32_t k = 0; std::getline(in, qp); ++k) {
        if (qp.empty()) continue;
        OGraph q;
        if (!load_graph(qp, q)) return 2;
        CandSpace cs = build_cfl(q, g);
        if (!cs.ok) {
            std::cout << "T " << k << " empty" << std::endl;
            continue;
        }
        uint64_t c = 0;
        const int st = tree_count(q, g, cs, c);
        if (st == 0) std::cout << "T " << k << " ok " << c << std::endl;
        else if (st == 1) std::cout << "T " << k << " overflow" << std::endl;
        else std::cout << "T " << k << " skip" << std::endl;
    }
    return 0;
}

// The lower bounds of the queries of a list file against one data graph:
// "B <k> <bound>" (decimal, saturated at 2^127; the largest of the general
// bound, for trees the far-class tree bound, and the first-round pair bound),
// "B <k> none" when the rules form no bound, "B <k> empty" for an empty
// candidate set.
int orc_bound_list(const char *dpath, const char *list) {
    OGraph g;
    if (!load_graph(dpath, g)) return 2;
    std::ifstream in(list);
    std::string qp;
    for (uint32_t k = 0; std::getline(in, qp); ++k) {
        if (qp.empty()) continue;
        OGraph q;
        if (!load_graph(qp, q)) return 2;
        CandSpace cs = build_cfl(q, g);
        if (!cs.ok) {
            std::cout << "B " << k << " empty" << std::endl;
            continue;
        }
        unsigned __int128 lb = 0, tb = 0, pb = 0;
        const bool general = lower_bound(q, g, cs, lb) == 0;
        // the device reports the largest of its bounds
        const bool tree = tree_class_bound(q, g, cs, tb);
        if (tree && tb > lb) lb = tb;
        const bool pair = pair_bound(q, g, cs, pb);
        if (pair && pb > lb) lb = pb;
        if (!general && !tree && !pair) {
            std::cout << "B " << k << " none" << std::endl;
            continue;
        }
        char buf[64];
        int p = 63;
        buf[p] = 0;
        do {
            buf[--p] = (char)('0' + (int)(lb % 10));
            lb /= 10;
        } while (lb);
        std::cout << "B " << k << " " << (buf + p) << std::endl;
    }
    return 0;
}

}  // extern "C"

#ifdef ORACLE_MAIN
// CLI: asdm_oracle -q Q -d D [-c csv] [-e emb] [-w csdump]; prints the
// reference's "Number of matches:" line.  asdm_oracle -d D -t LIST: the tree
// counts of the queries listed in LIST (orc_tree_list); -b LIST: their
// overflow lower bounds (orc_bound_list).
int main(int argc, char **argv) {
    std::string qp, dp, csv, emb, csd, tl, bl;
    for (int i = 1; i + 1 < argc; ++i) {
        std::string a = argv[i];
        if (a == "-t") tl = argv[i + 1];
        if (a == "-b") bl = argv[i + 1];
        if (a == "-q") qp = argv[i + 1];
        else if (a == "-d") dp = argv[i + 1];
        else if (a == "-c") csv = argv[i + 1];
        else if (a == "-e") emb = argv[i + 1];
        else if (a == "-w") csd = argv[i + 1];
    }
    if (!tl.empty()) return orc_tree_list(dp.c_str(), tl.c_str()) == 0 ? 0 : 1;
    if (!bl.empty()) return orc_bound_list(dp.c_str(), bl.c_str()) == 0 ? 0 : 1;
    int mode = !emb.empty() ? MODE_EMBED : (!csv.empty() ? MODE_LOCAL : MODE_COUNT);
    uint64_t c = 0;
    uint32_t fl = 0;
    int rc = orc_run(qp.c_str(), dp.c_str(), mode, &c, &fl, csv.c_str(), emb.c_str(), csd.c_str());
    if (rc == 2) { std::cout << "Can not open file ." << std::endl; return 1; }
    if (rc != 0) { std::cout << "error " << rc << std::endl; return 1; }
    std::cout << "Number of matches: " << c << std::endl;
    if (fl & 1) std::cout << "overflow" << std::endl;
    return 0;
}
#endif
