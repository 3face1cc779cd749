// The reference's binary graph cache: the layout Graph::writeToStream writes
// and Graph::readFromStream reads (relation/graph.cpp:293-332, with the
// stream helpers of utility/utils.h:54-109), all little-endian:
//   u32 |V|, u32 2|E| (directed edges), u32 L (max label + 1)
//   u32 labels[|V|], u32 offsets[|V|+1], u32 reverseID[2|E|], u32 nbrs[2|E|]
//   per vertex: u64 k, k x (u32 label, u32 count)        neighbour-label counts
//   per vertex: u64 k, k x (u32 label, u32 first edge)   label-run starts
//   u64 k, k x (u32 label, u32 count)                    vertices per label (every label < L)
//   u32 offset2[L+1]                                     label offsets of verticesByLabel
//   u32 verticesByLabel[|V|]
// (an array of size 0 is not written at all).  reverseID[e] is the position of
// the opposite direction of edge e.  The reader keeps the CSR and labels and
// checks the rest against them.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>

#include "internal.h"

using namespace asdm;

namespace {

struct Out {
    FILE *f;
    bool ok = true;
    void put(const void *p, size_t n) {
        if (n && std::fwrite(p, 1, n, f) != n) ok = false;
    }
    void u32(uint32_t x) { put(&x, 4); }
    void u64(uint64_t x) { put(&x, 8); }
};

// label runs of v: (label, first edge, count)
template <typename F>
void for_runs(const asdm_host_graph &g, uint32_t v, F &&f) {
    uint32_t e = g.off[v];
    while (e < g.off[v + 1]) {
        const uint32_t l = g.lab[g.nbr[e]];
        uint32_t k = e;
        while (k < g.off[v + 1] && g.lab[g.nbr[k]] == l) ++k;
        f(l, e, k - e);
        e = k;
    }
}

// position of w in v's adjacency (sorted by (label, id)), or ~0u
uint32_t edge_of(const asdm_host_graph &g, uint32_t v, uint32_t w) {
    uint32_t lo = g.off[v], hi = g.off[v + 1];
    const uint32_t lw = g.lab[w];
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t x = g.nbr[mid], lx = g.lab[x];
        if (lx < lw || (lx == lw && x < w)) lo = mid + 1; else hi = mid;
    }
    return lo < g.off[v + 1] && g.nbr[lo] == w ? lo : ~0u;
}

}  // namespace

extern "C" int asdm_host_graph_write_binary(const asdm_host_graph *g, const char *path) {
    clear_error();
    if (!g || !path) return fail(ASDM_ERR_INVALID, "null argument");
    if (g->m2 > 0xFFFFFFFFull) return fail(ASDM_ERR_INVALID, "edge count exceeds the format's 32 bits");
    // the reverse edge of every directed edge
    std::vector<uint32_t> rev(g->m2);
    for (uint32_t v = 0; v < g->n; ++v)
        for (uint32_t e = g->off[v]; e < g->off[v + 1]; ++e) {
            const uint32_t r = edge_of(*g, g->nbr[e], v);
            if (r == ~0u) return fail(ASDM_ERR_INVALID, "edge %u -> %u has no reverse", v, g->nbr[e]);
            rev[e] = r;
        }
    std::vector<uint32_t> lcount(g->nlabels, 0), offset2((size_t)g->nlabels + 1, 0), vbl(g->n);
    for (uint32_t v = 0; v < g->n; ++v) lcount[g->lab[v]]++;
    for (uint32_t l = 0; l < g->nlabels; ++l) offset2[l + 1] = offset2[l] + lcount[l];
    {
        std::vector<uint32_t> fill(offset2.begin(), offset2.end() - 1);
        for (uint32_t v = 0; v < g->n; ++v) vbl[fill[g->lab[v]]++] = v;
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(ASDM_ERR_IO, "Can not open file %s .", path);
    Out o{f};
    o.u32(g->n);
    o.u32((uint32_t)g->m2);
    o.u32(g->nlabels);
    o.put(g->lab.data(), 4ull * g->n);
    o.put(g->off.data(), 4ull * (g->n + 1));
    o.put(rev.data(), 4ull * g->m2);
    o.put(g->nbr.data(), 4ull * g->m2);
    for (int pass = 0; pass < 2; ++pass)
        for (uint32_t v = 0; v < g->n; ++v) {
            uint64_t k = 0;
            for_runs(*g, v, [&](uint32_t, uint32_t, uint32_t) { ++k; });
            o.u64(k);
            for_runs(*g, v, [&](uint32_t l, uint32_t first, uint32_t cnt) {
                o.u32(l);
                o.u32(pass == 0 ? cnt : first);
            });
        }
    o.u64(g->nlabels);
    for (uint32_t l = 0; l < g->nlabels; ++l) {
        o.u32(l);
        o.u32(lcount[l]);
    }
    o.put(offset2.data(), 4ull * (g->nlabels + 1));
    o.put(vbl.data(), 4ull * g->n);
    const bool ok = o.ok;
    if (std::fclose(f) != 0 || !ok) return fail(ASDM_ERR_IO, "write to %s failed", path);
    return ASDM_OK;
}

extern "C" int asdm_host_graph_load_binary(const char *path, asdm_host_graph **out) {
    clear_error();
    if (!path || !out) return fail(ASDM_ERR_INVALID, "null argument");
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) return fail(ASDM_ERR_IO, "Can not open the binary graph file.");
    std::vector<uint8_t> buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    size_t at = 0;
    bool ok = true;
    auto take = [&](void *dst, size_t n) {
        if (!ok || buf.size() - at < n) { ok = false; return; }
        if (n) std::memcpy(dst, buf.data() + at, n);
        at += n;
    };
    auto u32 = [&]() { uint32_t x = 0; take(&x, 4); return x; };
    auto u64 = [&]() { uint64_t x = 0; take(&x, 8); return x; };
    auto g = std::make_unique<asdm_host_graph>();
    g->n = u32();
    g->m2 = u32();
    g->nlabels = u32();
    if (!ok) return fail(ASDM_ERR_INVALID, "%s: truncated header", path);
    const uint64_t need = 4ull * (g->n + (g->n + 1ull) + 2 * g->m2);
    if (buf.size() - at < need) return fail(ASDM_ERR_INVALID, "%s: truncated arrays", path);
    g->lab.resize(g->n);
    g->off.resize(g->n + 1ull);
    g->nbr.resize(g->m2);
    std::vector<uint32_t> rev(g->m2);
    take(g->lab.data(), 4ull * g->n);
    take(g->off.data(), 4ull * (g->n + 1));
    take(rev.data(), 4ull * g->m2);
    take(g->nbr.data(), 4ull * g->m2);
    // structural checks, then the derived tables against the CSR
    if (g->off[0] != 0 || g->off[g->n] != g->m2) return fail(ASDM_ERR_INVALID, "%s: offsets do not span the edges", path);
    for (uint32_t v = 0; v < g->n; ++v) {
        if (g->off[v + 1] < g->off[v]) return fail(ASDM_ERR_INVALID, "%s: offsets not monotone", path);
        if (g->lab[v] >= g->nlabels) return fail(ASDM_ERR_INVALID, "%s: label out of range", path);
    }
    for (uint64_t e = 0; e < g->m2; ++e)
        if (g->nbr[e] >= g->n || rev[e] >= g->m2) return fail(ASDM_ERR_INVALID, "%s: edge entry out of range", path);
    for (int pass = 0; pass < 2 && ok; ++pass)
        for (uint32_t v = 0; v < g->n && ok; ++v) {
            const uint64_t k = u64();
            if (!ok || k > g->nlabels) { ok = false; break; }
            for (uint64_t i = 0; i < k; ++i) {
                u32();
                u32();
            }
        }
    const uint64_t nl = ok ? u64() : 0;
    if (!ok || nl > g->nlabels + 1ull) return fail(ASDM_ERR_INVALID, "%s: bad label tables", path);
    for (uint64_t i = 0; i < nl; ++i) {
        u32();
        u32();
    }
    std::vector<uint32_t> offset2((size_t)g->nlabels + 1), vbl(g->n);
    take(offset2.data(), 4ull * (g->nlabels + 1));
    take(vbl.data(), 4ull * g->n);
    if (!ok || at != buf.size()) return fail(ASDM_ERR_INVALID, "%s: not a binary graph file", path);
    *out = g.release();
    return ASDM_OK;
}
