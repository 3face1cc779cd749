// Host-side graphs: the 't/v/e' loader and writer, CSR construction, and the
// seeded synthetic generators (Chung-Lu data graphs, random-walk queries).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <numeric>
#include <sstream>

#include "internal.h"

namespace asdm {

static thread_local std::string g_error;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

void clear_error() { g_error.clear(); }

const char *last_error_cstr() { return g_error.c_str(); }

// ---------------------------------------------------------------- RNG
static uint64_t splitmix64(uint64_t &x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

Rng::Rng(uint64_t seed) {
    uint64_t x = seed;
    for (auto &w : s) w = splitmix64(x);
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

uint64_t Rng::next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
}

double Rng::uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }

uint64_t Rng::below(uint64_t bound) {
    // Lemire's multiply-shift with rejection; unbiased.
    __uint128_t m = (__uint128_t)next() * bound;
    uint64_t l = (uint64_t)m;
    if (l < bound) {
        uint64_t t = (0 - bound) % bound;
        while (l < t) {
            m = (__uint128_t)next() * bound;
            l = (uint64_t)m;
        }
    }
    return (uint64_t)(m >> 64);
}

// ---------------------------------------------------------------- CSR
int build_csr(uint32_t n, const uint32_t *labels, uint64_t m, const uint32_t *edges, asdm_host_graph &g) {
    if (2 * m >= 0xFFFFFFFFull) return fail(ASDM_ERR_INVALID, "graph has %llu edges; at most 2^31-1 supported",
                                            (unsigned long long)m);
    g.n = n;
    g.m2 = 2 * m;
    g.lab.assign(labels, labels + n);
    uint32_t maxl = 0;
    for (uint32_t v = 0; v < n; ++v) maxl = std::max(maxl, labels[v]);
    g.nlabels = n ? maxl + 1 : 0;
    g.off.assign((size_t)n + 1, 0);
    for (uint64_t i = 0; i < m; ++i) {
        uint32_t a = edges[2 * i], b = edges[2 * i + 1];
        if (a >= n || b >= n) return fail(ASDM_ERR_INVALID, "edge %llu has an endpoint out of range", (unsigned long long)i);
        if (a == b) return fail(ASDM_ERR_INVALID, "edge %llu is a self loop", (unsigned long long)i);
        g.off[a + 1]++;
        g.off[b + 1]++;
    }
    for (uint32_t v = 0; v < n; ++v) g.off[v + 1] += g.off[v];
    g.nbr.assign(g.m2, 0);
    std::vector<uint32_t> fill(g.off.begin(), g.off.end() - 1);
    for (uint64_t i = 0; i < m; ++i) {
        uint32_t a = edges[2 * i], b = edges[2 * i + 1];
        g.nbr[fill[a]++] = b;
        g.nbr[fill[b]++] = a;
    }
    const uint32_t *lab = g.lab.data();
    for (uint32_t v = 0; v < n; ++v) {
        std::sort(g.nbr.begin() + g.off[v], g.nbr.begin() + g.off[v + 1], [lab](uint32_t x, uint32_t y) {
            return lab[x] != lab[y] ? lab[x] < lab[y] : x < y;
        });
        for (uint32_t e = g.off[v] + 1; e < g.off[v + 1]; ++e)
            if (g.nbr[e] == g.nbr[e - 1]) return fail(ASDM_ERR_INVALID, "duplicate edge (%u, %u)", v, g.nbr[e]);
    }
    return ASDM_OK;
}

// Reads the whole file and tokenises it; mirrors Graph::loadGraphFromTextFile
// (relation/graph.cpp:68-148): the 'v' degree fixes the CSR offsets, 'e' edges
// are appended to both endpoints, any other token is skipped.
static int load_text(const char *path, asdm_host_graph &g) {
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(ASDM_ERR_IO, "Can not open file %s .", path);
    std::fseek(f, 0, SEEK_END);
    long sz = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    std::string text((size_t)std::max<long>(sz, 0), '\0');
    size_t got = sz > 0 ? std::fread(&text[0], 1, (size_t)sz, f) : 0;
    std::fclose(f);
    text.resize(got);
    const char *p = text.data(), *end = p + text.size();
    auto skip_ws = [&]() { while (p < end && (unsigned char)*p <= ' ') ++p; };
    auto read_u64 = [&](uint64_t &x) -> bool {
        skip_ws();
        if (p >= end || *p < '0' || *p > '9') return false;
        x = 0;
        while (p < end && *p >= '0' && *p <= '9') x = x * 10 + (uint64_t)(*p++ - '0');
        return true;
    };
    auto next_token_start = [&]() -> char {
        skip_ws();
        return p < end ? *p : '\0';
    };
    if (next_token_start() != 't') return fail(ASDM_ERR_INVALID, "%s: missing 't N M' header", path);
    ++p;
    uint64_t n = 0, m = 0;
    if (!read_u64(n) || !read_u64(m)) return fail(ASDM_ERR_INVALID, "%s: bad header", path);
    if (n >= 0xFFFFFFFFull || 2 * m >= 0xFFFFFFFFull) return fail(ASDM_ERR_INVALID, "%s: graph too large", path);
    g.n = (uint32_t)n;
    g.m2 = 2 * m;
    g.off.assign(n + 1, 0);
    g.lab.assign(n, 0);
    g.nbr.assign(g.m2, 0);
    std::vector<uint32_t> fill(n, 0);
    std::vector<uint32_t> degree(n, 0);
    uint32_t maxl = 0;
    uint64_t next_id = 0;
    while (true) {
        char c = next_token_start();
        if (c == '\0') break;
        const char *tok = p;
        while (p < end && (unsigned char)*p > ' ') ++p;
        bool single = (p - tok) == 1;
        if (single && c == 'v') {
            uint64_t id, l, d;
            if (!read_u64(id) || !read_u64(l) || !read_u64(d)) return fail(ASDM_ERR_INVALID, "%s: bad vertex line", path);
            if (id != next_id) return fail(ASDM_ERR_INVALID, "%s: vertex ids must be listed as 0..N-1 in order", path);
            ++next_id;
            g.lab[id] = (uint32_t)l;
            degree[id] = (uint32_t)d;
            g.off[id + 1] = g.off[id] + (uint32_t)d;
            maxl = std::max<uint32_t>(maxl, (uint32_t)l);
        } else if (single && c == 'e') {
            uint64_t a, b;
            if (!read_u64(a) || !read_u64(b)) return fail(ASDM_ERR_INVALID, "%s: bad edge line", path);
            if (a >= n || b >= n) return fail(ASDM_ERR_INVALID, "%s: edge endpoint out of range", path);
            if (fill[a] >= degree[a] || fill[b] >= degree[b])
                return fail(ASDM_ERR_INVALID, "%s: more edges at a vertex than its declared degree", path);
            g.nbr[g.off[a] + fill[a]++] = (uint32_t)b;
            g.nbr[g.off[b] + fill[b]++] = (uint32_t)a;
        }
    }
    if (next_id != n) return fail(ASDM_ERR_INVALID, "%s: %llu vertex lines for N = %llu", path,
                                  (unsigned long long)next_id, (unsigned long long)n);
    for (uint64_t v = 0; v < n; ++v)
        if (fill[v] != degree[v]) return fail(ASDM_ERR_INVALID, "%s: vertex %llu declares degree %u but has %u edges",
                                              path, (unsigned long long)v, degree[v], fill[v]);
    if (n && (uint64_t)g.off[n] != g.m2) return fail(ASDM_ERR_INVALID, "%s: degrees do not sum to 2M", path);
    g.nlabels = n ? maxl + 1 : 0;
    const uint32_t *lab = g.lab.data();
    for (uint32_t v = 0; v < g.n; ++v)
        std::sort(g.nbr.begin() + g.off[v], g.nbr.begin() + g.off[v + 1], [lab](uint32_t x, uint32_t y) {
            return lab[x] != lab[y] ? lab[x] < lab[y] : x < y;
        });
    return ASDM_OK;
}

int make_query(const uint32_t *q_offsets, const uint32_t *q_nbrs, const uint32_t *q_labels, uint32_t q_n,
               QueryGraph &q) {
    if (!q_offsets || !q_labels || (q_n && !q_nbrs && q_offsets[q_n] != 0))
        return fail(ASDM_ERR_INVALID, "null query array");
    if (q_n == 0 || q_n > kMaxQuery) return fail(ASDM_ERR_INVALID, "query size %u outside 1..%u", q_n, kMaxQuery);
    q.n = q_n;
    q.off.assign(q_offsets, q_offsets + q_n + 1);
    q.lab.assign(q_labels, q_labels + q_n);
    if (q.off[0] != 0) return fail(ASDM_ERR_INVALID, "query offsets must start at 0");
    for (uint32_t u = 0; u < q_n; ++u)
        if (q.off[u + 1] < q.off[u]) return fail(ASDM_ERR_INVALID, "query offsets not monotone");
    q.nbr.assign(q_nbrs, q_nbrs + q.off[q_n]);
    for (uint32_t u = 0; u < q_n; ++u) {
        if (q.deg(u) >= kMaxQuery) return fail(ASDM_ERR_INVALID, "query vertex degree too large");
        for (uint32_t e = q.off[u]; e < q.off[u + 1]; ++e) {
            uint32_t w = q.nbr[e];
            if (w >= q_n || w == u) return fail(ASDM_ERR_INVALID, "bad query edge (%u, %u)", u, w);
            if (e > q.off[u]) {
                uint32_t p = q.nbr[e - 1];
                bool sorted = q.lab[p] < q.lab[w] || (q.lab[p] == q.lab[w] && p < w);
                if (!sorted) return fail(ASDM_ERR_INVALID, "query neighbours of %u not sorted by (label, id)", u);
            }
            if (q.slot(w, u) < 0) return fail(ASDM_ERR_INVALID, "query edge (%u, %u) not symmetric", u, w);
        }
    }
    return ASDM_OK;
}

}  // namespace asdm

bool asdm_host_graph::adjacent(uint32_t a, uint32_t b) const {
    const uint32_t *lo = nbr.data() + off[a], *hi = nbr.data() + off[a + 1];
    const uint32_t lb = lab[b];
    const uint32_t *l = lab.data();
    const uint32_t *it = std::lower_bound(lo, hi, b, [l, lb](uint32_t x, uint32_t key) {
        return l[x] != lb ? l[x] < lb : x < key;
    });
    return it != hi && *it == b;
}

using namespace asdm;

extern "C" {

const char *asdm_last_error(void) { return asdm::last_error_cstr(); }

int asdm_host_graph_load(const char *path, asdm_host_graph **out) {
    clear_error();
    if (!path || !out) return fail(ASDM_ERR_INVALID, "null argument");
    auto g = std::make_unique<asdm_host_graph>();
    int rc = load_text(path, *g);
    if (rc != ASDM_OK) return rc;
    *out = g.release();
    return ASDM_OK;
}

int asdm_host_graph_from_edges(uint32_t n, const uint32_t *labels, uint64_t m, const uint32_t *edges,
                               asdm_host_graph **out) {
    clear_error();
    if (!out || (n && !labels) || (m && !edges)) return fail(ASDM_ERR_INVALID, "null argument");
    auto g = std::make_unique<asdm_host_graph>();
    int rc = build_csr(n, labels, m, edges, *g);
    if (rc != ASDM_OK) return rc;
    *out = g.release();
    return ASDM_OK;
}

int asdm_host_graph_info(const asdm_host_graph *g, uint32_t *n, uint64_t *m2, uint32_t *nlabels) {
    if (!g) return fail(ASDM_ERR_INVALID, "null graph");
    if (n) *n = g->n;
    if (m2) *m2 = g->m2;
    if (nlabels) *nlabels = g->nlabels;
    return ASDM_OK;
}

int asdm_host_graph_csr(const asdm_host_graph *g, const uint32_t **offsets, const uint32_t **nbrs,
                        const uint32_t **labels) {
    if (!g) return fail(ASDM_ERR_INVALID, "null graph");
    if (offsets) *offsets = g->off.data();
    if (nbrs) *nbrs = g->nbr.data();
    if (labels) *labels = g->lab.data();
    return ASDM_OK;
}

int asdm_host_graph_write(const asdm_host_graph *g, const char *path) {
    if (!g || !path) return fail(ASDM_ERR_INVALID, "null argument");
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(ASDM_ERR_IO, "Can not open file %s .", path);
    std::vector<char> buf;
    buf.reserve(1 << 22);
    char line[96];
    auto flush = [&]() {
        std::fwrite(buf.data(), 1, buf.size(), f);
        buf.clear();
    };
    auto put = [&](int len) {
        buf.insert(buf.end(), line, line + len);
        if (buf.size() > (1u << 22)) flush();
    };
    put(std::snprintf(line, sizeof line, "t %u %llu\n", g->n, (unsigned long long)(g->m2 / 2)));
    for (uint32_t v = 0; v < g->n; ++v) put(std::snprintf(line, sizeof line, "v %u %u %u\n", v, g->lab[v], g->deg(v)));
    for (uint32_t v = 0; v < g->n; ++v)
        for (uint32_t e = g->off[v]; e < g->off[v + 1]; ++e)
            if (v < g->nbr[e]) put(std::snprintf(line, sizeof line, "e %u %u\n", v, g->nbr[e]));
    flush();
    std::fclose(f);
    return ASDM_OK;
}

void asdm_host_graph_free(asdm_host_graph *g) { delete g; }

int asdm_gen_chung_lu(uint32_t n, uint64_t m, double gamma, uint32_t nlabels, double zipf_s, uint64_t seed,
                      asdm_host_graph **out) {
    return asdm_gen_chung_lu_capped(n, m, gamma, nlabels, zipf_s, 0.0, seed, out);
}

int asdm_gen_chung_lu_capped(uint32_t n, uint64_t m, double gamma, uint32_t nlabels, double zipf_s, double wmax,
                             uint64_t seed, asdm_host_graph **out) {
    clear_error();
    if (!out || n < 2 || m == 0 || gamma <= 1.0 || nlabels == 0)
        return fail(ASDM_ERR_INVALID, "bad Chung-Lu parameters");
    if (m > (uint64_t)n * (n - 1) / 4) return fail(ASDM_ERR_INVALID, "too many edges for %u vertices", n);
    const double alpha = 1.0 / (gamma - 1.0);
    // default: the structural cutoff w_max^2 = sum w
    const double target = wmax > 0 ? wmax : std::sqrt(2.0 * (double)m);
    auto wmax_for = [&](double i0) {
        double s = 0;
        for (uint32_t i = 0; i < n; ++i) s += std::pow(i + i0, -alpha);
        return 2.0 * (double)m * std::pow(i0, -alpha) / s;
    };
    double lo = 1e-3, hi = 1e9;
    if (wmax_for(lo) <= target) hi = lo;
    for (int it = 0; it < 100 && hi / lo > 1.0 + 1e-9; ++it) {
        double mid = std::sqrt(lo * hi);
        if (wmax_for(mid) > target) lo = mid; else hi = mid;
    }
    const double i0 = hi;
    std::vector<double> w(n);
    double sum = 0;
    for (uint32_t i = 0; i < n; ++i) sum += (w[i] = std::pow(i + i0, -alpha));
    // Vose alias table over the weights.
    std::vector<double> prob(n);
    std::vector<uint32_t> alias(n, 0);
    {
        std::vector<double> scaled(n);
        std::vector<uint32_t> small, large;
        for (uint32_t i = 0; i < n; ++i) {
            scaled[i] = w[i] * n / sum;
            (scaled[i] < 1.0 ? small : large).push_back(i);
        }
        while (!small.empty() && !large.empty()) {
            uint32_t s = small.back(); small.pop_back();
            uint32_t l = large.back(); large.pop_back();
            prob[s] = scaled[s];
            alias[s] = l;
            scaled[l] = (scaled[l] + scaled[s]) - 1.0;
            (scaled[l] < 1.0 ? small : large).push_back(l);
        }
        for (uint32_t i : large) prob[i] = 1.0;
        for (uint32_t i : small) prob[i] = 1.0;
    }
    Rng rng(seed);
    auto draw = [&]() -> uint32_t {
        uint32_t i = (uint32_t)rng.below(n);
        return rng.uniform() < prob[i] ? i : alias[i];
    };
    // Open-addressing set of undirected pairs.
    uint64_t cap = 1;
    while (cap < 2 * m + 16) cap <<= 1;
    std::vector<uint64_t> table(cap, ~0ull);
    std::vector<uint32_t> edges;
    edges.reserve(2 * m);
    uint64_t attempts = 0, max_attempts = 64 * m + 1000;
    while (edges.size() < 2 * m) {
        if (++attempts > max_attempts) return fail(ASDM_ERR_INVALID, "could not draw %llu distinct edges", (unsigned long long)m);
        uint32_t a = draw(), b = draw();
        if (a == b) continue;
        if (a > b) std::swap(a, b);
        uint64_t key = ((uint64_t)a << 32) | b;
        uint64_t h = key * 0x9E3779B97F4A7C15ull;
        uint64_t slot = (h ^ (h >> 29)) & (cap - 1);
        bool fresh = true;
        while (table[slot] != ~0ull) {
            if (table[slot] == key) { fresh = false; break; }
            slot = (slot + 1) & (cap - 1);
        }
        if (!fresh) continue;
        table[slot] = key;
        edges.push_back(a);
        edges.push_back(b);
    }
    std::vector<uint32_t>().swap(alias);
    std::vector<uint64_t>().swap(table);
    // Random vertex ids, so that id and expected degree are independent.
    std::vector<uint32_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0u);
    for (uint32_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[rng.below((uint64_t)i + 1)]);
    for (auto &x : edges) x = perm[x];
    // Zipf labels.
    std::vector<double> cdf(nlabels);
    double acc = 0;
    for (uint32_t k = 0; k < nlabels; ++k) cdf[k] = (acc += std::pow((double)k + 1.0, -zipf_s));
    std::vector<uint32_t> labels(n);
    for (uint32_t v = 0; v < n; ++v) {
        double r = rng.uniform() * acc;
        uint32_t k = (uint32_t)(std::upper_bound(cdf.begin(), cdf.end(), r) - cdf.begin());
        labels[v] = std::min(k, nlabels - 1);
    }
    auto g = std::make_unique<asdm_host_graph>();
    int rc = build_csr(n, labels.data(), m, edges.data(), *g);
    if (rc != ASDM_OK) return rc;
    *out = g.release();
    return ASDM_OK;
}

int asdm_gen_query(const asdm_host_graph *g, uint32_t size, int density, uint64_t seed, asdm_host_graph **out) {
    clear_error();
    if (!g || !out || size == 0 || size > kMaxQuery || density < 0 || density > 2)
        return fail(ASDM_ERR_INVALID, "bad query-generator parameters");
    Rng rng(seed);
    const double restart = 0.1;
    for (int attempt = 0; attempt < 20000; ++attempt) {
        uint32_t start = (uint32_t)rng.below(g->n);
        if (g->deg(start) == 0) continue;
        std::vector<uint32_t> picked{start};
        uint32_t cur = start;
        for (uint32_t step = 0; step < 200 * size && picked.size() < size; ++step) {
            if (rng.uniform() < restart) cur = start;
            uint32_t d = g->deg(cur);
            if (d == 0) break;
            cur = g->nbr[g->off[cur] + rng.below(d)];
            if (std::find(picked.begin(), picked.end(), cur) == picked.end()) picked.push_back(cur);
        }
        if (picked.size() < size) continue;
        std::vector<uint32_t> edges, labels(size);
        for (uint32_t i = 0; i < size; ++i) {
            labels[i] = g->lab[picked[i]];
            for (uint32_t j = i + 1; j < size; ++j)
                if (g->adjacent(picked[i], picked[j])) {
                    edges.push_back(i);
                    edges.push_back(j);
                }
        }
        uint64_t m = edges.size() / 2;
        bool any_too_dense = false;
        std::vector<uint32_t> degs(size, 0);
        for (uint32_t x : edges) degs[x]++;
        for (uint32_t d : degs) any_too_dense |= d >= kMaxQuery;
        if (any_too_dense) continue;
        const bool dense = 2.0 * (double)m / size >= 3.0;
        if ((density == 1 && !dense) || (density == 2 && dense)) continue;
        auto q = std::make_unique<asdm_host_graph>();
        int rc = build_csr(size, labels.data(), m, edges.data(), *q);
        if (rc != ASDM_OK) return rc;
        *out = q.release();
        return ASDM_OK;
    }
    return fail(ASDM_ERR_INVALID, "no query of size %u with the requested density found", size);
}

}  // extern "C"
