// The `.card` plan cache: reader for the reference's files, writer for the
// files prepare.out produces, and lookups for the planner.
//
// Layout (all little-endian), as written by the reference's prepare.out
// (executable/prepare.cpp:62-71):
//   for each non-virtual bag, SubsetStructure::saveToSteam
//   (plan/subset_structure.cpp:455-560):
//     u64 |elements|, u32 elements[]; u32 n; u64 |cc|, u64 cc[];
//     subsets      : u64 k, k x (u64 m, u64[m])
//     subsetOf     : u64 k, k x (u64 j, j x (u64 m, i32[m]))
//     supersetOf   : same as subsetOf
//     orders       : u64 k, k x (u64 j, j x (u64 m, u32[m]))
//     subsetToCost : u64 k, k x (u64 m, i64[m])      (cost x 100)
//     remainingOrders / remainingCost: as orders / subsetToCost
//   then saveSubsetToCard (plan/estimator.cpp:981-992):
//     u64 count, count x (u64 subset bitmask, f64 cardinality)
//   then i32 planning time x 10^4.
// The number of bag records is not stored; the reader takes the first k for
// which the rest of the file is exactly the cardinality map and the time.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <memory>
#include <unordered_map>

#include "internal.h"

struct asdm_card {
    uint32_t bags = 0;
    std::unordered_map<uint64_t, double> card;   // subset bitmask (1 << query vertex) -> cardinality
    std::vector<std::pair<uint64_t, double>> ordered;  // file order, for writing back
    double plan_seconds = 0.0;
};

namespace asdm {
namespace {

struct Reader {
    const uint8_t *p, *end;
    bool ok = true;
    bool take(void *dst, size_t n) {
        if (!ok || (size_t)(end - p) < n) return ok = false;
        if (dst) std::memcpy(dst, p, n);
        p += n;
        return true;
    }
    uint64_t u64() {
        uint64_t x = 0;
        take(&x, 8);
        return x;
    }
    // u64 count then count x elem bytes
    void vec(size_t elem) {
        const uint64_t m = u64();
        if (!ok || m > (uint64_t)(end - p) / (elem ? elem : 1)) { ok = false; return; }
        take(nullptr, m * elem);
    }
    void vec2(size_t elem) {
        const uint64_t k = u64();
        for (uint64_t i = 0; ok && i < k; ++i) vec(elem);
    }
    void vec3(size_t elem) {
        const uint64_t k = u64();
        for (uint64_t i = 0; ok && i < k; ++i) vec2(elem);
    }
};

bool skip_bag(Reader &r) {
    r.vec(4);              // elements
    r.take(nullptr, 4);    // n
    r.vec(8);              // cc
    r.vec2(8);             // subsets
    r.vec3(4);             // subsetOf
    r.vec3(4);             // supersetOf
    r.vec3(4);             // orders
    r.vec2(8);             // subsetToCost
    r.vec3(4);             // remainingOrders
    r.vec2(8);             // remainingCost
    return r.ok;
}

}  // namespace
}  // namespace asdm

using namespace asdm;

extern "C" int asdm_card_load(const char *path, asdm_card **out) {
    clear_error();
    if (!path || !out) return fail(ASDM_ERR_INVALID, "null argument");
    std::ifstream in(path, std::ios::binary);
    if (!in.is_open()) return fail(ASDM_ERR_IO, "Can not open file %s .", path);
    std::vector<uint8_t> buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    const uint8_t *begin = buf.data(), *end = buf.data() + buf.size();
    for (uint32_t k = 0; k <= 64; ++k) {
        Reader r{begin, end};
        bool ok = true;
        for (uint32_t b = 0; b < k && ok; ++b) ok = skip_bag(r);
        if (!ok) break;  // fewer than k records fit: no later k can either
        Reader m = r;
        const uint64_t cnt = m.u64();
        if (!m.ok || (uint64_t)(end - m.p) != cnt * 16 + 4) continue;
        auto c = std::make_unique<asdm_card>();
        c->bags = k;
        for (uint64_t i = 0; i < cnt; ++i) {
            uint64_t key;
            double v;
            m.take(&key, 8);
            m.take(&v, 8);
            c->card[key] = v;
            c->ordered.emplace_back(key, v);
        }
        int32_t t = 0;
        m.take(&t, 4);
        c->plan_seconds = t / 10000.0;
        *out = c.release();
        return ASDM_OK;
    }
    return fail(ASDM_ERR_INVALID, "%s: not a .card file", path);
}

extern "C" int asdm_card_create(asdm_card **out) {
    if (!out) return fail(ASDM_ERR_INVALID, "null argument");
    *out = new asdm_card();
    return ASDM_OK;
}

extern "C" int asdm_card_set(asdm_card *c, uint64_t subset, double card) {
    if (!c) return fail(ASDM_ERR_INVALID, "null argument");
    if (c->card.find(subset) == c->card.end()) c->ordered.emplace_back(subset, card);
    else
        for (auto &kv : c->ordered)
            if (kv.first == subset) kv.second = card;
    c->card[subset] = card;
    return ASDM_OK;
}

extern "C" int asdm_card_info(const asdm_card *c, uint32_t *bags, uint64_t *entries, double *plan_seconds) {
    if (!c) return fail(ASDM_ERR_INVALID, "null argument");
    if (bags) *bags = c->bags;
    if (entries) *entries = c->card.size();
    if (plan_seconds) *plan_seconds = c->plan_seconds;
    return ASDM_OK;
}

extern "C" int asdm_card_lookup(const asdm_card *c, uint64_t subset, double *card) {
    if (!c || !card) return fail(ASDM_ERR_INVALID, "null argument");
    auto it = c->card.find(subset);
    if (it == c->card.end()) return fail(ASDM_ERR_INVALID, "subset %llx not in the card", (unsigned long long)subset);
    *card = it->second;
    return ASDM_OK;
}

// Writes a file with no bag records: the cardinality map (values truncated to
// two decimals, as saveSubsetToCard does) and the planning time.
extern "C" int asdm_card_write(const asdm_card *c, const char *path, double plan_seconds) {
    if (!c || !path) return fail(ASDM_ERR_INVALID, "null argument");
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(ASDM_ERR_IO, "Can not open file %s .", path);
    uint64_t cnt = c->ordered.size();
    std::fwrite(&cnt, 8, 1, f);
    for (auto &kv : c->ordered) {
        const double scaled = static_cast<double>(static_cast<int64_t>(kv.second * 100.0)) / 100.0;
        std::fwrite(&kv.first, 8, 1, f);
        std::fwrite(&scaled, 8, 1, f);
    }
    const int32_t t = static_cast<int32_t>(plan_seconds * 10000);
    std::fwrite(&t, 4, 1, f);
    std::fclose(f);
    return ASDM_OK;
}

extern "C" void asdm_card_free(asdm_card *c) { delete c; }

// lookups for the planner
double card_lookup_or(const asdm_card *c, uint64_t subset, double fallback) {
    if (!c) return fallback;
    auto it = c->card.find(subset);
    return it == c->card.end() ? fallback : it->second;
}
