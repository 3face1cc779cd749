// K4-K8: exact enumeration over the candidate space.
//
// One warp runs an iterative depth-first search over the matching order
// (the attribute-at-a-time leapfrog join the reference executes in
// adaptiveShareJoin/adaptiveGlobalJoin, matching/adaptive.cpp:115-330,
// 1179-2279, and attributeOpen, :901-1000).  The candidates of level k are the
// intersection of the candidate-edge lists of its earlier query neighbours
// (ComputeSetIntersection::LeapfrogJoin, utility/compute_set_intersection.cpp:193-233),
// computed lazily 32 elements at a time: the shortest list drives, each lane
// takes one driver element and gallops in every other list from a shared
// cursor (the leapfrog seek, :177-191), and __ballot_sync/__popc compact the
// survivors into the level's stack slot.  Injectivity (the reference's
// visited[] array) only has to be checked against earlier levels that carry
// the same label and are not adjacent to level k; adjacent levels can never
// hold the same vertex.  The last level is counted, not descended: its count
// is |intersection| minus the same-label earlier vertices that lie in it,
// which is exactly what traverse()'s numTuples(visited) shortcut computes for
// ALL_LEVEL builds (matching/join.cpp:852-877).  LOCAL mode walks the last
// level element by element to add one to local[v][u_last] per match and adds
// the completion count to every prefix vertex (produceResult's
// ++gLocalCount[φ(u)][u], matching/join.cpp:1035-1041); EMBED mode also
// writes each match as a row indexed by query vertex (COLLECT_RESULT,
// :1032-1034).  Root tasks are the candidates of the first level, claimed
// with one atomicAdd each; hubs are split across warps by work donation.
#include <algorithm>
#include <cstring>
#include <memory>
#include <mutex>
#include <numeric>

#include "cs.cuh"

namespace asdm {

int build_plan(const asdm_cs &cs, const uint32_t *user_order, asdm_plan &p, const asdm_card *card = nullptr);
bool tree_countable(const QueryGraph &q);
bool tree_countable_conflicts(const QueryGraph &q);
int tree_counts(asdm_graph *G, const std::vector<asdm_cs *> &cs, std::vector<uint64_t> &counts,
                std::vector<char> &done, const std::vector<unsigned long long *> *local = nullptr);
int overflow_bounds(asdm_graph *G, const std::vector<asdm_cs *> &cs, std::vector<char> &proven,
                    std::vector<uint64_t> *lower = nullptr);

namespace {

constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr uint32_t kFull = 0xffffffffu;

enum : uint32_t { kFlagOverflow = 1, kFlagTimeout = 2, kFlagCapacity = 4, kFlagLimit = 16 };
constexpr uint32_t kStopFlags = kFlagOverflow | kFlagTimeout | kFlagLimit;
enum : int {
    kCtrTask = 0, kCtrCount = 1, kCtrFlags = 2, kCtrRows = 3, kCtrInter = 4, kCtrElems = 5,
    kCtrHead = 6, kCtrTail = 7, kCtrActive = 8, kCtrIdle = 9, kCtrDonated = 10, kCtrTailLane = 11,
    kCtrTailWarp = 12, kCtrIdleNs = 13, kCtrN = 16
};
// Work-donation ring (a bounded multi-producer multi-consumer queue with a
// sequence number per slot): a record is [query, level s, lo, hi, idx[0..s-1]].
constexpr uint32_t kRecWords = 4 + 32;
constexpr uint64_t kQueueCap = 1u << 16;      // power of two
// An idle warp polls the ring until no warp is working, a stop flag is set or
// the run's deadline passes; without a deadline it leaves after kIdleMaxNs
// (the working warps then finish their own ranges, so no work is lost).
constexpr uint64_t kIdleMaxNs = 3600ull * 1000000000ull;
constexpr uint32_t kIdleSleepMaxNs = 2048;   // poll back-off ceiling

struct DLevel {
    const uint32_t *cand;  // C(u)
    uint32_t ncand;
    uint32_t u;            // query vertex of this level
    uint32_t nback;        // earlier adjacent levels
    uint32_t back_first;   // first slot in the DBack array
    uint32_t nconf;        // earlier same-label non-adjacent levels
    uint32_t conf_first;
};
static_assert(sizeof(DLevel) == 32, "DLevel layout");

struct DBack {
    const uint32_t *off;   // candidate-edge offsets of (u_j -> u_k), indexed by idx[j]
    const uint32_t *list;  // candidate-edge entries (indices into C(u_k))
    uint32_t level;        // j
    uint32_t pad;
};
static_assert(sizeof(DBack) == 24, "DBack layout");

struct EnumArgs {
    const DLevel *lv;
    const DBack *bk;
    const uint32_t *conf;
    uint32_t n, nb, nc, nq;
    unsigned long long ntasks;  // root blocks
    unsigned long long pairs;   // (level-0, level-1) candidate pairs (level-0 candidates when n == 1)
    unsigned long long blk;     // pairs per root block
    unsigned long long *ctr;
    unsigned long long *local;  // |Vg| x nq, MODE_LOCAL
    uint32_t *rows;             // row_cap x nq, MODE_EMBED
    uint64_t row_cap;
    uint64_t limit_ns;          // 0 = none; else per-warp wall-clock budget
    unsigned long long count_limit;  // 0 = none
    uint32_t lane_leaf_max;     // longest shortest-list a lane evaluates alone at the last level
    uint32_t merge_ratio;       // a list probe merges (instead of galloping) up to this length ratio
    uint32_t *queue;            // kQueueCap records of kRecWords words
    unsigned long long *qseq;   // kQueueCap slot sequence numbers
    // batches of queries (enum_batch_kernel): one QDesc per query, root tasks
    // of query q are task_pre[q] .. task_pre[q+1]
    const struct QDesc *qd;
    const unsigned long long *task_pre;
    uint32_t nquery, maxn, maxnb;
    unsigned long long *qcounts;
    unsigned int *qflags;
    // per-query time budget (batches): warp-nanoseconds a query may use,
    // summed over warps (0 = none), and what each query has used
    unsigned long long q_budget_ns;
    unsigned long long *qwork;
    // closed form of the last two levels (single-query kernel; QDesc for batches)
    const unsigned long long *ps;
    const uint32_t *rev_off, *rev_list;
    uint32_t tail;
    unsigned long long *qcycles;  // batches, optional: SM cycles warps spent on each query
    const uint32_t *xmap_a, *xmap_z;
    unsigned long long *lw;       // LOCAL mode: leaf weights (see Warp::lw)
};

struct QDesc {
    const DLevel *lv;
    const DBack *bk;
    const uint32_t *conf;
    unsigned long long *local;  // |Vg| x n (MODE_LOCAL batches)
    unsigned long long pairs, blk;
    uint32_t n, nb, nc, tail;
    const unsigned long long *ps;
    const uint32_t *rev_off, *rev_list;
    // lane tails at level d = n-3: index in C(u_{n-2}) / C(u_{n-1}) of each
    // candidate of level d, where level d is a conflict of that level (or null)
    const uint32_t *xmap_a, *xmap_z;
    unsigned long long *lw;  // LOCAL mode: leaf weights (or null)
};

// The last two levels of a COUNT-mode plan are counted in closed form when
// each has exactly one backward edge (always so for tree-shaped queries):
// kTailChain when the last level's edge comes from level n-2 (needs prefix
// sums of the last level's list lengths along level n-2's driver edge, and
// the reverse candidate edges last level -> level n-2), kTailLeaf when it
// comes from an earlier level (the last level's list is then fixed by the
// prefix).
// kTailIsect: level n-2 has two backward edges (a cycle closed there) and
// the last level one; only the lane-parallel form at level n-3 handles it.
enum : uint32_t { kTailNone = 0, kTailChain = 1, kTailLeaf = 2, kTailIsect = 3 };

__host__ __device__ constexpr uint32_t warp_words(uint32_t n, uint32_t nb) { return 39 * n + 3 * nb + 96; }

// The last level is evaluated one survivor per lane (instead of one warp per
// survivor) when it has at most this many earlier neighbours and its shortest
// list is at most kLaneLeafMax long.
constexpr uint32_t kLaneLeafLists = 4;
constexpr uint32_t kSelf = 0xFFFFFFFEu;
constexpr uint32_t kSelfD = 0xFFFFFFFDu;   // the conflict is the lane's own level-d vertex
// Lane-parallel closed form at level n-3: at most this many conflict levels
// per tail level, and this many list entries of intersection work per lane.
constexpr uint32_t kLaneTailConf = 4;
constexpr uint32_t kLaneTailWork = 64;

__host__ __device__ inline uint32_t plan_words(uint32_t n, uint32_t nb, uint32_t nc) {
    return (uint32_t)((n * sizeof(DLevel) + nb * sizeof(DBack)) / 4) + ((nc + 3) & ~3u);
}

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Largest i in [0, n) with off[i] <= t, given off[0] <= t < off[n]:
// 32-way search, every lane probes one point per round.
__device__ __forceinline__ uint32_t warp_find_row32(const uint32_t *__restrict__ off, uint32_t n, unsigned long long t,
                                                    uint32_t lane) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 32) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t p = lo + lane * step;
        const uint32_t m = __ballot_sync(kFull, p < hi && off[p] <= t);
        const uint32_t nlo = lo + (31 - __clz(m)) * step;
        hi = min(hi, nlo + step);
        lo = nlo;
    }
    const uint32_t p = lo + lane;
    const uint32_t m = __ballot_sync(kFull, p < hi && off[p] <= t);
    return lo + (31 - __clz(m));
}

// Largest i in [0, n) with pre[i] <= t (64-bit prefix array).
__device__ __forceinline__ uint32_t warp_find_row64(const unsigned long long *__restrict__ pre, uint32_t n,
                                                    unsigned long long t, uint32_t lane) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 32) {
        const uint32_t step = (hi - lo + 31) / 32;
        const uint32_t p = lo + lane * step;
        const uint32_t m = __ballot_sync(kFull, p < hi && pre[p] <= t);
        const uint32_t nlo = lo + (31 - __clz(m)) * step;
        hi = min(hi, nlo + step);
        lo = nlo;
    }
    const uint32_t p = lo + lane;
    const uint32_t m = __ballot_sync(kFull, p < hi && pre[p] <= t);
    return lo + (31 - __clz(m));
}

template <uint32_t MODE, bool MULTI = false>
struct Warp {
    const EnumArgs &a;
    const DLevel *L;
    const DBack *B;
    const uint32_t *CF;
    uint32_t *idx, *vid, *buf, *cnt, *pos, *dpos, *dend, *drv, *sstart, *slen, *scur, *fidx, *fta, *ftz;
    uint32_t lane;
    uint32_t n;            // levels of the current query
    uint32_t q = 0;        // current query (batches)
    unsigned long long *local;  // |Vg| x n local counts of the current query (MODE_LOCAL)
    unsigned long long count = 0, inter = 0, elems = 0, tails_lane = 0, tails_warp = 0;
    bool overflow = false;
    uint64_t t_mark = 0;   // lane 0: when this warp's time was last charged to its query
    const unsigned long long *ps;        // kTailChain: prefix sums over the driver edge of level n-2
    const uint32_t *rev_off, *rev_list;  // kTailChain: candidate edges last level -> level n-2
    uint32_t tail;                       // kTail* of the current query
    const uint32_t *xmap_a, *xmap_z;     // cross indices for lane tails (or null)
    // LOCAL mode with a one-list last level: per candidate of the list's
    // source level, how many prefixes counted that candidate's whole list;
    // a pass after the kernel adds them to the last level's local counts
    unsigned long long *lw;

    // w: this warp's shared-memory words, laid out for queries of up to maxn
    // levels and maxnb backward edges.
    __device__ Warp(const EnumArgs &args, const DLevel *l, const DBack *b, const uint32_t *cf, uint32_t *w, uint32_t ln,
                    uint32_t levels, uint32_t maxn, uint32_t maxnb)
        : a(args), L(l), B(b), CF(cf), lane(ln), n(levels), local(args.local), ps(args.ps), rev_off(args.rev_off),
          rev_list(args.rev_list), tail(args.tail), xmap_a(args.xmap_a), xmap_z(args.xmap_z), lw(args.lw) {
        idx = w;
        vid = idx + maxn;
        buf = vid + maxn;
        cnt = buf + 32 * maxn;
        pos = cnt + maxn;
        dpos = pos + maxn;
        dend = dpos + maxn;
        drv = dend + maxn;
        sstart = drv + maxn;
        slen = sstart + maxnb;
        scur = slen + maxnb;
        fidx = scur + maxnb;
        fta = fidx + 32;
        ftz = fta + 32;
    }

    // Charges this warp's time since the last mark to its query's budget
    // (lane 0; batches with a per-query time budget).
    __device__ __forceinline__ void charge() {
        if (MULTI && a.q_budget_ns && lane == 0) {
            const uint64_t now = globaltimer();
            const unsigned long long dt = now - t_mark;
            t_mark = now;
            const unsigned long long used = atomicAdd(&a.qwork[q], dt) + dt;
            if (used > a.q_budget_ns) atomicOr(&a.qflags[q], kFlagTimeout);
        }
    }

    // Starts charging time to the current query (lane 0).
    __device__ __forceinline__ void mark() {
        if (MULTI && a.q_budget_ns && lane == 0) t_mark = globaltimer();
    }

    // Batches: whether the current query was stopped (count limit reached or
    // time budget used up); its remaining work is abandoned.
    __device__ __forceinline__ bool query_stopped() {
        if (!MULTI || !(a.count_limit || a.q_budget_ns)) return false;
        charge();
        uint32_t st = 0;
        if (lane == 0) st = *(volatile unsigned int *)&a.qflags[q] & (kFlagLimit | kFlagTimeout);
        return __shfl_sync(kFull, st, 0) != 0;
    }

    // Switches to query qq of a batch (its plan is read from global memory).
    __device__ void bind(uint32_t qq) {
        if (qq == q) return;
        flush_count();
        q = qq;
        const QDesc d = a.qd[qq];
        L = d.lv;
        B = d.bk;
        CF = d.conf;
        n = d.n;
        local = d.local;
        ps = d.ps;
        rev_off = d.rev_off;
        rev_list = d.rev_list;
        tail = d.tail;
        xmap_a = d.xmap_a;
        xmap_z = d.xmap_z;
        lw = d.lw;
    }

    __device__ __forceinline__ bool closed_at(uint32_t d) const {
        return MODE == ASDM_MODE_COUNT && (tail == kTailChain || tail == kTailLeaf) && d + 2 == n;
    }

    // |a ∩ b| of two ascending lists, warp-wide: each lane looks up entries
    // of the shorter list in the longer one.
    __device__ uint32_t isect_count(const uint32_t *x, uint32_t nx, const uint32_t *y, uint32_t ny) const {
        const bool xs = nx <= ny;
        const uint32_t *sl = xs ? x : y, *tl = xs ? y : x;
        const uint32_t ns = xs ? nx : ny, nt = xs ? ny : nx;
        uint32_t hits = 0;
        for (uint32_t i = lane; i < ns; i += 32) {
            const uint32_t v = sl[i];
            const uint32_t q = lower_bound_u32(tl, nt, v);
            hits += q < nt && tl[q] == v;
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) hits += __shfl_xor_sync(kFull, hits, o);
        return hits;
    }

    // The same for lists of candidate indices into two candidate sets of one
    // label, compared by vertex id (cx[x[i]] against cy[y[j]]; both ascend).
    __device__ uint32_t isect_count_vid(const uint32_t *x, uint32_t nx, const uint32_t *cx, const uint32_t *y,
                                        uint32_t ny, const uint32_t *cy) const {
        const bool xs = nx <= ny;
        const uint32_t *sl = xs ? x : y, *tl = xs ? y : x, *cs = xs ? cx : cy, *ct = xs ? cy : cx;
        const uint32_t ns = xs ? nx : ny, nt = xs ? ny : nx;
        uint32_t hits = 0;
        for (uint32_t i = lane; i < ns; i += 32) {
            const uint32_t v = cs[sl[i]];
            uint32_t lo = 0, hi = nt;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (ct[tl[mid]] < v) lo = mid + 1; else hi = mid;
            }
            hits += lo < nt && ct[tl[lo]] == v;
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) hits += __shfl_xor_sync(kFull, hits, o);
        return hits;
    }

    __device__ __forceinline__ bool lane_tail_ok(uint32_t d) const {
        return MODE == ASDM_MODE_COUNT && tail != kTailNone && d + 3 == n && L[d + 1].nconf <= kLaneTailConf &&
               L[d + 2].nconf <= kLaneTailConf;
    }

    // For a node at level d-1 whose level-d entries get lane-parallel tails:
    // the indices of the prefix's conflict vertices in C(u_{d+1}) (fta) and in
    // C(u_{d+2}) (ftz); kSelfD where the conflict level is d itself, kSelf
    // where it is level d+1 (the last level's conflict with level n-2).
    __device__ void prepare_lane_tail(uint32_t d) {
        const DLevel La = L[d + 1], Lz = L[d + 2];
        if (lane < La.nconf) {
            const uint32_t c = CF[La.conf_first + lane];
            uint32_t y = kSelfD;
            if (c < d) {
                const uint32_t v = vid[c];
                y = lower_bound_u32(La.cand, La.ncand, v);
                if (y >= La.ncand || La.cand[y] != v) y = kNone;
            }
            fta[lane] = y;
        }
        if (lane < Lz.nconf) {
            const uint32_t c = CF[Lz.conf_first + lane];
            uint32_t y = c == d + 1 ? kSelf : kSelfD;
            if (c < d) {
                const uint32_t v = vid[c];
                y = lower_bound_u32(Lz.cand, Lz.ncand, v);
                if (y >= Lz.ncand || Lz.cand[y] != v) y = kNone;
            }
            ftz[lane] = y;
        }
        __syncwarp();
    }

    // |x ∩ y| of two ascending lists by one lane: the shorter list's entries
    // looked up in the longer one.
    __device__ __forceinline__ static uint32_t lane_isect(const uint32_t *x, uint32_t nx, const uint32_t *y, uint32_t ny) {
        if (nx > ny) {
            const uint32_t *t = x; x = y; y = t;
            const uint32_t tn = nx; nx = ny; ny = tn;
        }
        uint32_t hits = 0, cur = 0;
        for (uint32_t i = 0; i < nx && cur < ny; ++i) {
            cur = gallop_lb(y, cur, ny, x[i]);
            hits += cur < ny && y[cur] == x[i];
        }
        return hits;
    }

    // The same by vertex id for candidate-index lists of two candidate sets of one label.
    __device__ __forceinline__ static uint32_t lane_isect_vid(const uint32_t *x, uint32_t nx, const uint32_t *cx,
                                                              const uint32_t *y, uint32_t ny, const uint32_t *cy) {
        uint32_t hits = 0, i = 0, j = 0;
        while (i < nx && j < ny) {
            const uint32_t a = cx[x[i]], b = cy[y[j]];
            hits += a == b;
            i += a <= b;
            j += b <= a;
        }
        return hits;
    }

    // kTailIsect for one level-d entry x (d = n-3), by this lane alone: D = the intersection of level d+1's
    // two lists, then per survivor y the last level: |list(y)| minus the
    // conflict vertices in it (the last level's edge from level d+1), or the
    // fixed list's length minus its conflict vertices and y's own vertex
    // (edge from an earlier level).  Entries of D that are level-(d+1)
    // conflicts are skipped.
    __device__ __forceinline__ bool lane_tail_isect(uint32_t d, uint32_t x, const uint32_t *ya, const uint32_t *yz, bool self,
                                    unsigned long long &out, unsigned long long &touched) {
        const uint32_t a = d + 1;
        const DLevel La = L[a], Lz = L[a + 1];
        const DBack b1 = B[La.back_first], b2 = B[La.back_first + 1], bz = B[Lz.back_first];
        const uint32_t i1 = b1.level == d ? x : idx[b1.level], i2 = b2.level == d ? x : idx[b2.level];
        const uint32_t *l1 = b1.list + b1.off[i1], *l2 = b2.list + b2.off[i2];
        uint32_t n1 = b1.off[i1 + 1] - b1.off[i1], n2 = b2.off[i2 + 1] - b2.off[i2];
        if (n1 > n2) {
            const uint32_t *t = l1; l1 = l2; l2 = t;
            const uint32_t tn = n1; n1 = n2; n2 = tn;
        }
        if (n1 > kLaneTailWork) return false;
        const bool chain = bz.level == a;
        const uint32_t *LL = nullptr;
        uint32_t nl = 0, m = 0;
        if (!chain) {
            const uint32_t ijz = bz.level == d ? x : idx[bz.level];
            LL = bz.list + bz.off[ijz];
            nl = bz.off[ijz + 1] - bz.off[ijz];
#pragma unroll
            for (uint32_t k = 0; k < kLaneTailConf; ++k) {
                if (yz[k] == kNone) continue;
                const uint32_t q = lower_bound_u32(LL, nl, yz[k]);
                m += q < nl && LL[q] == yz[k];
            }
        }
        unsigned long long sum = 0;
        uint32_t cur = 0;
        for (uint32_t i = 0; i < n1 && cur < n2; ++i) {
            const uint32_t y = l1[i];
            cur = gallop_lb(l2, cur, n2, y);
            if (cur >= n2 || l2[cur] != y) continue;
            bool excl = false;
#pragma unroll
            for (uint32_t k = 0; k < kLaneTailConf; ++k) excl |= ya[k] == y;
            if (excl) continue;
            if (chain) {
                const uint32_t a0 = bz.off[y], a1 = bz.off[y + 1];
                unsigned long long c = a1 - a0;
#pragma unroll
                for (uint32_t k = 0; k < kLaneTailConf; ++k) {
                    if (yz[k] == kNone) continue;
                    const uint32_t q = lower_bound_u32(bz.list + a0, a1 - a0, yz[k]);
                    c -= (q < a1 - a0 && bz.list[a0 + q] == yz[k]) ? 1ull : 0ull;
                }
                sum += c;
            } else {
                unsigned long long c = nl - m;
                if (self) {
                    // y's own vertex in the fixed list
                    const uint32_t v = La.cand[y];
                    uint32_t l2i = 0, h2 = nl;
                    while (l2i < h2) {
                        const uint32_t mid = (l2i + h2) >> 1;
                        if (Lz.cand[LL[mid]] < v) l2i = mid + 1; else h2 = mid;
                    }
                    c -= (l2i < nl && Lz.cand[LL[l2i]] == v) ? 1ull : 0ull;
                }
                sum += c;
            }
        }
        touched += n1 + 4;
        out = sum;
        return true;
    }

    // The closed form of the last two levels for one level-d entry x (d =
    // n-3), by this lane alone; false (x left to the warp-wide path) when an
    // intersection would be long.  Same arithmetic as tail2 with the whole
    // driver list of level d+1.
    __device__ bool lane_tail(uint32_t d, uint32_t x, unsigned long long &out, unsigned long long &touched) {
        const uint32_t a = d + 1;
        const DLevel La = L[a], Lz = L[a + 1];
        const DBack ba = B[La.back_first], bz = B[Lz.back_first];
        const uint32_t ija = ba.level == d ? x : idx[ba.level];
        const uint32_t s0 = ba.off[ija], nd = ba.off[ija + 1] - s0;
        const uint32_t *D = ba.list + s0;
        const uint32_t vx = L[d].cand[x];
        // conflict indices, resolving the ones that are x's own vertex
        uint32_t ya[kLaneTailConf], yz[kLaneTailConf];
        bool self = false;
#pragma unroll
        for (uint32_t k = 0; k < kLaneTailConf; ++k) {
            ya[k] = kNone;
            yz[k] = kNone;
            if (k < La.nconf) {
                uint32_t y = fta[k];
                if (y == kSelfD) {
                    if (xmap_a) {
                        y = xmap_a[x];
                    } else {
                        y = lower_bound_u32(La.cand, La.ncand, vx);
                        if (y >= La.ncand || La.cand[y] != vx) y = kNone;
                    }
                }
                ya[k] = y;
            }
            if (k < Lz.nconf) {
                uint32_t y = ftz[k];
                if (y == kSelfD) {
                    if (xmap_z) {
                        y = xmap_z[x];
                    } else {
                        y = lower_bound_u32(Lz.cand, Lz.ncand, vx);
                        if (y >= Lz.ncand || Lz.cand[y] != vx) y = kNone;
                    }
                } else if (y == kSelf) {
                    self = true;
                    y = kNone;
                }
                yz[k] = y;
            }
        }
        if (tail == kTailIsect) return lane_tail_isect(d, x, ya, yz, self, out, touched);
        // entries of D that are level-(d+1) conflicts
        uint32_t xe[kLaneTailConf];
        uint32_t nexcl = 0;
#pragma unroll
        for (uint32_t k = 0; k < kLaneTailConf; ++k) {
            xe[k] = kNone;
            if (ya[k] != kNone) {
                const uint32_t p = lower_bound_u32(D, nd, ya[k]);
                if (p < nd && D[p] == ya[k]) { xe[k] = ya[k]; ++nexcl; }
            }
        }
        unsigned long long sum;
        uint32_t work = 0;
        touched += 4;
        if (tail == kTailChain) {
            sum = ps[s0 + nd] - ps[s0];
#pragma unroll
            for (uint32_t k = 0; k < kLaneTailConf; ++k) {
                if (yz[k] == kNone) continue;
                const uint32_t r0 = rev_off[yz[k]], nr = rev_off[yz[k] + 1] - r0;
                work += min(nd, nr);
                if (work > kLaneTailWork) return false;
                sum -= lane_isect(D, nd, rev_list + r0, nr);
            }
#pragma unroll
            for (uint32_t k = 0; k < kLaneTailConf; ++k) {
                if (xe[k] == kNone) continue;
                const uint32_t a0 = bz.off[xe[k]], a1 = bz.off[xe[k] + 1];
                unsigned long long c = a1 - a0;
#pragma unroll
                for (uint32_t j = 0; j < kLaneTailConf; ++j) {
                    if (yz[j] == kNone) continue;
                    const uint32_t q = lower_bound_u32(bz.list + a0, a1 - a0, yz[j]);
                    c -= (q < a1 - a0 && bz.list[a0 + q] == yz[j]) ? 1ull : 0ull;
                }
                sum -= c;
            }
        } else {
            const uint32_t ijz = bz.level == d ? x : idx[bz.level];
            const uint32_t a0 = bz.off[ijz], nl = bz.off[ijz + 1] - a0;
            const uint32_t *LL = bz.list + a0;
            uint32_t m = 0;
#pragma unroll
            for (uint32_t k = 0; k < kLaneTailConf; ++k) {
                if (yz[k] == kNone) continue;
                const uint32_t q = lower_bound_u32(LL, nl, yz[k]);
                m += q < nl && LL[q] == yz[k];
            }
            sum = (unsigned long long)(nd - nexcl) * (unsigned long long)(nl - m);
            if (self) {
                work += nd + nl;
                if (work > kLaneTailWork) return false;
                uint32_t hits = lane_isect_vid(D, nd, La.cand, LL, nl, Lz.cand);
#pragma unroll
                for (uint32_t k = 0; k < kLaneTailConf; ++k) {
                    if (xe[k] == kNone) continue;
                    const uint32_t v = La.cand[xe[k]];
                    uint32_t l2 = 0, h2 = nl;
                    while (l2 < h2) {
                        const uint32_t mid = (l2 + h2) >> 1;
                        if (Lz.cand[LL[mid]] < v) l2 = mid + 1; else h2 = mid;
                    }
                    hits -= (l2 < nl && Lz.cand[LL[l2]] == v) ? 1u : 0u;
                }
                sum -= hits;
            }
        }
        touched += work;
        out = sum;
        return true;
    }

    // The last two levels in closed form for driver positions [lo, hi) of
    // level d = n-2 (prefix fixed down to level d-1; last-level conflict
    // indices prepared in fidx).  Entries x of the driver range D that are
    // conflicts at level d are taken out with their whole contribution.
    //   kTailChain: sum over x in D of |list(x)| (prefix sums), minus, per
    //     last-level conflict vertex y, the x in D adjacent to y (D intersected
    //     with y's reverse candidate-edge list);
    //   kTailLeaf: the last level's list LL is fixed: |D'| x (|LL| minus the
    //     conflict vertices in LL), minus the x whose own vertex is in LL when
    //     level d is itself a conflict of the last level.
    __device__ void tail2(uint32_t d, uint32_t lo, uint32_t hi) {
        ++tails_warp;
        const DLevel lv = L[d];
        const uint32_t dslot = lv.back_first;
        const uint32_t s0 = sstart[dslot];
        const uint32_t *D = B[dslot].list + s0 + lo;
        const uint32_t nd = hi - lo;
        const DLevel lvL = L[n - 1];
        const DBack bL = B[lvL.back_first];
        // this lane's level-d conflict vertex, when it is an entry of D
        uint32_t xc = kNone;
        if (lane < lv.nconf) {
            const uint32_t v = vid[CF[lv.conf_first + lane]];
            const uint32_t y = lower_bound_u32(lv.cand, lv.ncand, v);
            if (y < lv.ncand && lv.cand[y] == v) {
                const uint32_t p = lower_bound_u32(D, nd, y);
                if (p < nd && D[p] == y) xc = y;
            }
        }
        unsigned long long sum = 0, touched = 2;
        if (tail == kTailChain) {
            sum = ps[s0 + hi] - ps[s0 + lo];
            touched += 2;
            for (uint32_t k = 0; k < lvL.nconf; ++k) {
                const uint32_t y = fidx[k];
                if (y >= kSelf) continue;  // not a candidate there (level d is adjacent, never itself)
                const uint32_t r0 = rev_off[y], r1 = rev_off[y + 1];
                sum -= isect_count(D, nd, rev_list + r0, r1 - r0);
                touched += 2 + min(nd, r1 - r0);
            }
            unsigned long long back = 0;
            if (xc != kNone) {
                const uint32_t a0 = bL.off[xc], a1 = bL.off[xc + 1];
                back = a1 - a0;
                for (uint32_t k = 0; k < lvL.nconf; ++k) {
                    const uint32_t y = fidx[k];
                    if (y >= kSelf) continue;
                    const uint32_t q = lower_bound_u32(bL.list + a0, a1 - a0, y);
                    back -= (q < a1 - a0 && bL.list[a0 + q] == y) ? 1ull : 0ull;
                }
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) back += __shfl_xor_sync(kFull, back, o);
            sum -= back;
        } else {
            const uint32_t ij = idx[bL.level];
            const uint32_t a0 = bL.off[ij], a1 = bL.off[ij + 1];
            const uint32_t *LL = bL.list + a0;
            const uint32_t nl = a1 - a0;
            uint32_t m = 0;
            bool self = false;
            if (lane < lvL.nconf) {
                const uint32_t y = fidx[lane];
                if (y == kSelf) {
                    self = true;
                } else if (y != kNone) {
                    const uint32_t q = lower_bound_u32(LL, nl, y);
                    m = q < nl && LL[q] == y;
                }
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) m += __shfl_xor_sync(kFull, m, o);
            self = __any_sync(kFull, self);
            const uint32_t nexcl = __popc(__ballot_sync(kFull, xc != kNone));
            sum = (unsigned long long)(nd - nexcl) * (unsigned long long)(nl - m);
            if (self) {
                // x whose own vertex lies in LL (excluded x not counted)
                uint32_t hits = isect_count_vid(D, nd, lv.cand, LL, nl, lvL.cand);
                bool xin = false;
                if (xc != kNone) {
                    const uint32_t v = lv.cand[xc];
                    uint32_t l2 = 0, h2 = nl;
                    while (l2 < h2) {
                        const uint32_t mid = (l2 + h2) >> 1;
                        if (lvL.cand[LL[mid]] < v) l2 = mid + 1; else h2 = mid;
                    }
                    xin = l2 < nl && lvL.cand[LL[l2]] == v;
                }
                hits -= __popc(__ballot_sync(kFull, xin));
                sum -= hits;
                touched += min(nd, nl);
            }
        }
        add_count(sum);
        elems += touched;
    }

    __device__ __forceinline__ bool lane_leaf_ok() const {
        return MODE == ASDM_MODE_COUNT && L[n - 1].nback <= kLaneLeafLists;
    }

    // LOCAL mode with a one-list last level and leaf weights: the last level
    // of every level-(n-2) survivor is handled by its lane
    __device__ __forceinline__ bool local_leaf_ok() const {
        return MODE == ASDM_MODE_LOCAL && lw && L[n - 1].nback == 1;
    }

    // For the level before the last: the candidate index in C(u_last) of every
    // earlier vertex the last level must avoid (kNone when it is not a
    // candidate there, kSelf when it is level d's own vertex).
    __device__ void prepare_lane_leaf(uint32_t d) {
        const DLevel lvL = L[n - 1];
        if (lane < lvL.nconf) {
            const uint32_t c = CF[lvL.conf_first + lane];
            uint32_t y = kSelf;
            if (c < d) {
                const uint32_t v = vid[c];
                y = lower_bound_u32(lvL.cand, lvL.ncand, v);
                if (y >= lvL.ncand || lvL.cand[y] != v) y = kNone;
            }
            fidx[lane] = y;
        }
        __syncwarp();
    }

    // Last-level count for survivor x of level d = n-2, computed by this lane
    // alone.  Returns false (and leaves the survivor to the warp-wide path)
    // when the lists are too long for one lane.
    __device__ bool lane_leaf(uint32_t d, uint32_t x, unsigned long long &out, unsigned long long &touched) {
        const DLevel lvL = L[n - 1];
        const uint32_t m = lvL.nback;
        const uint32_t *p[kLaneLeafLists];
        uint32_t len[kLaneLeafLists];
        uint32_t best = 0xFFFFFFFFu, bi = 0, tot = 0;
#pragma unroll
        for (uint32_t k = 0; k < kLaneLeafLists; ++k) {
            p[k] = nullptr;
            len[k] = 0;
            if (k < m) {
                const DBack bk = B[lvL.back_first + k];
                const uint32_t ij = bk.level == d ? x : idx[bk.level];
                const uint32_t a0 = bk.off[ij], a1 = bk.off[ij + 1];
                p[k] = bk.list + a0;
                len[k] = a1 - a0;
                tot += len[k];
                if (len[k] < best) { best = len[k]; bi = k; }
            }
        }
        if (m > 1 && best > a.lane_leaf_max) return false;
        // a single list is not read: its length (two offsets) is the count
        touched += m == 1 ? 2 : tot;
        unsigned long long c = 0;
        if (m == 1) {
            c = len[0];
        } else if (best) {
            // the shortest list drives; the others are galloped from cursors
            const uint32_t *dp = p[0];
            uint32_t dl = len[0];
#pragma unroll
            for (uint32_t k = 1; k < kLaneLeafLists; ++k)
                if (k == bi) { const uint32_t *tp = p[0]; p[0] = p[k]; p[k] = tp; uint32_t tl = len[0]; len[0] = len[k]; len[k] = tl; }
            dp = p[0];
            dl = len[0];
            uint32_t cur[kLaneLeafLists] = {0, 0, 0, 0};
            for (uint32_t i = 0; i < dl; ++i) {
                const uint32_t v = dp[i];
                bool in = true, done = false;
#pragma unroll
                for (uint32_t k = 1; k < kLaneLeafLists; ++k) {
                    if (k < m && in) {
                        const uint32_t q = gallop_lb(p[k], cur[k], len[k], v);
                        cur[k] = q;
                        if (q >= len[k]) { done = true; in = false; }
                        else in = p[k][q] == v;
                    }
                }
                c += in;
                if (done) break;
            }
        }
        if (c && lvL.nconf) {
            // same-label earlier vertices that sit in every list are not matches
            for (uint32_t k = 0; k < lvL.nconf; ++k) {
                uint32_t y = fidx[k];
                if (y == kSelf) {
                    const uint32_t v = L[d].cand[x];
                    y = lower_bound_u32(lvL.cand, lvL.ncand, v);
                    if (y >= lvL.ncand || lvL.cand[y] != v) y = kNone;
                }
                if (y == kNone) continue;
                bool in = true;
#pragma unroll
                for (uint32_t j = 0; j < kLaneLeafLists; ++j) {
                    if (j < m && in) {
                        const uint32_t q = lower_bound_u32(p[j], len[j], y);
                        in = q < len[j] && p[j][q] == y;
                    }
                }
                c -= in;
            }
        }
        out = c;
        return true;
    }

    __device__ __forceinline__ void add_count(unsigned long long c) {
        const unsigned long long nc = count + c;
        overflow |= nc < count;
        count = nc;
    }

    // Moves this warp's count into the global total (lane 0), checking for
    // uint64 wrap-around and the caller's count limit.
    __device__ void flush_count() {
        if (lane == 0 && (count || overflow)) {
            if (MULTI) {
                // per-query totals; an overflow marks only that query
                const unsigned long long old = atomicAdd(&a.qcounts[q], count);
                if (overflow || old + count < old) atomicOr(&a.qflags[q], kFlagOverflow);
                if (a.count_limit && old + count > a.count_limit) atomicOr(&a.qflags[q], kFlagLimit);
                atomicAdd(&a.ctr[kCtrCount], count);
            } else {
                const unsigned long long old = atomicAdd(&a.ctr[kCtrCount], count);
                uint32_t f = 0;
                if (overflow || old + count < old) f |= kFlagOverflow;
                if (a.count_limit && old + count > a.count_limit) f |= kFlagLimit;
                if (f) atomicOr((unsigned int *)&a.ctr[kCtrFlags], f);
            }
        }
        count = 0;
        overflow = false;
    }

    // Loads the candidate-edge lists of level d's earlier neighbours into the
    // level's slots and picks the shortest as driver.  Returns its length.
    __device__ uint32_t setup(uint32_t d, bool whole = true) {
        const DLevel lv = L[d];
        uint32_t s_len = 0xFFFFFFFFu;
        if (lane < lv.nback) {
            const DBack bk = B[lv.back_first + lane];
            const uint32_t ij = idx[bk.level];
            const uint32_t s0 = bk.off[ij];
            s_len = bk.off[ij + 1] - s0;
            sstart[lv.back_first + lane] = s0;
            slen[lv.back_first + lane] = s_len;
            scur[lv.back_first + lane] = 0;
        }
        uint32_t key = s_len, who = lane;
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const uint32_t k2 = __shfl_xor_sync(kFull, key, o), w2 = __shfl_xor_sync(kFull, who, o);
            if (k2 < key || (k2 == key && w2 < who)) { key = k2; who = w2; }
        }
        uint32_t tot = lane < lv.nback ? s_len : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) tot += __shfl_xor_sync(kFull, tot, o);
        // a counted last level with one list reads only its two offsets; a
        // level searched over part of its driver list is counted by the caller
        if (whole) elems += (MODE == ASDM_MODE_COUNT && d + 1 == n && lv.nback == 1) ? 2 : tot;
        inter += lv.nback >= 2;
        if (lane == 0) {
            drv[d] = who;
            dpos[d] = 0;
            dend[d] = key;
            cnt[d] = 0;
            pos[d] = 0;
        }
        __syncwarp();
        return key;
    }

    // Gives the upper half of the undispatched driver range of the shallowest
    // open level to the donation ring (called when more warps are idle than
    // records are waiting).
    __device__ void try_donate(uint32_t base, uint32_t d) {
        uint32_t s = kNone;
        for (uint32_t l = base; l <= d; ++l)
            if (dend[l] > dpos[l]) { s = l; break; }
        if (s == kNone) return;
        unsigned long long pos = ~0ull;
        if (lane == 0) {
            volatile unsigned long long *vc = (volatile unsigned long long *)a.ctr;
            unsigned long long p = vc[kCtrTail];
            for (int tries = 0; tries < 64; ++tries) {
                const unsigned long long seq = *(volatile unsigned long long *)&a.qseq[p & (kQueueCap - 1)];
                if (seq == p) {
                    const unsigned long long prev = atomicCAS(&a.ctr[kCtrTail], p, p + 1);
                    if (prev == p) { pos = p; break; }
                    p = prev;
                } else if (seq < p) {
                    break;  // ring full
                } else {
                    p = vc[kCtrTail];
                }
            }
        }
        pos = __shfl_sync(kFull, pos, 0);
        if (pos == ~0ull) return;
        const uint32_t lo = dpos[s] + (dend[s] - dpos[s]) / 2, hi = dend[s];
        uint32_t *rec = a.queue + (pos & (kQueueCap - 1)) * kRecWords;
        if (lane < s) rec[4 + lane] = idx[lane];
        if (lane == 0) {
            rec[0] = q;
            rec[1] = s;
            rec[2] = lo;
            rec[3] = hi;
        }
        __threadfence();
        __syncwarp();
        if (lane == 0) {
            atomicExch(&a.qseq[pos & (kQueueCap - 1)], pos + 1);
            atomicAdd(&a.ctr[kCtrDonated], 1ull);
            dend[s] = lo;
        }
        __syncwarp();
    }

    // Idle: polls the donation ring.  Returns the claimed position, or ~0
    // when no warp is working any more, a stop flag is set, or the wait's
    // time bound (the run's deadline, else kIdleMaxNs) has passed.  The
    // caller copies the record and then calls release().
    __device__ unsigned long long take_queued(uint64_t deadline) {
        unsigned long long pos = ~0ull;
        if (lane == 0) {
            volatile unsigned long long *vc = (volatile unsigned long long *)a.ctr;
            atomicAdd(&a.ctr[kCtrIdle], 1ull);
            const uint64_t t0 = globaltimer();
            const uint64_t until = deadline ? deadline : t0 + kIdleMaxNs;
            uint32_t nap = 128;
            for (uint32_t it = 0;; ++it) {
                const unsigned long long p = vc[kCtrHead];
                const unsigned long long seq = *(volatile unsigned long long *)&a.qseq[p & (kQueueCap - 1)];
                if (seq == p + 1) {
                    if (atomicCAS(&a.ctr[kCtrHead], p, p + 1) == p) { pos = p; break; }
                    nap = 128;
                } else if (seq < p + 1) {
                    if (vc[kCtrActive] == 0 || (vc[kCtrFlags] & kStopFlags)) break;
                    if ((it & 255u) == 255u && globaltimer() > until) break;
                    __nanosleep(nap);
                    nap = min(2 * nap, kIdleSleepMaxNs);
                }
            }
            if (pos != ~0ull) atomicAdd(&a.ctr[kCtrActive], 1ull);
            atomicAdd(&a.ctr[kCtrIdleNs], (unsigned long long)(globaltimer() - t0));
            atomicAdd(&a.ctr[kCtrIdle], ~0ull);
            __threadfence();
        }
        return __shfl_sync(kFull, pos, 0);
    }

    __device__ void release(unsigned long long pos) {
        __syncwarp();
        if (lane == 0) {
            __threadfence();
            atomicExch(&a.qseq[pos & (kQueueCap - 1)], pos + kQueueCap);
        }
    }

    // Membership of x (this lane's driver element) in every non-driver list
    // of level d from the shared cursors; advances the cursors.  drem is the
    // number of driver entries from this round's first to the end of the
    // range.  A list whose unread part is at most merge_ratio x drem long is
    // merged with the drivers a window of 32 entries at a time (about
    // len / drem windows per round); a longer one is galloped by every lane.
    __device__ __forceinline__ bool probe(const DLevel &lv, uint32_t dslot, uint32_t x, bool valid, uint32_t lastlane,
                                          uint32_t drem) {
        bool ok = valid;
        for (uint32_t s = 0; s < lv.nback; ++s) {
            const uint32_t sl = lv.back_first + s;
            if (sl == dslot) continue;
            if (!__any_sync(kFull, ok)) break;
            const uint32_t *lst = B[sl].list + sstart[sl];
            const uint32_t len = slen[sl];
            const uint32_t cur = scur[sl];
            uint32_t nc;
            if ((uint64_t)(len - cur) <= (uint64_t)a.merge_ratio * drem) {
                ok = warp_merge_member(lst, cur, len, x, ok, lastlane, lane, nc) && ok;
            } else {
                const uint32_t q = valid ? gallop_lb(lst, cur, len, x) : len;
                ok = ok && q < len && lst[q] == x;
                nc = __shfl_sync(kFull, q, lastlane);
            }
            __syncwarp();
            if (lane == 0) scur[sl] = nc;
            __syncwarp();
        }
        return ok;
    }

    __device__ __forceinline__ bool no_conflict(const DLevel &lv, uint32_t vx) {
        bool ok = true;
        for (uint32_t c = 0; c < lv.nconf; ++c) ok &= vx != vid[CF[lv.conf_first + c]];
        return ok;
    }

    // Next 32 driver elements of a non-last level into its stack slot.
    __device__ void fill_chunk(uint32_t d) {
        const DLevel lv = L[d];
        const uint32_t dslot = lv.back_first + drv[d];
        const uint32_t *dl = B[dslot].list + sstart[dslot];
        const uint32_t dlen = dend[d];
        const uint32_t p0 = dpos[d];
        const uint32_t p = p0 + lane;
        const bool valid = p < dlen;
        const uint32_t x = valid ? dl[p] : 0xFFFFFFFFu;
        const uint32_t lastlane = min(31u, dlen - 1 - p0);
        bool ok = probe(lv, dslot, x, valid, lastlane, dlen - p0);
        if (lv.nconf && __any_sync(kFull, ok)) {
            const uint32_t vx = ok ? lv.cand[x] : 0;
            ok = ok && no_conflict(lv, vx);
        }
        if (d + 2 == n && lane_leaf_ok()) {
            // count the last level of every survivor lane-parallel; survivors
            // with long lists stay buffered for the warp-wide leaf
            unsigned long long c = 0, touched = 0;
            const bool done = ok && lane_leaf(d, x, c, touched);
            ok = ok && !done;
            const uint32_t dm = __ballot_sync(kFull, done);
            inter += (L[n - 1].nback >= 2) ? __popc(dm) : 0;
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                c += __shfl_xor_sync(kFull, c, o);
                touched += __shfl_xor_sync(kFull, touched, o);
            }
            add_count(c);
            elems += touched;
        } else if (d + 2 == n && local_leaf_ok()) {
            // LOCAL: every survivor's last level by its lane: its count (list
            // length minus the same-label earlier vertices lying in it), its
            // own local count, a leaf weight for the pass after the kernel
            // (which adds 1 to every list entry; the conflict vertices in the
            // list are taken back out here)
            unsigned long long c = 0;
            if (ok) {
                const DLevel lvL = L[n - 1];
                const DBack bk = B[lvL.back_first];
                const uint32_t ij = bk.level == d ? x : idx[bk.level];
                const uint32_t a0 = bk.off[ij], a1 = bk.off[ij + 1];
                c = a1 - a0;
                for (uint32_t k = 0; k < lvL.nconf && c; ++k) {
                    uint32_t y = fidx[k];
                    if (y == kSelf) {
                        const uint32_t v = lv.cand[x];
                        y = lower_bound_u32(lvL.cand, lvL.ncand, v);
                        if (y >= lvL.ncand || lvL.cand[y] != v) y = kNone;
                    }
                    if (y == kNone) continue;
                    const uint32_t q = lower_bound_u32(bk.list + a0, a1 - a0, y);
                    if (q < a1 - a0 && bk.list[a0 + q] == y) {
                        --c;
                        atomicAdd(&local[(unsigned long long)lvL.cand[y] * n + lvL.u], ~0ull);  // -1
                    }
                }
                if (a1 > a0) atomicAdd(&lw[ij], 1ull);
                if (c) atomicAdd(&local[(unsigned long long)lv.cand[x] * n + lv.u], c);
                elems += 2;
            }
            ok = false;
#pragma unroll
            for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
            if (c && lane < d) atomicAdd(&local[(unsigned long long)vid[lane] * n + L[lane].u], c);
            add_count(c);
        } else if (d + 3 == n && lane_tail_ok(d)) {
            // the last two levels of every entry lane-parallel; entries whose
            // intersections are long stay buffered for the warp-wide tail
            unsigned long long c = 0, touched = 0;
            const bool done = ok && lane_tail(d, x, c, touched);
            ok = ok && !done;
            tails_lane += __popc(__ballot_sync(kFull, done));
#pragma unroll
            for (int o = 16; o; o >>= 1) {
                c += __shfl_xor_sync(kFull, c, o);
                touched += __shfl_xor_sync(kFull, touched, o);
            }
            add_count(c);
            elems += touched;
        }
        const uint32_t mask = __ballot_sync(kFull, ok);
        if (ok) buf[32 * d + __popc(mask & ((1u << lane) - 1))] = x;
        __syncwarp();
        if (lane == 0) {
            cnt[d] = __popc(mask);
            pos[d] = 0;
            dpos[d] = p0 + 32;
        }
        __syncwarp();
    }

    __device__ void emit_rows(uint32_t d, uint32_t vx, bool ok, uint32_t mask) {
        unsigned long long base = 0;
        if (lane == 0 && mask) base = atomicAdd(&a.ctr[kCtrRows], (unsigned long long)__popc(mask));
        base = __shfl_sync(kFull, base, 0);
        if (ok) {
            const unsigned long long r = base + __popc(mask & ((1u << lane) - 1));
            if (r < a.row_cap) {
                uint32_t *row = a.rows + r * n;
                for (uint32_t j = 0; j < d; ++j) row[L[j].u] = vid[j];
                row[L[d].u] = vx;
            } else {
                atomicOr((unsigned int *)&a.ctr[kCtrFlags], kFlagCapacity);
            }
        }
    }

    // The last level: count (and in LOCAL/EMBED modes, emit) its matches.
    __device__ void leaf(uint32_t d) {
        // driver positions [lo, hi): the whole list, or a root block's part of it
        const DLevel lv = L[d];
        const uint32_t dslot = lv.back_first + drv[d];
        const uint32_t *dl = B[dslot].list + sstart[dslot];
        const uint32_t lo = dpos[d], hi = dend[d];
        unsigned long long total = 0;
        if (MODE == ASDM_MODE_COUNT) {
            if (lv.nback == 1) {
                total = hi - lo;
            } else {
                for (uint32_t p0 = lo; p0 < hi; p0 += 32) {
                    const uint32_t p = p0 + lane;
                    const bool valid = p < hi;
                    const uint32_t x = valid ? dl[p] : 0xFFFFFFFFu;
                    const bool ok = probe(lv, dslot, x, valid, min(31u, hi - 1 - p0), hi - p0);
                    total += __popc(__ballot_sync(kFull, ok));
                }
            }
            if (lv.nconf && total) {
                // same-label earlier vertices inside the intersection are not matches
                bool present = false;
                if (lane < lv.nconf) {
                    const uint32_t v = vid[CF[lv.conf_first + lane]];
                    const uint32_t y = lower_bound_u32(lv.cand, lv.ncand, v);
                    present = y < lv.ncand && lv.cand[y] == v;
                    for (uint32_t s = 0; present && s < lv.nback; ++s) {
                        const uint32_t sl = lv.back_first + s;
                        const uint32_t *lst = B[sl].list + sstart[sl];
                        const uint32_t len = slen[sl];
                        const uint32_t q = lower_bound_u32(lst, len, y);
                        present = q < len && lst[q] == y && (sl != dslot || (q >= lo && q < hi));
                    }
                }
                total -= __popc(__ballot_sync(kFull, present));
            }
        } else if (MODE == ASDM_MODE_LOCAL && lw && lv.nback == 1 && lo == 0 && hi == slen[dslot]) {
            // the whole list of one candidate: one weight for the pass after
            // the kernel, minus the same-label earlier vertices lying in it
            total = hi - lo;
            bool present = false;
            uint32_t v = 0;
            if (lane < lv.nconf) {
                v = vid[CF[lv.conf_first + lane]];
                const uint32_t y = lower_bound_u32(lv.cand, lv.ncand, v);
                if (y < lv.ncand && lv.cand[y] == v) {
                    const uint32_t q = lower_bound_u32(dl, hi, y);
                    present = q < hi && dl[q] == y;
                }
            }
            if (present) atomicAdd(&local[(unsigned long long)v * n + lv.u], ~0ull);  // -1
            total -= __popc(__ballot_sync(kFull, present));
            if (lane == 0) atomicAdd(&lw[idx[B[dslot].level]], 1ull);
            if (total && lane < d) atomicAdd(&local[(unsigned long long)vid[lane] * n + L[lane].u], total);
        } else {
            for (uint32_t p0 = lo; p0 < hi; p0 += 32) {
                const uint32_t p = p0 + lane;
                const bool valid = p < hi;
                const uint32_t x = valid ? dl[p] : 0xFFFFFFFFu;
                bool ok = probe(lv, dslot, x, valid, min(31u, hi - 1 - p0), hi - p0);
                const uint32_t vx = ok ? lv.cand[x] : 0;
                ok = ok && no_conflict(lv, vx);
                const uint32_t mask = __ballot_sync(kFull, ok);
                total += __popc(mask);
                if ((MODE & ASDM_MODE_LOCAL) && ok) atomicAdd(&local[(unsigned long long)vx * n + lv.u], 1ull);
                if (MODE & ASDM_MODE_EMBED) emit_rows(d, vx, ok, mask);
            }
            if ((MODE & ASDM_MODE_LOCAL) && total && lane < d)
                atomicAdd(&local[(unsigned long long)vid[lane] * n + L[lane].u], total);
        }
        add_count(total);
    }

    // A full match at the last level when the query has one or two vertices.
    __device__ void single(uint32_t d) {
        add_count(1);
        if (MODE & ASDM_MODE_LOCAL) {
            if (lane <= d) atomicAdd(&local[(unsigned long long)vid[lane] * n + L[lane].u], 1ull);
        }
        if (MODE & ASDM_MODE_EMBED) {
            const uint32_t vx = vid[d];
            emit_rows(d, vx, lane == 0, 1u);
        }
    }
};

// Depth-first search from level `base` (already set up) down to the last
// level; returns false when a stop flag (overflow, time or count limit,
// internal error) ended it early.
template <uint32_t MODE, bool MULTI>
__device__ bool dfs(const EnumArgs &a, Warp<MODE, MULTI> &W, uint32_t lane, uint32_t base, uint32_t &iter,
                    uint64_t deadline) {
    volatile unsigned int *flags = reinterpret_cast<volatile unsigned int *>(&a.ctr[kCtrFlags]);
    const uint32_t n = W.n;
    uint32_t d = base;
    while (d >= base) {
        if ((++iter & 63u) == 0) {
            uint32_t st = 0, want = 0;
            W.flush_count();
            if (lane == 0) {
                st = *flags & kStopFlags;
                if (!st && deadline && globaltimer() > deadline) {
                    atomicOr((unsigned int *)&a.ctr[kCtrFlags], kFlagTimeout);
                    st = kFlagTimeout;
                }
                volatile unsigned long long *vc = (volatile unsigned long long *)a.ctr;
                const unsigned long long idle = vc[kCtrIdle], pend = vc[kCtrTail] - vc[kCtrHead];
                want = idle > pend && (long long)pend >= 0;
            }
            if (__shfl_sync(kFull, st, 0)) return false;
            if (W.query_stopped()) return true;  // abandon this query's subtree
            if (__shfl_sync(kFull, want, 0)) W.try_donate(base, d);
        }
        if (W.pos[d] < W.cnt[d]) {
            const uint32_t x = W.buf[32 * d + W.pos[d]];
            __syncwarp();
            if (lane == 0) {
                W.pos[d] += 1;
                W.idx[d] = x;
                W.vid[d] = W.L[d].cand[x];
            }
            __syncwarp();
            ++d;
            const bool closed = W.closed_at(d);
            const uint32_t len = W.setup(d, !closed);
            if (closed) {
                if (len) {
                    W.prepare_lane_leaf(d);
                    W.tail2(d, 0, len);
                }
                --d;
            } else if (d == n - 1) {
                if (len) W.leaf(d);
                --d;
            } else if (len == 0) {
                --d;
            } else if (d + 2 == n && (W.lane_leaf_ok() || W.local_leaf_ok())) {
                W.prepare_lane_leaf(d);
            } else if (W.lane_tail_ok(d)) {
                W.prepare_lane_tail(d);
            }
            continue;
        }
        if (W.dpos[d] < W.dend[d]) {
            W.fill_chunk(d);
            continue;
        }
        --d;
    }
    return true;
}

// Level `s` set up from the prefix in W.idx[0..s-1], restricted to driver
// positions [lo, hi); then searched to the end.
template <uint32_t MODE, bool MULTI>
__device__ __forceinline__ bool run_range(const EnumArgs &a, Warp<MODE, MULTI> &W, uint32_t lane, uint32_t s, uint32_t lo, uint32_t hi,
                          uint32_t &iter, uint64_t deadline) {
    if (W.closed_at(s)) {
        W.setup(s, false);
        if (hi > lo) {
            W.prepare_lane_leaf(s);
            W.tail2(s, lo, hi);
        }
        return true;
    }
    W.setup(s, false);
    {
        // list entries this range touches: the driver positions [lo, hi), one
        // probe of every other list per driver entry, and the lists' offsets
        const DLevel lv = W.L[s];
        const bool by_length = MODE == ASDM_MODE_COUNT && s + 1 == W.n && lv.nback == 1;
        W.elems += 2ull * lv.nback + (by_length ? 0ull : (unsigned long long)(hi - lo) * lv.nback);
    }
    if (lane == 0) {
        W.dpos[s] = lo;
        W.dend[s] = hi;
    }
    __syncwarp();
    if (s == W.n - 1) {
        if (hi > lo) W.leaf(s);
        return true;
    }
    if (s + 2 == W.n && (W.lane_leaf_ok() || W.local_leaf_ok())) W.prepare_lane_leaf(s);
    else if (W.lane_tail_ok(s)) W.prepare_lane_tail(s);
    return dfs(a, W, lane, s, iter, deadline);
}

// The warp loop shared by the single-query kernel and the batch kernel.
// Root tasks are blocks of consecutive (level-0, level-1) candidate pairs of
// one query (pairs ordered by level-0 candidate, then by position in its
// level-1 list); a block is decoded with one warp-wide search and run as
// level-1 ranges.  When roots run out, warps steal donated ranges.
template <uint32_t MODE, bool MULTI>
__device__ void warp_loop(const EnumArgs &a, Warp<MODE, MULTI> &W, uint32_t lane) {
    const unsigned long long nblocks = MULTI ? a.task_pre[a.nquery] : a.ntasks;
    uint32_t iter = 0;
    bool stop = false, roots_left = true;
    uint64_t deadline = 0;
    if (a.limit_ns && lane == 0) deadline = globaltimer() + a.limit_ns;
    // a warp counts as active (kCtrActive) from its first root task until the
    // roots run out, not per task: fewer atomics on one hot counter
    if (lane == 0) atomicAdd(&a.ctr[kCtrActive], 1ull);
    while (!stop) {
        if (roots_left) {
            unsigned long long b = 0;
            if (lane == 0) {
                b = atomicAdd(&a.ctr[kCtrTask], 1ull);
                if (b >= nblocks) atomicAdd(&a.ctr[kCtrActive], ~0ull);
            }
            b = __shfl_sync(kFull, b, 0);
            if (b < nblocks) {
                const long long c0 = clock64();
                unsigned long long K = a.blk, P = a.pairs;
                if (MULTI) {
                    const uint32_t qq = warp_find_row64(a.task_pre, a.nquery, b, lane);
                    W.bind(qq);
                    b -= a.task_pre[qq];
                    K = a.qd[qq].blk;
                    P = a.qd[qq].pairs;
                }
                unsigned long long t = b * K;
                unsigned long long t_end = min(t + K, P);
                // a query past its count limit or time budget is abandoned: its remaining
                // root tasks are skipped at once (the task counter jumps past them)
                W.mark();
                if (W.query_stopped()) {
                    t_end = t;
                    if (MULTI && lane == 0) atomicMax(&a.ctr[kCtrTask], a.task_pre[W.q + 1]);
                }
                if (W.n == 1) {
                    for (; t < t_end; ++t) {
                        if (lane == 0) {
                            W.idx[0] = (uint32_t)t;
                            W.vid[0] = W.L[0].cand[(uint32_t)t];
                        }
                        __syncwarp();
                        W.single(0);
                    }
                } else {
                    // level-1 lists of the level-0 candidates, as CSR offsets
                    const uint32_t *off01 = W.B[W.L[1].back_first].off;
                    uint32_t i0 = warp_find_row32(off01, W.L[0].ncand, t, lane);
                    while (t < t_end && !stop) {
                        const uint32_t r0 = off01[i0], r1 = off01[i0 + 1];
                        if (r1 <= t) {
                            ++i0;
                            continue;
                        }
                        const uint32_t seg_hi = (uint32_t)min((unsigned long long)r1, t_end);
                        if (lane == 0) {
                            W.idx[0] = i0;
                            W.vid[0] = W.L[0].cand[i0];
                        }
                        __syncwarp();
                        stop = !run_range(a, W, lane, 1, (uint32_t)t - r0, seg_hi - r0, iter, deadline);
                        t = seg_hi;
                        ++i0;
                    }
                }
                W.charge();
                if (lane == 0 && MULTI && a.qcycles)
                    atomicAdd(&a.qcycles[W.q], (unsigned long long)(clock64() - c0));
                continue;
            }
            roots_left = false;
        }
        const unsigned long long qpos = W.take_queued(deadline);
        if (qpos == ~0ull) break;
        const volatile uint32_t *rec = a.queue + (qpos & (kQueueCap - 1)) * kRecWords;
        if (MULTI) W.bind(rec[0]);
        const uint32_t s = rec[1], lo = rec[2], hi = rec[3];
        if (lane < s) {
            const uint32_t x = rec[4 + lane];
            W.idx[lane] = x;
            W.vid[lane] = W.L[lane].cand[x];
        }
        W.release(qpos);
        __syncwarp();
        const long long c0 = clock64();
        W.mark();
        if (!W.query_stopped()) stop = !run_range(a, W, lane, s, lo, hi, iter, deadline);
        W.charge();
        if (lane == 0) {
            if (MULTI && a.qcycles) atomicAdd(&a.qcycles[W.q], (unsigned long long)(clock64() - c0));
            atomicAdd(&a.ctr[kCtrActive], ~0ull);
        }
    }
    // a warp stopped while it still had roots leaves the active count
    if (roots_left && lane == 0) atomicAdd(&a.ctr[kCtrActive], ~0ull);
    // flush per-warp totals
    W.flush_count();
    if (lane == 0) {
        atomicAdd(&a.ctr[kCtrInter], W.inter);
        atomicAdd(&a.ctr[kCtrElems], W.elems);
        atomicAdd(&a.ctr[kCtrTailLane], W.tails_lane);
        atomicAdd(&a.ctr[kCtrTailWarp], W.tails_warp);
    }
}

template <uint32_t MODE>
__global__ void __launch_bounds__(kThreads) enum_kernel(EnumArgs a) {
    extern __shared__ __align__(16) uint32_t sm[];
    DLevel *L = reinterpret_cast<DLevel *>(sm);
    DBack *B = reinterpret_cast<DBack *>(L + a.n);
    uint32_t *CF = reinterpret_cast<uint32_t *>(B + a.nb);
    {
        const uint32_t *src_l = reinterpret_cast<const uint32_t *>(a.lv);
        uint32_t *dst_l = reinterpret_cast<uint32_t *>(L);
        for (uint32_t i = threadIdx.x; i < a.n * (uint32_t)(sizeof(DLevel) / 4); i += blockDim.x) dst_l[i] = src_l[i];
        const uint32_t *src_b = reinterpret_cast<const uint32_t *>(a.bk);
        uint32_t *dst_b = reinterpret_cast<uint32_t *>(B);
        for (uint32_t i = threadIdx.x; i < a.nb * (uint32_t)(sizeof(DBack) / 4); i += blockDim.x) dst_b[i] = src_b[i];
        for (uint32_t i = threadIdx.x; i < a.nc; i += blockDim.x) CF[i] = a.conf[i];
    }
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *wmem = sm + plan_words(a.n, a.nb, a.nc) + warp * warp_words(a.n, a.nb);
    Warp<MODE, false> W(a, L, B, CF, wmem, lane, a.n, a.n, a.nb);
    warp_loop<MODE, false>(a, W, lane);
}

// Many queries in one persistent launch (COUNT mode): root tasks of every
// query form one range claimed by atomicAdd, plans are read from global
// memory, counts go to per-query totals.
template <int MINB, uint32_t MODE = ASDM_MODE_COUNT>
__global__ void __launch_bounds__(kThreads, MINB) enum_batch_kernel(EnumArgs a) {
    extern __shared__ __align__(16) uint32_t sm[];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t *wmem = sm + warp * warp_words(a.maxn, a.maxnb);
    const QDesc d0 = a.qd[0];
    Warp<MODE, true> W(a, d0.lv, d0.bk, d0.conf, wmem, lane, d0.n, a.maxn, a.maxnb);
    W.local = d0.local;
    W.ps = d0.ps;
    W.rev_off = d0.rev_off;
    W.rev_list = d0.rev_list;
    W.tail = d0.tail;
    W.xmap_a = d0.xmap_a;
    W.xmap_z = d0.xmap_z;
    W.lw = d0.lw;
    warp_loop<MODE, true>(a, W, lane);
}

// Prefix sums for kTailChain plans: entry t of a segment (one plan's driver
// edge of level n-2, in candidate-edge order) gets the length of the last
// level's list of that entry; a scan over all segments follows.
struct TailSeg {
    const uint32_t *list;   // candidate-edge entries of level n-2's driver edge
    const uint32_t *off2;   // offsets of the last level's lists, by candidate of level n-2
    unsigned long long start, len;
};

__global__ void tail_lens(const TailSeg *__restrict__ seg, uint32_t nseg, unsigned long long total,
                          uint32_t *__restrict__ lens) {
    for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nseg;  // the last segment starting at or before t
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (seg[mid].start <= t) lo = mid; else hi = mid;
        }
        const uint32_t x = seg[lo].list[t - seg[lo].start];
        lens[t] = seg[lo].off2[x + 1] - seg[lo].off2[x];
    }
}

// LOCAL mode: the last level's local counts from the leaf weights.  Segment
// k covers the candidates of one query's leaf source level: weight w[i] is
// added to every last-level candidate in list(i).
struct PushSeg {
    const unsigned long long *w;
    const uint32_t *off;          // candidate-edge offsets (source level -> last level)
    const uint32_t *list;         // entries: indices into C(u_last)
    const uint32_t *cand;         // C(u_last)
    unsigned long long *local;    // |Vg| x n block of the query
    uint32_t n, u;                // query size, last query vertex
    unsigned long long start, len;
};

__global__ void push_leaf(const PushSeg *__restrict__ seg, uint32_t nseg, unsigned long long total) {
    for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nseg;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (seg[mid].start <= t) lo = mid; else hi = mid;
        }
        const PushSeg sg = seg[lo];
        const unsigned long long i = t - sg.start;
        const unsigned long long c = sg.w[i];
        if (!c) continue;
        for (uint32_t k = sg.off[i]; k < sg.off[i + 1]; ++k)
            atomicAdd(&sg.local[(unsigned long long)sg.cand[sg.list[k]] * sg.n + sg.u], c);
    }
}

// Leaf weights of LOCAL-mode plans whose last level has one backward edge:
// one zeroed device array (*d_w, the caller frees), per plan a pointer or null.
int leaf_weights(const std::vector<const asdm_cs *> &cs, const std::vector<const asdm_plan *> &plans,
                 std::vector<unsigned long long *> &lw, unsigned long long **d_w, cudaStream_t s) {
    *d_w = nullptr;
    lw.assign(cs.size(), nullptr);
    std::vector<uint64_t> at(cs.size(), 0);
    uint64_t total = 0;
    for (size_t i = 0; i < cs.size(); ++i) {
        const asdm_plan &p = *plans[i];
        const size_t n = p.order.size();
        if (n < 2 || n != cs[i]->q.n || p.back[n - 1].size() != 1) continue;
        at[i] = total;
        total += cs[i]->ncand[p.order[p.back[n - 1][0].first]];
        lw[i] = reinterpret_cast<unsigned long long *>(1);  // marker until the array exists
    }
    if (total == 0) {
        lw.assign(cs.size(), nullptr);
        return ASDM_OK;
    }
    ASDM_TRY(dalloc(d_w, total, s));
    ASDM_CUDA(cudaMemsetAsync(*d_w, 0, total * sizeof(unsigned long long), s));
    for (size_t i = 0; i < cs.size(); ++i)
        if (lw[i]) lw[i] = *d_w + at[i];
    return ASDM_OK;
}

// The pass after the kernel for those plans (local blocks as given).
int push_leaf_weights(const std::vector<const asdm_cs *> &cs, const std::vector<const asdm_plan *> &plans,
                      const std::vector<unsigned long long *> &lw, const std::vector<unsigned long long *> &local,
                      int num_sms, cudaStream_t s) {
    std::vector<PushSeg> segs;
    unsigned long long total = 0;
    for (size_t i = 0; i < cs.size(); ++i) {
        if (!lw[i]) continue;
        const asdm_cs &c = *cs[i];
        const asdm_plan &p = *plans[i];
        const size_t n = p.order.size();
        const uint32_t e = p.back[n - 1][0].second;
        const uint32_t src = p.order[p.back[n - 1][0].first], ul = p.order[n - 1];
        PushSeg sg{lw[i], c.d_eoff + c.eoff_base[e], c.d_elist + c.elist_base[e], c.d_cand + c.cand_base[ul],
                   local[i], (uint32_t)n, ul, total, c.ncand[src]};
        segs.push_back(sg);
        total += c.ncand[src];
    }
    if (segs.empty() || total == 0) return ASDM_OK;
    PushSeg *d_seg = nullptr;
    ASDM_TRY(dalloc(&d_seg, segs.size(), s));
    int rc = ASDM_OK;
    if (cudaMemcpyAsync(d_seg, segs.data(), segs.size() * sizeof(PushSeg), cudaMemcpyHostToDevice, s) != cudaSuccess) {
        rc = fail(ASDM_ERR_CUDA, "leaf-weight upload failed");
    } else {
        const unsigned grid = (unsigned)std::min<unsigned long long>((total + 255) / 256, (unsigned long long)num_sms * 32);
        push_leaf<<<grid, 256, 0, s>>>(d_seg, (uint32_t)segs.size(), total);
        ::asdm::count_launch();
        if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "leaf-weight pass failed");
    }
    cudaStreamSynchronize(s);  // the upload reads a host vector
    dfree(d_seg, s);
    return rc;
}

// Cross indices: for candidate i of one query vertex, its index in the
// candidate set of another query vertex of the same label (or kNone).
struct XSeg {
    const uint32_t *from;   // candidate set the map is indexed by
    const uint32_t *to;     // candidate set the indices point into
    uint32_t *out;
    uint32_t nto;
    uint32_t pad;
    unsigned long long start, len;
};

__global__ void cross_index(const XSeg *__restrict__ seg, uint32_t nseg, unsigned long long total) {
    for (unsigned long long t = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nseg;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (seg[mid].start <= t) lo = mid; else hi = mid;
        }
        const XSeg sg = seg[lo];
        const unsigned long long i = t - sg.start;
        const uint32_t v = sg.from[i];
        const uint32_t j = lower_bound_u32(sg.to, sg.nto, v);
        sg.out[i] = (j < sg.nto && sg.to[j] == v) ? j : kNone;
    }
}

__global__ void queue_init(unsigned long long *seq) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kQueueCap) seq[i] = i;
}

template <uint32_t MODE>
int launch(const EnumArgs &a, uint32_t smem, int num_sms, cudaStream_t s) {
    auto k = enum_kernel<MODE>;
    ASDM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    ASDM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, smem));
    if (per_sm <= 0) return fail(ASDM_ERR_INVALID, "query too large for one block's shared memory (%u bytes)", smem);
    // persistent grid: warps without a root task steal donated work
    const unsigned grid = (unsigned)std::max(1, per_sm * num_sms);
    k<<<grid, kThreads, smem, s>>>(a);
    ::asdm::count_launch();
    ASDM_CUDA(cudaGetLastError());
    return ASDM_OK;
}

}  // namespace

// Closed form of the last two levels for a COUNT-mode plan (kTail*).
uint32_t tail_mode(const asdm_plan &plan) {
    const size_t n = plan.order.size();
    if (n < 3 || plan.back[n - 1].size() != 1) return kTailNone;
    if (plan.back[n - 2].size() == 2) return n >= 4 ? kTailIsect : kTailNone;
    if (plan.back[n - 2].size() != 1) return kTailNone;
    return plan.back[n - 1][0].first == n - 2 ? kTailChain : kTailLeaf;
}

// Tail data of every plan whose mode is given in `mode` (kTailChain plans get
// prefix sums in one device array, *d_ps, which the caller frees; plans past
// kTailSumCap entries fall back to kTailNone).
constexpr unsigned long long kTailSumCap = 1ull << 29;
struct TailData {
    uint32_t mode = kTailNone;
    const unsigned long long *ps = nullptr;
    const uint32_t *rev_off = nullptr, *rev_list = nullptr;
    const uint32_t *xmap_a = nullptr, *xmap_z = nullptr;
};

// Cross-index maps for the lane tails of every plan whose level n-3 is a
// conflict level of level n-2 or n-1 (one device array, *d_x, caller frees).
int build_xmaps(const std::vector<const asdm_cs *> &cs, const std::vector<const asdm_plan *> &plans,
                std::vector<TailData> &td, uint32_t **d_x, cudaStream_t s) {
    *d_x = nullptr;
    std::vector<XSeg> segs;
    std::vector<std::pair<size_t, int>> owner;  // (plan, 0 = a / 1 = z)
    unsigned long long total = 0;
    for (size_t i = 0; i < cs.size(); ++i) {
        if (td[i].mode == kTailNone) continue;
        const asdm_plan &p = *plans[i];
        const size_t n = p.order.size();
        if (n < 4) continue;
        const uint32_t d = (uint32_t)n - 3;
        const asdm_cs &c = *cs[i];
        const uint32_t ud = p.order[d];
        for (int which = 0; which < 2; ++which) {
            const uint32_t t = (uint32_t)n - 2 + which;
            if (std::find(p.conf[t].begin(), p.conf[t].end(), d) == p.conf[t].end()) continue;
            const uint32_t ut = p.order[t];
            XSeg sg{c.d_cand + c.cand_base[ud], c.d_cand + c.cand_base[ut], nullptr, c.ncand[ut], 0, total,
                    c.ncand[ud]};
            segs.push_back(sg);
            owner.emplace_back(i, which);
            total += c.ncand[ud];
        }
    }
    if (segs.empty()) return ASDM_OK;
    ASDM_TRY(dalloc(d_x, total, s));
    for (auto &sg : segs) sg.out = *d_x + sg.start;
    XSeg *d_seg = nullptr;
    int rc = dalloc(&d_seg, segs.size(), s);
    if (rc == ASDM_OK &&
        cudaMemcpyAsync(d_seg, segs.data(), segs.size() * sizeof(XSeg), cudaMemcpyHostToDevice, s) != cudaSuccess)
        rc = fail(ASDM_ERR_CUDA, "cross-index upload failed");
    if (rc == ASDM_OK && total) {
        const unsigned grid = (unsigned)std::min<unsigned long long>((total + 255) / 256, 148ull * 32);
        cross_index<<<grid, 256, 0, s>>>(d_seg, (uint32_t)segs.size(), total);
        ::asdm::count_launch();
        if (cudaGetLastError() != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "cross-index kernel failed");
    }
    cudaStreamSynchronize(s);  // the upload reads a host vector
    dfree(d_seg, s);
    if (rc != ASDM_OK) {
        dfree(*d_x, s);
        return rc;
    }
    for (size_t k = 0; k < segs.size(); ++k) {
        if (owner[k].second == 0) td[owner[k].first].xmap_a = segs[k].out;
        else td[owner[k].first].xmap_z = segs[k].out;
    }
    return ASDM_OK;
}

int build_tails(const std::vector<const asdm_cs *> &cs, const std::vector<const asdm_plan *> &plans,
                std::vector<TailData> &out, unsigned long long **d_ps, cudaStream_t s) {
    *d_ps = nullptr;
    out.assign(cs.size(), TailData{});
    std::vector<TailSeg> segs;
    std::vector<size_t> seg_of;
    unsigned long long total = 0;
    for (size_t i = 0; i < cs.size(); ++i) {
        const asdm_cs &c = *cs[i];
        const asdm_plan &p = *plans[i];
        const uint32_t m = tail_mode(p);
        if (m == kTailNone) continue;
        const size_t n = p.order.size();
        if (m != kTailChain) {
            out[i].mode = m;
            continue;
        }
        const uint32_t e1 = p.back[n - 2][0].second, e2 = p.back[n - 1][0].second;
        const uint32_t ua = p.order[n - 2], ub = p.order[n - 1];
        const int k = c.q.slot(ub, ua);
        if (k < 0) continue;
        const uint32_t er = c.q.off[ub] + (uint32_t)k;
        const unsigned long long len = c.etotal[e1];
        if (total + len > kTailSumCap) continue;  // element path for this plan
        segs.push_back(TailSeg{c.d_elist + c.elist_base[e1], c.d_eoff + c.eoff_base[e2], total, len});
        seg_of.push_back(i);
        out[i].mode = m;
        out[i].rev_off = c.d_eoff + c.eoff_base[er];
        out[i].rev_list = c.d_elist + c.elist_base[er];
        total += len;
    }
    if (segs.empty()) return ASDM_OK;
    TailSeg *d_seg = nullptr;
    uint32_t *d_lens = nullptr;
    int rc = ASDM_OK;
    do {
        if ((rc = dalloc(d_ps, total + 1, s))) break;
        if ((rc = dalloc(&d_seg, segs.size(), s))) break;
        if ((rc = dalloc(&d_lens, std::max<unsigned long long>(total, 1), s))) break;
        if (cudaMemcpyAsync(d_seg, segs.data(), segs.size() * sizeof(TailSeg), cudaMemcpyHostToDevice, s) !=
            cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "tail segment upload failed");
            break;
        }
        if (total) {
            const unsigned grid = (unsigned)std::min<unsigned long long>((total + 255) / 256, 148ull * 32);
            tail_lens<<<grid, 256, 0, s>>>(d_seg, (uint32_t)segs.size(), total, d_lens);
            ::asdm::count_launch();
            if (cudaGetLastError() != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "tail length kernel failed");
                break;
            }
        }
        rc = scan_exclusive_u32(d_lens, reinterpret_cast<uint64_t *>(*d_ps), total, true, s);
    } while (false);
    // the copy above reads a host vector: wait before it goes out of scope
    cudaStreamSynchronize(s);
    dfree(d_lens, s);
    dfree(d_seg, s);
    if (rc != ASDM_OK) {
        dfree(*d_ps, s);
        *d_ps = nullptr;
        for (auto &t : out) t = TailData{};
        return rc;
    }
    for (size_t k = 0; k < segs.size(); ++k) out[seg_of[k]].ps = *d_ps + segs[k].start;
    return ASDM_OK;
}

unsigned long long root_pairs(const asdm_cs &cs, const asdm_plan &plan) {
    return plan.order.size() == 1 ? cs.ncand[plan.order[0]] : cs.etotal[plan.back[1][0].second];
}

// Root tasks: blocks of consecutive (level-0, level-1) candidate pairs, about
// 64K blocks per query, between 1 and 65,536 pairs per block (a few dozen
// tasks per resident warp are enough: work donation splits heavy ranges, and
// every task costs an atomic on one shared counter).  `min_blk` raises the
// block size.
void root_blocks(const asdm_cs &cs, const asdm_plan &plan, unsigned long long &pairs, unsigned long long &blk,
                 unsigned long long &nblocks, unsigned long long min_blk = 1) {
    pairs = root_pairs(cs, plan);
    blk = std::min<unsigned long long>(65536, std::max<unsigned long long>(min_blk, pairs / 65536));
    nblocks = (pairs + blk - 1) / blk;
}

int run_plan(asdm_cs &cs, const asdm_plan &plan, const asdm_run_opts &opt, asdm_run_stats &st) {
    asdm_graph *G = cs.g;
    cudaStream_t s = G->stream;
    const QueryGraph &q = cs.q;
    const uint32_t n = q.n;
    const uint32_t mode = opt.mode & (ASDM_MODE_LOCAL | ASDM_MODE_EMBED);
    st = asdm_run_stats{};
    if (opt.local_counts && (mode & ASDM_MODE_LOCAL))
        std::fill(opt.local_counts, opt.local_counts + (uint64_t)G->d.n * n, 0ull);
    if (!cs.nonempty) return ASDM_OK;
    if (mode == ASDM_MODE_LOCAL && opt.local_counts && plan.order.size() == n && tree_countable(q)) {
        // conflict-free tree: counts and local counts from the tree program
        const uint64_t local_n = (uint64_t)G->d.n * n;
        unsigned long long *blk = nullptr;
        ASDM_TRY(dalloc(&blk, local_n, s));
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, s);
        std::vector<uint64_t> tc;
        std::vector<char> done;
        std::vector<unsigned long long *> blocks{blk};
        int trc = cudaMemsetAsync(blk, 0, local_n * sizeof(unsigned long long), s) == cudaSuccess
                      ? tree_counts(G, {&cs}, tc, done, &blocks)
                      : fail(ASDM_ERR_CUDA, "local-count reset failed");
        cudaEventRecord(t1, s);
        cudaEventSynchronize(t1);
        float tms = 0.f;
        cudaEventElapsedTime(&tms, t0, t1);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        if (trc == ASDM_OK && done[0] &&
            (cudaMemcpyAsync(opt.local_counts, blk, local_n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s) !=
                 cudaSuccess ||
             cudaStreamSynchronize(s) != cudaSuccess))
            trc = fail(ASDM_ERR_CUDA, "local-count readback failed");
        dfree(blk, s);
        cudaStreamSynchronize(s);
        if (trc != ASDM_OK) return trc;
        if (done[0]) {
            st.count = tc[0];
            st.kernel_ms = tms;
            if (opt.count_limit && st.count > opt.count_limit) return fail(ASDM_ERR_LIMIT, "count limit reached");
            return ASDM_OK;
        }
    }
    if (mode == ASDM_MODE_COUNT && plan.order.size() == n && tree_countable_conflicts(q)) {
        // tree: the tree program counts it (the enumeration below only when
        // the program overflows)
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, s);
        std::vector<uint64_t> tc;
        std::vector<char> done;
        const int trc = tree_counts(G, {&cs}, tc, done);
        cudaEventRecord(t1, s);
        cudaEventSynchronize(t1);
        float tms = 0.f;
        cudaEventElapsedTime(&tms, t0, t1);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        if (trc != ASDM_OK) return trc;
        if (done[0]) {
            st.count = tc[0];
            st.kernel_ms = tms;
            if (opt.count_limit && st.count > opt.count_limit) return fail(ASDM_ERR_LIMIT, "count limit reached");
            return ASDM_OK;
        }
    }
    if (plan.order.size() == n) {
        // a lower bound at or above 2^64 settles the query without enumeration
        // (in every mode: local counts or embeddings of such a query do not fit)
        std::vector<char> proven;
        ASDM_TRY(overflow_bounds(G, {&cs}, proven));
        if (proven[0]) return fail(ASDM_ERR_OVERFLOW, "match count exceeds 2^64-1 (shown by a lower bound)");
    }
    // device plan
    std::vector<DLevel> lv(n);
    std::vector<DBack> bk;
    std::vector<uint32_t> cf;
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t u = plan.order[k];
        lv[k].cand = cs.d_cand + cs.cand_base[u];
        lv[k].ncand = cs.ncand[u];
        lv[k].u = u;
        lv[k].nback = (uint32_t)plan.back[k].size();
        lv[k].back_first = (uint32_t)bk.size();
        for (auto &jb : plan.back[k]) {
            const uint32_t e = jb.second;
            bk.push_back(DBack{cs.d_eoff + cs.eoff_base[e], cs.d_elist + cs.elist_base[e], jb.first, 0});
        }
        lv[k].nconf = (uint32_t)plan.conf[k].size();
        lv[k].conf_first = (uint32_t)cf.size();
        cf.insert(cf.end(), plan.conf[k].begin(), plan.conf[k].end());
    }
    const uint32_t nb = (uint32_t)bk.size(), nc = (uint32_t)cf.size();
    const uint64_t pbytes = n * sizeof(DLevel) + nb * sizeof(DBack) + nc * sizeof(uint32_t);
    std::vector<uint8_t> hp(pbytes);
    std::memcpy(hp.data(), lv.data(), n * sizeof(DLevel));
    std::memcpy(hp.data() + n * sizeof(DLevel), bk.data(), nb * sizeof(DBack));
    std::memcpy(hp.data() + n * sizeof(DLevel) + nb * sizeof(DBack), cf.data(), nc * sizeof(uint32_t));
    uint8_t *d_plan = nullptr;
    unsigned long long *d_ctr = nullptr, *d_local = nullptr, *d_ps = nullptr;
    uint32_t *d_rows = nullptr, *d_queue = nullptr, *d_xmap = nullptr;
    unsigned long long *d_lw = nullptr;
    int rc = ASDM_OK;
    auto cleanup = [&]() {
        dfree(d_ps, s);
        dfree(d_xmap, s);
        dfree(d_lw, s);
        dfree(d_plan, s);
        dfree(d_ctr, s);
        dfree(d_local, s);
        dfree(d_rows, s);
        dfree(d_queue, s);
    };
    EnumArgs a{};
    uint64_t row_cap = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    do {
        if ((rc = dalloc(&d_plan, pbytes, s))) break;
        if ((rc = dalloc(&d_ctr, kCtrN, s))) break;
        if ((rc = dalloc(&d_queue, kQueueCap * kRecWords + 2 * kQueueCap, s))) break;
        queue_init<<<(unsigned)(kQueueCap / 256), 256, 0, s>>>(
            reinterpret_cast<unsigned long long *>(d_queue + kQueueCap * kRecWords));
        ::asdm::count_launch();
        if (cudaGetLastError() != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "queue reset failed");
            break;
        }
        if (cudaMemcpyAsync(d_plan, hp.data(), pbytes, cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemsetAsync(d_ctr, 0, kCtrN * sizeof(unsigned long long), s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "plan upload failed");
            break;
        }
        const uint64_t local_n = (uint64_t)G->d.n * n;
        if (mode & ASDM_MODE_LOCAL) {
            if ((rc = dalloc(&d_local, local_n, s))) break;
            if (cudaMemsetAsync(d_local, 0, local_n * sizeof(unsigned long long), s) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "memset failed");
                break;
            }
        }
        if (mode & ASDM_MODE_EMBED) {
            row_cap = opt.embeddings ? opt.emb_capacity : 0;
            if ((rc = dalloc(&d_rows, std::max<uint64_t>(row_cap, 1) * n, s))) break;
        }
        a.lv = reinterpret_cast<const DLevel *>(d_plan);
        a.bk = reinterpret_cast<const DBack *>(d_plan + n * sizeof(DLevel));
        a.conf = reinterpret_cast<const uint32_t *>(d_plan + n * sizeof(DLevel) + nb * sizeof(DBack));
        a.n = n;
        a.nb = nb;
        a.nc = nc;
        a.nq = n;
        root_blocks(cs, plan, a.pairs, a.blk, a.ntasks);
        a.ctr = d_ctr;
        a.local = d_local;
        a.rows = d_rows;
        a.row_cap = row_cap;
        a.queue = d_queue;
        a.qseq = reinterpret_cast<unsigned long long *>(d_queue + kQueueCap * kRecWords);
        a.limit_ns = opt.time_limit_s > 0 ? (uint64_t)(opt.time_limit_s * 1e9) : 0;
        a.count_limit = opt.count_limit;
        a.lane_leaf_max = G->tuning.lane_leaf_max;
        a.merge_ratio = G->tuning.merge_ratio;
        if (mode == ASDM_MODE_COUNT) {
            std::vector<TailData> td;
            if ((rc = build_tails({&cs}, {&plan}, td, &d_ps, s))) break;
            if ((rc = build_xmaps({&cs}, {&plan}, td, &d_xmap, s))) break;
            a.tail = td[0].mode;
            a.ps = td[0].ps;
            a.rev_off = td[0].rev_off;
            a.rev_list = td[0].rev_list;
            a.xmap_a = td[0].xmap_a;
            a.xmap_z = td[0].xmap_z;
        }
        if (mode == ASDM_MODE_LOCAL) {
            std::vector<unsigned long long *> lwv;
            if ((rc = leaf_weights({&cs}, {&plan}, lwv, &d_lw, s))) break;
            a.lw = lwv[0];
        }
        const uint32_t smem = 4u * (plan_words(n, nb, nc) + kWarps * warp_words(n, nb));
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, s);
        if (a.ntasks) {
            switch (mode) {
                case ASDM_MODE_COUNT: rc = launch<ASDM_MODE_COUNT>(a, smem, G->num_sms, s); break;
                case ASDM_MODE_LOCAL: rc = launch<ASDM_MODE_LOCAL>(a, smem, G->num_sms, s); break;
                case ASDM_MODE_EMBED: rc = launch<ASDM_MODE_EMBED>(a, smem, G->num_sms, s); break;
                default: rc = launch<ASDM_MODE_LOCAL | ASDM_MODE_EMBED>(a, smem, G->num_sms, s); break;
            }
            if (rc) break;
        }
        cudaEventRecord(e1, s);
        unsigned long long ctr[kCtrN];
        if (cudaMemcpyAsync(ctr, d_ctr, sizeof ctr, cudaMemcpyDeviceToHost, s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "counter readback failed");
            break;
        }
        cudaError_t se = cudaStreamSynchronize(s);
        if (se != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "enumeration kernel failed: %s", cudaGetErrorString(se));
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        st.kernel_ms = ms;
        st.tails_lane = ctr[kCtrTailLane];
        st.tails_warp = ctr[kCtrTailWarp];
        st.count = ctr[kCtrCount];
        st.intersections = ctr[kCtrInter];
        st.list_bytes = 4ull * ctr[kCtrElems];
        st.tasks = std::min<uint64_t>(ctr[kCtrTask], a.ntasks);  // claimed root tasks
        const uint32_t flags = (uint32_t)ctr[kCtrFlags];
        if (flags & kFlagOverflow) { rc = fail(ASDM_ERR_OVERFLOW, "match count exceeds 2^64-1"); break; }
        if (flags & kFlagTimeout) { rc = fail(ASDM_ERR_TIMEOUT, "time limit reached"); break; }
        if (flags & kFlagLimit) { rc = fail(ASDM_ERR_LIMIT, "count limit reached"); break; }
        if (a.lw && (rc = push_leaf_weights({&cs}, {&plan}, {a.lw}, {d_local}, G->num_sms, s))) break;
        if ((mode & ASDM_MODE_LOCAL) && opt.local_counts) {
            if (cudaMemcpyAsync(opt.local_counts, d_local, local_n * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "local-count readback failed");
                break;
            }
        }
        if (mode & ASDM_MODE_EMBED) {
            const uint64_t rows = ctr[kCtrRows];
            st.emb_rows = std::min<uint64_t>(rows, row_cap);
            if (rows > row_cap) {
                rc = fail(ASDM_ERR_CAPACITY, "%llu embeddings, buffer holds %llu", (unsigned long long)rows,
                          (unsigned long long)row_cap);
                break;
            }
            if (rows) {
                std::vector<uint32_t> tmp(rows * n);
                if (cudaMemcpyAsync(tmp.data(), d_rows, rows * n * sizeof(uint32_t), cudaMemcpyDeviceToHost, s) !=
                        cudaSuccess ||
                    cudaStreamSynchronize(s) != cudaSuccess) {
                    rc = fail(ASDM_ERR_CUDA, "embedding readback failed");
                    break;
                }
                std::vector<uint64_t> perm(rows);
                std::iota(perm.begin(), perm.end(), 0ull);
                std::sort(perm.begin(), perm.end(), [&](uint64_t x, uint64_t y) {
                    return std::lexicographical_compare(tmp.begin() + x * n, tmp.begin() + x * n + n,
                                                        tmp.begin() + y * n, tmp.begin() + y * n + n);
                });
                for (uint64_t r = 0; r < rows; ++r)
                    std::memcpy(opt.embeddings + r * n, tmp.data() + perm[r] * n, n * sizeof(uint32_t));
            }
        }
    } while (false);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cleanup();
    cudaStreamSynchronize(s);
    return rc;
}


// Batched form: one persistent launch counts every query of a group.
// counts[i] / status[i] receive each query's result.
// Queries settled without enumeration, before any plan is needed: tree
// queries counted by the tree program (in LOCAL mode the conflict-free ones,
// with their local counts, a few queries at a time), then queries whose count
// a device lower bound shows to be at least 2^64 (ASDM_ERR_OVERFLOW).  Only
// queries with full[i] set (whole queries, not prefixes) take part.  live
// holds the positions still open on entry and on return; counts and status of
// the settled ones are written, their device time is added to agg->kernel_ms.
int settle_queries(asdm_graph *G, const std::vector<asdm_cs *> &cs, const std::vector<char> &full,
                   std::vector<uint32_t> &live, uint64_t count_limit, uint64_t *counts, int *status,
                   asdm_run_stats *agg, uint64_t *const *local_out) {
    cudaStream_t s = G->stream;
    const uint32_t Q = (uint32_t)cs.size();
    if (live.empty()) return ASDM_OK;
    float tree_ms = 0.f;
    if (local_out) {
        std::vector<uint32_t> tid;
        for (uint32_t i : live)
            if (full[i] && tree_countable(cs[i]->q)) tid.push_back(i);
        std::vector<char> settled(Q, 0);
        cudaEvent_t t0, t1;
        cudaEventCreate(&t0);
        cudaEventCreate(&t1);
        cudaEventRecord(t0, s);
        int trc = ASDM_OK;
        for (size_t at = 0; at < tid.size() && trc == ASDM_OK;) {
            // up to 2 GiB of local-count blocks per round
            std::vector<asdm_cs *> tcs;
            std::vector<uint32_t> ids;
            uint64_t words = 0;
            for (; at < tid.size(); ++at) {
                const uint64_t need = (uint64_t)G->d.n * cs[tid[at]]->q.n;
                if (!ids.empty() && words + need > (1ull << 28)) break;
                tcs.push_back(cs[tid[at]]);
                ids.push_back(tid[at]);
                words += need;
            }
            unsigned long long *blk = nullptr;
            if ((trc = dalloc(&blk, words, s))) break;
            std::vector<unsigned long long *> blocks;
            uint64_t o = 0;
            for (uint32_t i : ids) {
                blocks.push_back(blk + o);
                o += (uint64_t)G->d.n * cs[i]->q.n;
            }
            std::vector<uint64_t> tc;
            std::vector<char> done;
            trc = cudaMemsetAsync(blk, 0, words * sizeof(unsigned long long), s) == cudaSuccess
                      ? tree_counts(G, tcs, tc, done, &blocks)
                      : fail(ASDM_ERR_CUDA, "local-count reset failed");
            for (size_t k = 0; k < ids.size() && trc == ASDM_OK; ++k) {
                if (!done[k]) continue;
                const uint32_t i = ids[k];
                if (local_out[i] &&
                    cudaMemcpyAsync(local_out[i], blocks[k], (uint64_t)G->d.n * cs[i]->q.n * sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, s) != cudaSuccess)
                    trc = fail(ASDM_ERR_CUDA, "local-count readback failed");
                settled[i] = 1;
                counts[i] = tc[k];
                if (count_limit && tc[k] > count_limit) status[i] = ASDM_ERR_LIMIT;
                if (agg) agg->count += tc[k];
            }
            if (cudaStreamSynchronize(s) != cudaSuccess && trc == ASDM_OK) trc = fail(ASDM_ERR_CUDA, "local-count readback failed");
            dfree(blk, s);
        }
        cudaEventRecord(t1, s);
        cudaEventSynchronize(t1);
        cudaEventElapsedTime(&tree_ms, t0, t1);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        if (trc != ASDM_OK) return trc;
        std::vector<uint32_t> rest;
        for (uint32_t i : live)
            if (!settled[i]) rest.push_back(i);
        live.swap(rest);
        if (agg) agg->kernel_ms += tree_ms;
        if (live.empty()) return ASDM_OK;
    }
    if (!local_out) {
        std::vector<asdm_cs *> tcs;
        std::vector<uint32_t> tid;
        for (uint32_t i : live)
            if (full[i] && tree_countable_conflicts(cs[i]->q)) {
                tcs.push_back(cs[i]);
                tid.push_back(i);
            }
        if (!tcs.empty()) {
            cudaEvent_t t0, t1;
            cudaEventCreate(&t0);
            cudaEventCreate(&t1);
            cudaEventRecord(t0, s);
            std::vector<uint64_t> tc;
            std::vector<char> done;
            const int trc = tree_counts(G, tcs, tc, done);
            cudaEventRecord(t1, s);
            cudaEventSynchronize(t1);
            cudaEventElapsedTime(&tree_ms, t0, t1);
            cudaEventDestroy(t0);
            cudaEventDestroy(t1);
            if (trc != ASDM_OK) return trc;
            std::vector<char> settled(Q, 0);
            for (size_t k = 0; k < tid.size(); ++k)
                if (done[k]) {
                    const uint32_t i = tid[k];
                    settled[i] = 1;
                    counts[i] = tc[k];
                    if (count_limit && tc[k] > count_limit) status[i] = ASDM_ERR_LIMIT;
                    if (agg) agg->count += tc[k];
                }
            std::vector<uint32_t> rest;
            for (uint32_t i : live)
                if (!settled[i]) rest.push_back(i);
            live.swap(rest);
            if (agg) agg->kernel_ms += tree_ms;
            if (live.empty()) return ASDM_OK;
        }
    }
    {
        // queries whose count a lower bound shows to be at least 2^64 are
        // settled as overflows (in LOCAL mode too: their matrices would have
        // a column summing past 2^64 - 1)
        std::vector<asdm_cs *> ocs;
        std::vector<uint32_t> oid;
        for (uint32_t i : live)
            if (full[i]) {
                ocs.push_back(cs[i]);
                oid.push_back(i);
            }
        if (!ocs.empty()) {
            cudaEvent_t t0, t1;
            cudaEventCreate(&t0);
            cudaEventCreate(&t1);
            cudaEventRecord(t0, G->stream);
            std::vector<char> proven;
            const int brc = overflow_bounds(G, ocs, proven);
            cudaEventRecord(t1, G->stream);
            cudaEventSynchronize(t1);
            float bms = 0.f;
            cudaEventElapsedTime(&bms, t0, t1);
            cudaEventDestroy(t0);
            cudaEventDestroy(t1);
            if (brc != ASDM_OK) return brc;
            std::vector<char> settled(Q, 0);
            for (size_t k = 0; k < oid.size(); ++k)
                if (proven[k]) {
                    settled[oid[k]] = 1;
                    counts[oid[k]] = 0;
                    status[oid[k]] = ASDM_ERR_OVERFLOW;
                }
            std::vector<uint32_t> rest;
            for (uint32_t i : live)
                if (!settled[i]) rest.push_back(i);
            live.swap(rest);
            if (agg) agg->kernel_ms += bms;
            if (live.empty()) return ASDM_OK;
        }
    }
    return ASDM_OK;
}

int run_batch_count(asdm_graph *G, const std::vector<asdm_cs *> &cs, const std::vector<const asdm_plan *> &plans,
                    double time_limit_s, uint64_t count_limit, uint64_t *counts, int *status, asdm_run_stats *agg,
                    uint64_t *const *local_out, uint64_t *cycles, double query_time_s, bool settled) {
    cudaStream_t s = G->stream;
    const uint32_t Q = (uint32_t)cs.size();
    std::vector<uint32_t> live;  // queries with a non-empty candidate space
    for (uint32_t i = 0; i < Q; ++i) {
        counts[i] = 0;
        status[i] = ASDM_OK;
        if (cycles) cycles[i] = 0;
        if (cs[i]->nonempty) live.push_back(i);
    }
    if (agg) *agg = asdm_run_stats{};
    if (live.empty()) return ASDM_OK;
    if (!settled) {
        std::vector<char> full(Q, 0);
        for (uint32_t i = 0; i < Q; ++i) full[i] = plans[i]->order.size() == cs[i]->q.n;
        ASDM_TRY(settle_queries(G, cs, full, live, count_limit, counts, status, agg, local_out));
        if (live.empty()) return ASDM_OK;
    }
    const uint32_t L = (uint32_t)live.size();
    // host images of all plans, then one upload
    std::vector<uint8_t> hp;
    struct Off { uint64_t lv, bk, cf; };
    std::vector<Off> offs(L);
    std::vector<QDesc> qd(L);
    std::vector<unsigned long long> task_pre(L + 1, 0);
    uint32_t maxn = 1, maxnb = 1;
    // Root blocks of "light" plans (at most 4 levels with a closed-form tail:
    // every pair then costs O(1)) hold at least root_block_min pairs, which
    // saves per-task overhead; other plans keep fine blocks, which balance
    // heavy subtrees.
    const unsigned long long light_blk = std::max<uint32_t>(1, G->tuning.root_block_min);
    auto append = [&](const void *src, size_t bytes) {
        const uint64_t at = (hp.size() + 15) & ~15ull;
        hp.resize(at + bytes);
        if (bytes && src) std::memcpy(hp.data() + at, src, bytes);
        return at;
    };
    for (uint32_t li = 0; li < L; ++li) {
        const asdm_cs &c = *cs[live[li]];
        const asdm_plan &plan = *plans[live[li]];
        const uint32_t n = (uint32_t)plan.order.size();  // q.n, or a prefix's depth
        std::vector<DLevel> lv(n);
        std::vector<DBack> bk;
        std::vector<uint32_t> cf;
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t u = plan.order[k];
            lv[k].cand = c.d_cand + c.cand_base[u];
            lv[k].ncand = c.ncand[u];
            lv[k].u = u;
            lv[k].nback = (uint32_t)plan.back[k].size();
            lv[k].back_first = (uint32_t)bk.size();
            for (auto &jb : plan.back[k])
                bk.push_back(DBack{c.d_eoff + c.eoff_base[jb.second], c.d_elist + c.elist_base[jb.second], jb.first, 0});
            lv[k].nconf = (uint32_t)plan.conf[k].size();
            lv[k].conf_first = (uint32_t)cf.size();
            cf.insert(cf.end(), plan.conf[k].begin(), plan.conf[k].end());
        }
        offs[li].lv = append(lv.data(), lv.size() * sizeof(DLevel));
        offs[li].bk = append(bk.data(), bk.size() * sizeof(DBack));
        offs[li].cf = append(cf.data(), cf.size() * sizeof(uint32_t));
        qd[li].n = n;
        qd[li].nb = (uint32_t)bk.size();
        qd[li].nc = (uint32_t)cf.size();
        unsigned long long nt = 0;
        const uint32_t tm = tail_mode(plan);
        const bool light = local_out == nullptr && n <= 4 && (tm == kTailChain || tm == kTailLeaf);
        root_blocks(c, plan, qd[li].pairs, qd[li].blk, nt, light ? light_blk : 1);
        task_pre[li + 1] = task_pre[li] + nt;
        maxn = std::max(maxn, n);
        maxnb = std::max(maxnb, (uint32_t)bk.size());
    }
    const uint64_t qd_at = append(nullptr, L * sizeof(QDesc));
    const uint64_t tp_at = append(task_pre.data(), task_pre.size() * sizeof(unsigned long long));
    uint8_t *d_buf = nullptr;
    unsigned long long *d_ctr = nullptr, *d_qcounts = nullptr, *d_local = nullptr, *d_ps = nullptr, *d_cyc = nullptr;
    unsigned long long *d_qwork = nullptr;
    uint32_t *d_queue = nullptr, *d_xmap = nullptr;
    unsigned long long *d_lw = nullptr;
    std::vector<unsigned long long *> lwv;
    unsigned int *d_qflags = nullptr;
    int rc = ASDM_OK;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    // local counts (LOCAL mode): one |Vg| x n block per live query
    const bool local_mode = local_out != nullptr;
    std::vector<uint64_t> local_base(L + 1, 0);
    for (uint32_t li = 0; li < L; ++li)
        local_base[li + 1] = local_base[li] + (local_mode ? (uint64_t)G->d.n * cs[live[li]]->q.n : 0);
    do {
        if (local_mode) {
            if ((rc = dalloc(&d_local, local_base[L], s))) break;
            if (cudaMemsetAsync(d_local, 0, local_base[L] * sizeof(unsigned long long), s) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "local-count reset failed");
                break;
            }
        }
        if ((rc = dalloc(&d_buf, hp.size(), s)) || (rc = dalloc(&d_ctr, kCtrN, s)) ||
            (rc = dalloc(&d_qcounts, 2ull * L, s)) || (rc = dalloc(&d_qflags, L, s)) ||
            (rc = dalloc(&d_queue, kQueueCap * kRecWords + 2 * kQueueCap, s)))
            break;
        d_qwork = d_qcounts + L;
        if (!local_mode) {
            std::vector<const asdm_cs *> tcs(L);
            std::vector<const asdm_plan *> tpl(L);
            for (uint32_t li = 0; li < L; ++li) {
                tcs[li] = cs[live[li]];
                tpl[li] = plans[live[li]];
            }
            std::vector<TailData> td;
            if ((rc = build_tails(tcs, tpl, td, &d_ps, s))) break;
            if ((rc = build_xmaps(tcs, tpl, td, &d_xmap, s))) break;
            for (uint32_t li = 0; li < L; ++li) {
                qd[li].tail = td[li].mode;
                qd[li].ps = td[li].ps;
                qd[li].rev_off = td[li].rev_off;
                qd[li].rev_list = td[li].rev_list;
                qd[li].xmap_a = td[li].xmap_a;
                qd[li].xmap_z = td[li].xmap_z;
            }
        }
        if (local_mode) {
            std::vector<const asdm_cs *> tcs(L);
            std::vector<const asdm_plan *> tpl(L);
            for (uint32_t li = 0; li < L; ++li) {
                tcs[li] = cs[live[li]];
                tpl[li] = plans[live[li]];
            }
            if ((rc = leaf_weights(tcs, tpl, lwv, &d_lw, s))) break;
            for (uint32_t li = 0; li < L; ++li) qd[li].lw = lwv[li];
        }
        for (uint32_t li = 0; li < L; ++li) {
            qd[li].lv = reinterpret_cast<const DLevel *>(d_buf + offs[li].lv);
            qd[li].bk = reinterpret_cast<const DBack *>(d_buf + offs[li].bk);
            qd[li].conf = reinterpret_cast<const uint32_t *>(d_buf + offs[li].cf);
            qd[li].local = local_mode ? d_local + local_base[li] : nullptr;
        }
        std::memcpy(hp.data() + qd_at, qd.data(), L * sizeof(QDesc));
        if (cudaMemcpyAsync(d_buf, hp.data(), hp.size(), cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaMemsetAsync(d_ctr, 0, kCtrN * sizeof(unsigned long long), s) != cudaSuccess ||
            cudaMemsetAsync(d_qcounts, 0, 2ull * L * sizeof(unsigned long long), s) != cudaSuccess ||
            cudaMemsetAsync(d_qflags, 0, L * sizeof(unsigned int), s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "batch upload failed");
            break;
        }
        unsigned long long *d_seq = reinterpret_cast<unsigned long long *>(d_queue + kQueueCap * kRecWords);
        queue_init<<<(unsigned)(kQueueCap / 256), 256, 0, s>>>(d_seq);
        ::asdm::count_launch();
        EnumArgs a{};
        a.ctr = d_ctr;
        a.queue = d_queue;
        a.qseq = d_seq;
        a.qd = reinterpret_cast<const QDesc *>(d_buf + qd_at);
        a.task_pre = reinterpret_cast<const unsigned long long *>(d_buf + tp_at);
        a.nquery = L;
        a.maxn = maxn;
        a.maxnb = maxnb;
        a.qcounts = d_qcounts;
        a.qflags = d_qflags;
        a.qwork = d_qwork;
        if (cycles) {
            if ((rc = dalloc(&d_cyc, L, s))) break;
            if (cudaMemsetAsync(d_cyc, 0, L * sizeof(unsigned long long), s) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "cycle counter reset failed");
                break;
            }
            a.qcycles = d_cyc;
        }
        a.limit_ns = time_limit_s > 0 ? (uint64_t)(time_limit_s * 1e9) : 0;
        a.count_limit = count_limit;
        const uint32_t smem = 4u * kWarps * warp_words(maxn, maxnb);
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, s);
        a.lane_leaf_max = G->tuning.lane_leaf_max;
        a.merge_ratio = G->tuning.merge_ratio;
        if (task_pre[L]) {
            // register-budget variant chosen by the tuner (min blocks per SM)
            void (*k)(EnumArgs) = enum_batch_kernel<1>;
            switch (G->tuning.enum_min_blocks) {
                case 2: k = enum_batch_kernel<2>; break;
                case 3: k = enum_batch_kernel<3>; break;
                case 4: k = enum_batch_kernel<4>; break;
                case 5: k = enum_batch_kernel<5>; break;
                case 6: k = enum_batch_kernel<6>; break;
                default: break;
            }
            if (local_mode) k = enum_batch_kernel<1, ASDM_MODE_LOCAL>;
            if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "shared-memory opt-in failed");
                break;
            }
            int per_sm = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kThreads, smem);
            if (per_sm <= 0) {
                rc = fail(ASDM_ERR_INVALID, "batch plans too large for shared memory (%u bytes)", smem);
                break;
            }
            // a query's budget: its time alone on the GPU, as warp-time over every resident warp
            if (query_time_s > 0)
                a.q_budget_ns = (unsigned long long)(query_time_s * 1e9 * (double)per_sm * G->num_sms * kWarps);
            k<<<(unsigned)(per_sm * G->num_sms), kThreads, smem, s>>>(a);
            ::asdm::count_launch();
            if (cudaGetLastError() != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "batch kernel launch failed");
                break;
            }
        }
        cudaEventRecord(e1, s);
        unsigned long long ctr[kCtrN];
        std::vector<unsigned long long> qc(2ull * L);  // counts, then warp-time charged
        std::vector<unsigned int> qf(L);
        if (cudaMemcpyAsync(ctr, d_ctr, sizeof ctr, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(qc.data(), d_qcounts, 2ull * L * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(qf.data(), d_qflags, L * sizeof(unsigned int), cudaMemcpyDeviceToHost, s) != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "batch readback failed");
            break;
        }
        cudaError_t se = cudaStreamSynchronize(s);
        if (se != cudaSuccess) {
            rc = fail(ASDM_ERR_CUDA, "batch kernel failed: %s", cudaGetErrorString(se));
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (cycles) {
            std::vector<unsigned long long> cy(L);
            if (cudaMemcpyAsync(cy.data(), d_cyc, L * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s) !=
                    cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                rc = fail(ASDM_ERR_CUDA, "cycle readback failed");
                break;
            }
            for (uint32_t li = 0; li < L; ++li) cycles[live[li]] = cy[li];
        }
        const uint32_t gflags = (uint32_t)ctr[kCtrFlags];
        for (uint32_t li = 0; li < L; ++li) {
            const uint32_t i = live[li];
            counts[i] = qc[li];
            // a proven overflow outranks a stop; a count limit reached is final too
            if (qf[li] & kFlagOverflow) status[i] = ASDM_ERR_OVERFLOW;
            else if (qf[li] & kFlagLimit) status[i] = ASDM_ERR_LIMIT;
            else if ((gflags | qf[li]) & kFlagTimeout) status[i] = ASDM_ERR_TIMEOUT;
        }
        if (agg) {
            agg->count += ctr[kCtrCount];
            agg->intersections = ctr[kCtrInter];
            agg->list_bytes = 4ull * ctr[kCtrElems];
            agg->tasks = task_pre[L];
            agg->kernel_ms += ms;
            agg->tails_lane = ctr[kCtrTailLane];
            agg->tails_warp = ctr[kCtrTailWarp];
            double busy = 0.0;
            for (uint32_t li = 0; li < L; ++li) busy += (double)qc[L + li];
            agg->busy_warp_ms += busy * 1e-6;
            agg->idle_warp_ms += (double)ctr[kCtrIdleNs] * 1e-6;
        }
        if (gflags & kFlagTimeout) rc = fail(ASDM_ERR_TIMEOUT, "time limit reached");
        if (rc == ASDM_OK && local_mode && d_lw) {
            std::vector<const asdm_cs *> tcs(L);
            std::vector<const asdm_plan *> tpl(L);
            std::vector<unsigned long long *> blocks(L);
            for (uint32_t li = 0; li < L; ++li) {
                tcs[li] = cs[live[li]];
                tpl[li] = plans[live[li]];
                blocks[li] = d_local + local_base[li];
            }
            rc = push_leaf_weights(tcs, tpl, lwv, blocks, G->num_sms, s);
        }
        if (rc == ASDM_OK && local_mode) {
            for (uint32_t li = 0; li < L && rc == ASDM_OK; ++li)
                if (local_out[live[li]] &&
                    cudaMemcpyAsync(local_out[live[li]], d_local + local_base[li],
                                    (local_base[li + 1] - local_base[li]) * sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, s) != cudaSuccess)
                    rc = fail(ASDM_ERR_CUDA, "local-count readback failed");
            if (rc == ASDM_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = fail(ASDM_ERR_CUDA, "local-count readback failed");
        }
    } while (false);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    dfree(d_ps, s);
    dfree(d_xmap, s);
    dfree(d_lw, s);
    dfree(d_cyc, s);
    dfree(d_buf, s);
    dfree(d_ctr, s);
    dfree(d_qcounts, s);
    dfree(d_qflags, s);
    dfree(d_queue, s);
    dfree(d_local, s);
    cudaStreamSynchronize(s);
    return rc;
}

}  // namespace asdm

using namespace asdm;

extern "C" int asdm_run_plan(asdm_cs *cs, const asdm_plan *plan, const asdm_run_opts *opts, asdm_run_stats *stats) {
    clear_error();
    if (!cs || !opts) return fail(ASDM_ERR_INVALID, "null argument");
    asdm_run_stats local_stats{};
    asdm_run_stats &st = stats ? *stats : local_stats;
    if ((opts->mode & ASDM_MODE_EMBED) && !opts->embeddings && opts->emb_capacity)
        return fail(ASDM_ERR_INVALID, "embedding buffer is null");
    if (!cs->nonempty) {
        st = asdm_run_stats{};
        if (opts->local_counts && (opts->mode & ASDM_MODE_LOCAL))
            std::fill(opts->local_counts, opts->local_counts + (uint64_t)cs->g->d.n * cs->q.n, 0ull);
        return ASDM_OK;
    }
    if (!plan) return fail(ASDM_ERR_INVALID, "null plan");
    if (plan->order.size() != cs->q.n) return fail(ASDM_ERR_INVALID, "plan does not match the query");
    return run_plan(*cs, *plan, *opts, st);
}

extern "C" int asdm_count_query(asdm_graph *g, const uint32_t *q_offsets, const uint32_t *q_nbrs,
                                const uint32_t *q_labels, uint32_t q_n, const asdm_run_opts *opts,
                                asdm_run_stats *stats) {
    clear_error();
    if (!g || !opts) return fail(ASDM_ERR_INVALID, "null argument");
    asdm_cs *cs = nullptr;
    int nonempty = 0;
    ASDM_TRY(asdm_candidate_space(g, q_offsets, q_nbrs, q_labels, q_n, &cs, &nonempty));
    asdm_plan *plan = nullptr;
    int rc = ASDM_OK;
    if (nonempty) rc = asdm_plan_create(cs, nullptr, &plan);
    if (rc == ASDM_OK) rc = asdm_run_plan(cs, plan, opts, stats);
    asdm_plan_free(plan);
    asdm_cs_free(cs);
    return rc;
}

extern "C" int asdm_cs_count_lower_bound(asdm_cs *cs, uint64_t *lower, int *exceeds) {
    clear_error();
    if (!cs || !lower || !exceeds) return fail(ASDM_ERR_INVALID, "null argument");
    *lower = 0;
    *exceeds = 0;
    if (!cs->nonempty) return ASDM_OK;
    std::vector<char> proven;
    std::vector<uint64_t> lb;
    ASDM_TRY(overflow_bounds(cs->g, {cs}, proven, &lb));
    *lower = lb[0];
    *exceeds = proven[0] ? 1 : 0;
    return ASDM_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free counting.
//
// Some callers cannot let a library allocate device memory while they run:
// a serving process whose GPU memory is entirely reserved up front by its own
// pool allocator (a cudaMalloc there can fail or push a co-tenant out of
// memory), or a latency-critical loop where cudaMalloc/cudaFree would add
// implicit device synchronisation.  asdm_run_plan_count_noalloc serves them:
// it runs the same COUNT-mode enumeration kernel as asdm_run_plan, but its
// scratch (the run counters, the device copy of the plan and the
// work-donation ring) lives in the fixed, file-scope device array below.
// The caller still passes the inputs (a candidate space and a plan) and the
// output (the stats struct).
//
// The array is kNoAllocScratchBytes (about 10 MiB) on every GPU that loads
// this library, held until the process exits.  Its host-side name is only a
// stand-in for the device symbol, so the device address is fetched with
// cudaGetSymbolAddress once per device (with that device current) by the
// first call made on that device; make that first call before any stream
// capture.  All calls share the one array and it keeps the last call's
// contents: every call re-zeroes the counters and re-initialises the ring
// before its launch.  Calls that overlap on the GPU (from several host
// threads or several streams) race on the array and must be serialised by
// the caller.
namespace asdm {
namespace {

constexpr uint64_t kNoAllocCtrBytes = 256;
constexpr uint64_t kNoAllocPlanBytes = 16384;  // >= 32 levels + 496 back edges + 496 conflict levels
constexpr uint64_t kNoAllocSeqBytes = kQueueCap * sizeof(unsigned long long);
constexpr uint64_t kNoAllocRingBytes = kQueueCap * kRecWords * sizeof(uint32_t);
constexpr uint64_t kNoAllocScratchBytes = kNoAllocCtrBytes + kNoAllocPlanBytes + kNoAllocSeqBytes + kNoAllocRingBytes;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
unsigned char *g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device (set up once).
int noalloc_scratch(int device, unsigned char **out) {
    if (device < 0 || device >= kNoAllocMaxDevices) return fail(ASDM_ERR_INVALID, "device %d out of range", device);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return fail(ASDM_ERR_CUDA, "cudaGetSymbolAddress of the no-alloc scratch failed: %s", cudaGetErrorString(e));
        g_noalloc_ptr[device] = static_cast<unsigned char *>(p);
    }
    *out = g_noalloc_ptr[device];
    return ASDM_OK;
}

}  // namespace
}  // namespace asdm

extern "C" int asdm_run_plan_count_noalloc(asdm_cs *cs, const asdm_plan *plan, double time_limit_s,
                                           uint64_t count_limit, asdm_run_stats *stats) {
    using namespace asdm;
    clear_error();
    if (!cs || !stats) return fail(ASDM_ERR_INVALID, "null argument");
    *stats = asdm_run_stats{};
    if (!cs->nonempty) return ASDM_OK;
    if (!plan || plan->order.size() != cs->q.n) return fail(ASDM_ERR_INVALID, "plan does not match the query");
    asdm_graph *G = cs->g;
    cudaStream_t s = G->stream;
    const uint32_t n = cs->q.n;
    // host image of the device plan (same layout as asdm_run_plan's)
    std::vector<DLevel> lv(n);
    std::vector<DBack> bk;
    std::vector<uint32_t> cf;
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t u = plan->order[k];
        lv[k].cand = cs->d_cand + cs->cand_base[u];
        lv[k].ncand = cs->ncand[u];
        lv[k].u = u;
        lv[k].nback = (uint32_t)plan->back[k].size();
        lv[k].back_first = (uint32_t)bk.size();
        for (auto &jb : plan->back[k])
            bk.push_back(DBack{cs->d_eoff + cs->eoff_base[jb.second], cs->d_elist + cs->elist_base[jb.second], jb.first, 0});
        lv[k].nconf = (uint32_t)plan->conf[k].size();
        lv[k].conf_first = (uint32_t)cf.size();
        cf.insert(cf.end(), plan->conf[k].begin(), plan->conf[k].end());
    }
    const uint32_t nb = (uint32_t)bk.size(), nc = (uint32_t)cf.size();
    const uint64_t pbytes = n * sizeof(DLevel) + nb * sizeof(DBack) + nc * sizeof(uint32_t);
    if (pbytes > kNoAllocPlanBytes)
        return fail(ASDM_ERR_INVALID, "plan needs %llu bytes; the no-alloc scratch holds %llu",
                    (unsigned long long)pbytes, (unsigned long long)kNoAllocPlanBytes);
    std::vector<uint8_t> hp(pbytes);
    std::memcpy(hp.data(), lv.data(), n * sizeof(DLevel));
    std::memcpy(hp.data() + n * sizeof(DLevel), bk.data(), nb * sizeof(DBack));
    std::memcpy(hp.data() + n * sizeof(DLevel) + nb * sizeof(DBack), cf.data(), nc * sizeof(uint32_t));

    int current = -1;
    ASDM_CUDA(cudaGetDevice(&current));
    if (current != G->device)
        return fail(ASDM_ERR_INVALID, "call with the graph's device (%d) current, not %d", G->device, current);
    unsigned char *base = nullptr;
    ASDM_TRY(noalloc_scratch(G->device, &base));
    unsigned long long *d_ctr = reinterpret_cast<unsigned long long *>(base);
    uint8_t *d_plan = base + kNoAllocCtrBytes;
    unsigned long long *d_seq = reinterpret_cast<unsigned long long *>(base + kNoAllocCtrBytes + kNoAllocPlanBytes);
    uint32_t *d_ring = reinterpret_cast<uint32_t *>(base + kNoAllocCtrBytes + kNoAllocPlanBytes + kNoAllocSeqBytes);

    ASDM_CUDA(cudaMemcpyAsync(d_plan, hp.data(), pbytes, cudaMemcpyHostToDevice, s));
    ASDM_CUDA(cudaMemsetAsync(d_ctr, 0, kCtrN * sizeof(unsigned long long), s));
    queue_init<<<(unsigned)(kQueueCap / 256), 256, 0, s>>>(d_seq);
    ::asdm::count_launch();
    ASDM_CUDA(cudaGetLastError());

    EnumArgs a{};
    a.lv = reinterpret_cast<const DLevel *>(d_plan);
    a.bk = reinterpret_cast<const DBack *>(d_plan + n * sizeof(DLevel));
    a.conf = reinterpret_cast<const uint32_t *>(d_plan + n * sizeof(DLevel) + nb * sizeof(DBack));
    a.n = n;
    a.nb = nb;
    a.nc = nc;
    a.nq = n;
    root_blocks(*cs, *plan, a.pairs, a.blk, a.ntasks);
    a.ctr = d_ctr;
    a.queue = d_ring;
    a.qseq = d_seq;
    a.limit_ns = time_limit_s > 0 ? (uint64_t)(time_limit_s * 1e9) : 0;
    a.count_limit = count_limit;
    a.lane_leaf_max = G->tuning.lane_leaf_max;
    a.merge_ratio = G->tuning.merge_ratio;
    if (a.ntasks) {
        const uint32_t smem = 4u * (plan_words(n, nb, nc) + kWarps * warp_words(n, nb));
        ASDM_TRY(launch<ASDM_MODE_COUNT>(a, smem, G->num_sms, s));
    }
    unsigned long long ctr[kCtrN];
    ASDM_CUDA(cudaMemcpyAsync(ctr, d_ctr, sizeof ctr, cudaMemcpyDeviceToHost, s));
    ASDM_CUDA(cudaStreamSynchronize(s));
    stats->count = ctr[kCtrCount];
    stats->intersections = ctr[kCtrInter];
    stats->list_bytes = 4ull * ctr[kCtrElems];
    stats->tasks = std::min<uint64_t>(ctr[kCtrTask], a.ntasks);
    const uint32_t flags = (uint32_t)ctr[kCtrFlags];
    if (flags & kFlagOverflow) return fail(ASDM_ERR_OVERFLOW, "match count exceeds 2^64-1");
    if (flags & kFlagTimeout) return fail(ASDM_ERR_TIMEOUT, "time limit reached");
    if (flags & kFlagLimit) return fail(ASDM_ERR_LIMIT, "count limit reached");
    return ASDM_OK;
}
