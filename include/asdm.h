/*
 * asdm.h — C ABI of the B200 matching and counting engine (libasdm_b200.so).
 *
 * Drop-in boundary for ASDMatch's matching and counting path.  Every entry
 * point is extern "C", takes plain pointers and sizes, returns an int status
 * (ASDM_OK = 0) and never traps; asdm_last_error() gives a one-line reason for
 * the calling thread's last failure.  Handles are opaque.  Host buffers are
 * owned by the caller; device memory is owned by the library.
 *
 * Each declaration names the reference interface it replaces
 * (path:line inside the reference project magic62442/ASDMatch).
 */
#ifndef ASDM_H
#define ASDM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define ASDM_OK 0
#define ASDM_ERR_INVALID 1   /* bad argument or malformed graph               */
#define ASDM_ERR_IO 2        /* file cannot be opened ("Can not open file")   */
#define ASDM_ERR_CUDA 3      /* CUDA runtime error (no device, launch error)  */
#define ASDM_ERR_OOM 4       /* device allocation failed or budget exceeded   */
#define ASDM_ERR_OVERFLOW 5  /* a uint64 count or local count overflowed      */
#define ASDM_ERR_TIMEOUT 6   /* the run's time limit was reached              */
#define ASDM_ERR_CAPACITY 7  /* embedding buffer smaller than the match count */
#define ASDM_ERR_INTERNAL 8  /* device-side consistency check failed          */
#define ASDM_ERR_LIMIT 9     /* the run's count limit was reached             */

/* ---- run modes (bit mask); the reference selects these at compile time
 *      with ALL_LEVEL / LOCAL_COUNT / COLLECT_RESULT (config/config.h:38-40) */
#define ASDM_MODE_COUNT 0u   /* exact uint64 count (ALL_LEVEL)                 */
#define ASDM_MODE_LOCAL 1u   /* + |Vg| x |Vq| local counts (LOCAL_COUNT)       */
#define ASDM_MODE_EMBED 2u   /* + the embeddings themselves (COLLECT_RESULT)   */

typedef struct asdm_host_graph asdm_host_graph; /* host CSR, reference layout  */
typedef struct asdm_graph asdm_graph;           /* device-resident data graph  */
typedef struct asdm_cs asdm_cs;                 /* device candidate space      */
typedef struct asdm_plan asdm_plan;             /* matching order + level info */
typedef struct asdm_card asdm_card;             /* .card cardinality cache     */
typedef struct asdm_estimator asdm_estimator;   /* learned cardinality model   */

/* Returns a static, thread-local description of the last failure. */
const char *asdm_last_error(void);
/* Library version string. */
const char *asdm_version(void);
/* Number of kernels the library has launched since it was loaded (all
 * threads); lets callers count the device work of a region.  No reference
 * counterpart (the reference runs on the CPU). */
uint64_t asdm_kernel_launches(void);

/* ---- host graphs ------------------------------------------------------- */

/* Replaces Graph::loadGraphFromTextFile (relation/graph.cpp:68-148): 't N M'
 * header, 'v id label degree' (degree fixes the CSR offsets), 'e a b' edges,
 * other tokens skipped; neighbours sorted by (label, id). ASDM_ERR_IO if the
 * file cannot be opened. */
int asdm_host_graph_load(const char *path, asdm_host_graph **out);
/* Builds a host graph from an undirected edge list (edges[2*i], edges[2*i+1]);
 * same layout as the loader. Replaces nothing (synthetic inputs). */
int asdm_host_graph_from_edges(uint32_t n, const uint32_t *labels, uint64_t m,
                               const uint32_t *edges, asdm_host_graph **out);
/* Size queries and zero-copy views of the CSR (offsets[n+1], nbrs[m2],
 * labels[n]); the views live as long as the graph (relation/graph.h:58-104). */
int asdm_host_graph_info(const asdm_host_graph *g, uint32_t *n, uint64_t *m2, uint32_t *nlabels);
int asdm_host_graph_csr(const asdm_host_graph *g, const uint32_t **offsets, const uint32_t **nbrs,
                        const uint32_t **labels);
/* Writes the graph in 't/v/e' text (Graph::writeToTextFile, relation/graph.h:157). */
int asdm_host_graph_write(const asdm_host_graph *g, const char *path);
/* The reference's binary graph cache (Graph::writeToStream / readFromStream,
 * relation/graph.cpp:293-332): byte-identical to what the reference writes
 * for the same graph; the reader keeps CSR and labels. */
int asdm_host_graph_write_binary(const asdm_host_graph *g, const char *path);
int asdm_host_graph_load_binary(const char *path, asdm_host_graph **out);
void asdm_host_graph_free(asdm_host_graph *g);

/* Seeded Chung-Lu power-law graph: weights (i+i0)^(-1/(gamma-1)) with i0 set so
 * that the largest weight is sqrt(2m), endpoint pairs drawn by weight until m
 * distinct non-loop edges exist, labels i.i.d. Zipf(zipf_s) over nlabels,
 * vertex ids randomly permuted.  No reference counterpart (synthetic input). */
int asdm_gen_chung_lu(uint32_t n, uint64_t m, double gamma, uint32_t nlabels, double zipf_s,
                      uint64_t seed, asdm_host_graph **out);
/* Same with the largest expected degree set to wmax instead of sqrt(2m)
 * (wmax <= 0 keeps sqrt(2m)). */
int asdm_gen_chung_lu_capped(uint32_t n, uint64_t m, double gamma, uint32_t nlabels, double zipf_s,
                             double wmax, uint64_t seed, asdm_host_graph **out);
/* Connected query by random walk with restart from a seeded data vertex: the
 * induced subgraph on the first `size` distinct vertices, labels copied.
 * density: 0 any, 1 dense (average degree >= 3), 2 sparse (< 3).  No
 * reference counterpart (the reference ships its query sets as files). */
int asdm_gen_query(const asdm_host_graph *g, uint32_t size, int density, uint64_t seed,
                   asdm_host_graph **out);

/* ---- device data graph ------------------------------------------------- */

/* Uploads a CSR data graph whose neighbour lists are sorted by (label, id)
 * (the loader's layout) and builds the label index on the device.  Replaces
 * the data-side Graph of CandidateSpace(q, g) (relation/candidate_space.cpp:87,
 * relation/graph.h:34-56). ASDM_ERR_INVALID if a list is not (label,id)-sorted. */
int asdm_graph_upload(const uint32_t *offsets, const uint32_t *nbrs, const uint32_t *labels,
                      uint32_t n, uint64_t m2, uint32_t nlabels, asdm_graph **out);
/* Frees the device graph.  Free every candidate space built on it first: a
 * candidate space frees its device memory on the graph's stream and reads the
 * graph when it is freed. */
int asdm_graph_free(asdm_graph *g);
/* Knobs of the enumeration kernels, per data graph; chosen by the autotuner
 * (asdmatch_b200.autotune) by timing the caller's own batch.
 *   enum_min_blocks: register budget of the batched enumeration kernel, as
 *     resident 256-thread blocks per SM it must allow (1 = compiler's choice,
 *     up to 6); more blocks hide more load latency but spill registers.
 *   lane_leaf_max: the last query level is evaluated one partial match per
 *     lane (instead of one per warp) when its shortest list has at most this
 *     many entries (the merge / gallop split of the intersection).
 * No reference counterpart (the reference's intersection method is a
 * compile-time switch, config/config.h:16-20). */
typedef struct asdm_tuning {
    uint32_t enum_min_blocks;
    uint32_t lane_leaf_max;
    uint32_t planner;          /* ASDM_PLANNER_DP or ASDM_PLANNER_GREEDY */
    uint32_t root_block_min;   /* batches: fewest (level-0, level-1) pairs per root task of plans of at
                                  most 4 levels with a closed-form tail, 1..256 (default 64) */
    uint32_t padded_cap_log2;  /* candidate edges of a group are filled into lists padded to their
                                  label-run lengths when those total at most 2^this entries, else
                                  counted first and filled exactly (20..34, default 33: 32 GiB) */
    uint32_t merge_ratio;      /* intersection method: a list probed by a round of 32 driver entries
                                  is merged with them (32-entry windows) while its unread part is at
                                  most this many times the driver's unread part, else galloped
                                  (0 = always gallop; 0..1024, default 8) */
} asdm_tuning;
/* Order search: exhaustive over connected prefixes where the query is small
 * enough (at most 24 vertices and 4096 connected vertex subsets), else
 * greedy; or greedy always. */
#define ASDM_PLANNER_DP 0
#define ASDM_PLANNER_GREEDY 1
int asdm_graph_set_tuning(asdm_graph *g, const asdm_tuning *t);
int asdm_graph_get_tuning(const asdm_graph *g, asdm_tuning *t);

/* The CUDA stream (cudaStream_t) the library runs this graph's work on, so a
 * caller can record events around it.  No reference counterpart. */
int asdm_graph_stream(asdm_graph *g, void **stream);

/* ---- candidate space (K1-K3) ------------------------------------------- */

/* CFL candidate space of a query (CSR in the loader's layout) on the device:
 * CandidateSpace::CandidateSpace + buildCandCFL (relation/candidate_space.cpp:87-107,
 * 550-721) including buildCandidateEdge(false) (:458-487).  *nonempty = 0 when
 * some candidate set is empty (buildCandCFL returns false; the count is 0). */
int asdm_candidate_space(asdm_graph *g, const uint32_t *q_offsets, const uint32_t *q_nbrs,
                         const uint32_t *q_labels, uint32_t q_n, asdm_cs **out, int *nonempty);
/* |C(u)| for every query vertex (candidateSet[u].size()). */
int asdm_cs_sizes(const asdm_cs *cs, uint32_t *sizes);
/* C(u), sorted vertex ids (candidateSet[u], relation/candidate_space.h:47). */
int asdm_cs_read(const asdm_cs *cs, uint32_t u, uint32_t *out, uint32_t capacity);
/* Candidate edges of query edge (u, u2) (candidateEdge[u][v][u2], :49): offsets[|C(u)|+1]
 * and the neighbour vertex ids, in the order writeToStream prints them (:489-505).
 * *total receives the number of entries; ASDM_ERR_CAPACITY if it exceeds capacity. */
int asdm_cs_read_edges(const asdm_cs *cs, uint32_t u, uint32_t u2, uint32_t *offsets,
                       uint32_t *vertices, uint64_t capacity, uint64_t *total);
/* Candidate-edge entries of every directed query edge, in query-CSR order
 * (sum over v in C(u) of |candidateEdge[u][v][u2]|; the reference's query
 * edge weights, relation/candidate_space.cpp:507-524). */
int asdm_cs_edge_totals(const asdm_cs *cs, uint64_t *totals);
/* Algorithmic bytes and device milliseconds of the K1-K3 build (the
 * reference's "Filtering time", main.cpp:38). */
int asdm_cs_stats(const asdm_cs *cs, uint64_t *build_bytes, double *build_ms);
/* A 64-bit digest of the candidate space (every C(u) and every candidate-edge
 * list with its offsets, position-sensitive), computed on the device, so that
 * two builds can be compared without reading them back; *flags receives the
 * ASDM_CS_* bits of its build.  For tests at scale; no reference counterpart
 * (the reference compares CandidateSpace::writeToStream text,
 * relation/candidate_space.cpp:489-505). */
#define ASDM_CS_TWO_SCAN 1u   /* K3 counted, then filled (its group passed the padded-entry cap) */
#define ASDM_CS_LABEL_RUNS 2u /* the graph's dense label-run table was used                      */
int asdm_cs_digest(const asdm_cs *cs, uint64_t *digest, uint32_t *flags);
int asdm_cs_free(asdm_cs *cs);

/* ---- sorted-set intersection (K4) --------------------------------------- */

/* Batched k-way intersection of sorted uint32 lists on the device: for each of
 * `nsets` problems, list_ptr[list_first[s] .. list_first[s+1]) index into
 * (values, list_off); result s is written to out[out_off[s] ..) with its size
 * in out_count[s].  All arrays are host arrays.  Replaces
 * ComputeSetIntersection::LeapfrogJoin (utility/compute_set_intersection.cpp:193-233). */
int asdm_intersect_batch(const uint32_t *values, const uint64_t *list_off, uint64_t nlists,
                         const uint32_t *list_first, uint32_t nsets, const uint64_t *out_off,
                         uint32_t *out, uint32_t *out_count);

/* ---- plan ---------------------------------------------------------------- */

/* Matching order for the enumeration kernels.  order == NULL lets the planner
 * choose (cost model over candidate-edge sizes, the role of optCostPlan /
 * simplePlan, plan/optimizer.cpp:7-200,380-548); otherwise `order` is a
 * connected permutation of the query vertices. */
int asdm_plan_create(const asdm_cs *cs, const uint32_t *order, asdm_plan **out);
int asdm_plan_order(const asdm_plan *p, uint32_t *order);
/* The planner's estimated cost of the plan (partial matches times work per
 * extension), the figure the reference prints as "cost:" (minCost of
 * optCostPlan/simplePlan, main.cpp:100-114). */
int asdm_plan_cost(const asdm_plan *p, double *cost);
/* Planner guided by a cardinality cache: prefixes whose vertex set is in the
 * cache use the cached cardinality (ASDMatch.out -s; the reference loads the
 * same map with loadSubsetToCard, plan/estimator.cpp:994-1008). */
int asdm_plan_create_card(const asdm_cs *cs, const asdm_card *card, asdm_plan **out);

/* ---- .card plan cache ---------------------------------------------------- */

/* Reads a .card file: the reference's (prepare.out, executable/prepare.cpp:12-73:
 * per-bag SubsetStructure records, plan/subset_structure.cpp:455-560, then the
 * subset-cardinality map, plan/estimator.cpp:981-992, then the planning time)
 * or one written by asdm_card_write (no bag records). */
int asdm_card_load(const char *path, asdm_card **out);
int asdm_card_create(asdm_card **out);
/* subset = bitmask of query vertices (bit u = vertex u), as the reference keys it. */
int asdm_card_set(asdm_card *c, uint64_t subset, double card);
int asdm_card_lookup(const asdm_card *c, uint64_t subset, double *card);
int asdm_card_info(const asdm_card *c, uint32_t *bags, uint64_t *entries, double *plan_seconds);
/* Writes the map (values truncated to two decimals like saveSubsetToCard) and
 * the planning time, with no bag records. */
int asdm_card_write(const asdm_card *c, const char *path, double plan_seconds);
/* A cache filled with sampling estimates, made on the device: for every
 * connected induced sub-query of 3..max_subset vertices (0 = 6; fewer when
 * there are more than 4,096 such subsets), the mean weight of `walks` random
 * walks (0 = 512) through the candidate space along a connected order, each
 * walk multiplying the sizes of the candidate sets it meets and moving to a
 * uniformly drawn member (an unbiased estimate of the partial-match count).
 * Replaces cardEstimateLabeled (plan/estimator.cpp:173-291), the reference's
 * sampling estimator, as the input of the card-guided planner. */
int asdm_card_sample(asdm_cs *cs, uint32_t max_subset, uint32_t walks, uint64_t seed, asdm_card **out);
/* The same sampling estimates for given connected vertex subsets (bit u =
 * query vertex u): est[i] for masks[i], `walks` walks each (0 = 512). */
int asdm_sample_subsets(asdm_cs *cs, uint32_t nsub, const uint64_t *masks, uint32_t walks, uint64_t seed,
                        double *est);
void asdm_card_free(asdm_card *c);
int asdm_plan_free(asdm_plan *p);

/* ---- enumeration and counting (K5-K8) ----------------------------------- */

typedef struct asdm_run_opts {
    uint32_t mode;          /* ASDM_MODE_* bit mask                            */
    uint64_t budget_bytes;  /* -m budget for materialised prefixes (0 = 1.6e6 KB) */
    double time_limit_s;    /* 0 = unlimited; else ASDM_ERR_TIMEOUT past it    */
    uint64_t *local_counts; /* host |Vg| x |Vq| row-major (MODE_LOCAL) or NULL */
    uint32_t *embeddings;   /* host rows x |Vq|, sorted on return (MODE_EMBED) */
    uint64_t emb_capacity;  /* rows available in `embeddings`                  */
    uint64_t count_limit;   /* 0 = none; else stop with ASDM_ERR_LIMIT once the
                               count passes it (stats.count then >= the limit) */
} asdm_run_opts;

typedef struct asdm_run_stats {
    uint64_t count;          /* number of matches                               */
    uint64_t emb_rows;       /* rows written to `embeddings`                    */
    uint64_t intersections;  /* k-way intersections with k >= 2                 */
    uint64_t list_bytes;     /* algorithmic bytes of lists read by the kernels  */
    uint64_t tasks;          /* root tasks processed                            */
    double kernel_ms;        /* device time of the enumeration kernels          */
    double build_ms;         /* device time of the candidate-space build (K1-K3) */
    uint64_t build_bytes;    /* algorithmic bytes of that build                  */
    uint64_t tails_lane;     /* last-two-level closed forms evaluated one per lane */
    uint64_t tails_warp;     /* ... and warp-wide (long intersections)             */
    double busy_warp_ms;     /* batches with per-query budgets: warp-time charged to queries */
    double idle_warp_ms;     /* batches: warp-time spent waiting for donated work            */
} asdm_run_stats;

/* Exact enumeration of one query over its candidate space.  Replaces
 * adaptiveShareJoin (matching/adaptive.cpp:1179-2279) with the ALL_LEVEL
 * traverse/produceResult path (matching/join.cpp:819-907,1017-1097) and the
 * gLocalCount accumulation (matching/join.cpp:1035-1041). */
int asdm_run_plan(asdm_cs *cs, const asdm_plan *plan, const asdm_run_opts *opts,
                  asdm_run_stats *stats);

/* Counts like asdm_run_plan in ASDM_MODE_COUNT, but allocates no device memory:
 * for callers whose GPU memory is fully reserved by their own allocator, or
 * that cannot afford cudaMalloc/cudaFree (and their implicit synchronisation)
 * while they run.  The kernel's scratch (counters, device plan, work-donation
 * ring) is a fixed ~10 MiB file-scope device array, held by every GPU that
 * loads the library until exit.  The first call on a device looks up that
 * array's address (cudaGetSymbolAddress) with the graph's device current, so
 * make it before any stream capture.  Calls share the array and must not
 * overlap on the GPU; each call resets the parts that must start at zero.
 * Queries up to 32 vertices (a plan of at most 16 KiB); larger plans are
 * rejected with ASDM_ERR_INVALID.  Each call is synchronous: it returns after
 * the kernel has finished and its counters are read back.  It fills count,
 * intersections, list_bytes and tasks of `stats`; kernel_ms, tails_lane,
 * tails_warp, emb_rows, build_ms and build_bytes stay 0.  No counterpart in
 * the reference, which allocates with new[] throughout. */
int asdm_run_plan_count_noalloc(asdm_cs *cs, const asdm_plan *plan, double time_limit_s,
                                uint64_t count_limit, asdm_run_stats *stats);

/* A lower bound of the query's embedding count, formed on the device without
 * enumeration: query vertices of one label that may not share a data vertex
 * take candidates of distinct hash classes, a feedback vertex set is fixed to
 * its highest-degree candidates, and the remaining forest is counted by a
 * bottom-up program with sums and products saturating at 2^64 - 1.  *lower
 * receives the bound (2^64 - 1 when it reaches that), *exceeds 1 when the
 * bound shows the count is at least 2^64 — the case the counting entry points
 * report as ASDM_ERR_OVERFLOW without enumerating.  No counterpart in the
 * reference, whose ALL_LEVEL count is a size_t that wraps silently
 * (matching/join.cpp:1017-1097). */
int asdm_cs_count_lower_bound(asdm_cs *cs, uint64_t *lower, int *exceeds);

/* One call for a query end to end on a resident graph: candidate space, plan
 * and count (the whole of ASDMatch.out's main(), main.cpp:11-147, without I/O). */
int asdm_count_query(asdm_graph *g, const uint32_t *q_offsets, const uint32_t *q_nbrs,
                     const uint32_t *q_labels, uint32_t q_n, const asdm_run_opts *opts,
                     asdm_run_stats *stats);

/* Many queries against one resident data graph, batched (no reference
 * counterpart; the reference runs one query per process).  Query i is the CSR
 * slice q_offsets[q_off_base[i] ..], q_nbrs[q_nbr_base[i] ..],
 * q_labels[q_lab_base[i] ..] with q_sizes[i] vertices.  Queries are grouped
 * (up to 32 GiB of candidate-space state per group); each group builds its
 * candidate spaces with one launch per CFL phase and counts with one
 * persistent kernel over all (query, root task) pairs.  counts[i] and
 * status[i] receive each query's result; stats (nullable) the totals; the
 * call returns ASDM_OK when every status is ASDM_OK. */
int asdm_run_batch(asdm_graph *g, uint32_t nq, const uint32_t *q_sizes, const uint64_t *q_off_base,
                   const uint32_t *q_offsets, const uint64_t *q_nbr_base, const uint32_t *q_nbrs,
                   const uint64_t *q_lab_base, const uint32_t *q_labels, double time_limit_s,
                   uint64_t *counts, int *status, asdm_run_stats *stats);
/* Options of asdm_run_batch_ex. */
typedef struct asdm_batch_opts {
    double time_limit_s;            /* 0 = none (device time for the whole group)          */
    uint64_t count_limit;           /* 0 = none; a query past it stops with ASDM_ERR_LIMIT  */
    const asdm_card *const *cards;  /* per query cardinality cache for its plan, or NULL    */
    asdm_estimator *estimator;      /* learned estimates for the planner, or NULL           */
    uint32_t learned_max_subset;    /* largest prefix the estimator is asked about (0 = 6) */
    double query_time_limit_s;      /* 0 = none; else each query may use this much GPU time
                                       (its warp-time over all resident warps: the time it
                                       would run alone on the GPU) in the enumeration kernel,
                                       past which it alone stops with ASDM_ERR_TIMEOUT      */
} asdm_batch_opts;
/* asdm_run_batch with per-query count limits and plan caches (the learned
 * estimator's predictions reach the planner this way); local_counts as in
 * asdm_run_batch_local, or NULL for counts only. */
int asdm_run_batch_ex(asdm_graph *g, uint32_t nq, const uint32_t *q_sizes, const uint64_t *q_off_base,
                      const uint32_t *q_offsets, const uint64_t *q_nbr_base, const uint32_t *q_nbrs,
                      const uint64_t *q_lab_base, const uint32_t *q_labels, const asdm_batch_opts *opts,
                      uint64_t *counts, int *status, uint64_t *const *local_counts, asdm_run_stats *stats);
/* The same, also producing each query's |Vg| x |Vq_i| local-count matrix
 * (the reference's LOCAL_COUNT output, matching/join.cpp:1035-1041, one
 * process per query there) into local_counts[i] (row-major, may be NULL to
 * skip a query's matrix); the matrices of a group live on the device until
 * the group finishes. */
int asdm_run_batch_local(asdm_graph *g, uint32_t nq, const uint32_t *q_sizes, const uint64_t *q_off_base,
                         const uint32_t *q_offsets, const uint64_t *q_nbr_base, const uint32_t *q_nbrs,
                         const uint64_t *q_lab_base, const uint32_t *q_labels, double time_limit_s,
                         uint64_t *counts, int *status, uint64_t *const *local_counts,
                         asdm_run_stats *stats);

/* ---- learned cardinality estimator ------------------------------------- */

/* The three stages of the batched form as separate calls, for callers that
 * plan between filtering and enumeration (the learned estimator does):
 * candidate spaces of nq packed queries (layout as asdm_run_batch), built in
 * groups; out[i] is NULL where status[i] != 0, nonempty[i] as in
 * asdm_candidate_space.  Each out[i] is freed with asdm_cs_free. */
int asdm_candidate_space_batch(asdm_graph *g, uint32_t nq, const uint32_t *q_sizes, const uint64_t *q_off_base,
                               const uint32_t *q_offsets, const uint64_t *q_nbr_base, const uint32_t *q_nbrs,
                               const uint64_t *q_lab_base, const uint32_t *q_labels, asdm_cs **out, int *nonempty,
                               int *status);
/* Counts every (cs[i], plans[i]) in one persistent launch; all candidate
 * spaces on the same graph; opts->cards is ignored (plans are given). */
int asdm_run_planned(uint32_t nq, asdm_cs *const *cs, const asdm_plan *const *plans, const asdm_batch_opts *opts,
                     uint64_t *counts, int *status, asdm_run_stats *stats);
/* The same, also returning per query the SM clock cycles that warps spent
 * on its tasks (summed over warps): where a batch's enumeration time goes.
 * No reference counterpart. */
int asdm_run_planned_profile(uint32_t nq, asdm_cs *const *cs, const asdm_plan *const *plans,
                             const asdm_batch_opts *opts, uint64_t *counts, int *status, asdm_run_stats *stats,
                             uint64_t *cycles);

/* Partial-match counts of query-vertex prefixes inside a candidate space:
 * prefix i is orders[i*|Vq| .. i*|Vq| + depths[i]) (distinct vertices, each
 * after the first adjacent to an earlier one); counts[i] receives the number
 * of injective assignments of those vertices to their candidate sets along
 * candidate edges, i.e. the cardinality the reference's estimator samples
 * (cardEstimateLabeled, plan/estimator.cpp:173-291).  All prefixes run in one
 * batched launch; status[i] as in asdm_run_batch (ASDM_ERR_LIMIT past
 * count_limit, 0 = none). */
int asdm_prefix_counts(asdm_cs *cs, uint32_t nprefix, const uint32_t *orders, const uint32_t *depths,
                       double time_limit_s, uint64_t count_limit, uint64_t *counts, int *status);

/* The estimator's tensor-core GEMM on its own, for testing: C[M][N] =
 * sum_k A[m][k] * B[n][k] with A, B given as bf16 bit patterns (host arrays)
 * and C in fp32.  No reference counterpart (the reference estimates by
 * sampling, plan/estimator.cpp:173-291). */
int asdm_gemm_bf16(int M, int N, int K, const uint16_t *A, const uint16_t *B, float *C);

/* A 3-layer message-passing network over (sub-)query graphs, hidden width
 * 128, BF16 weights/activations with FP32 accumulation, predicting
 * log(1 + cardinality); forward, backward and Adam on the device.  It stands
 * in for the reference's sampling estimator (cardEstimateLabeled,
 * plan/estimator.cpp:173-291) as a source of subset cardinalities for the
 * planner; it changes plans, never counts.
 * A batch: n_nodes nodes with `in_features` fp32 features each (x, row-major),
 * a symmetric adjacency in CSR over the batch's nodes (adj_off[n_nodes+1],
 * adj), and node_graph[v] in [0, n_graphs). */
int asdm_est_create(uint32_t in_features, uint64_t seed, asdm_estimator **out);
int asdm_est_train_step(asdm_estimator *e, int n_nodes, int n_graphs, const float *x, const uint32_t *adj_off,
                        const uint32_t *adj, const uint32_t *node_graph, const float *target, float lr,
                        float *loss);
int asdm_est_predict(asdm_estimator *e, int n_nodes, int n_graphs, const float *x, const uint32_t *adj_off,
                     const uint32_t *adj, const uint32_t *node_graph, float *out);
/* fp32 parameter vector (for saving); count receives its length. */
int asdm_est_params(asdm_estimator *e, float *out, uint64_t capacity, uint64_t *count);
int asdm_est_set_params(asdm_estimator *e, const float *in, uint64_t count);
void asdm_est_free(asdm_estimator *e);
/* The estimator's input for sub-queries of a query with a built candidate
 * space: subset i is the vertex set masks[i] (bit u = query vertex u, at most
 * 64 vertices, connected).  Writes, per subset in order, its vertices in
 * ascending order as nodes: x (ASDM_EST_FEATURES floats per node), the local
 * adjacency in CSR over all nodes (adj_off, adj; adj_capacity entries), and
 * node_graph[node] = i.  *n_nodes / *n_adj receive the totals (call with
 * NULL outputs to size them). */
#define ASDM_EST_FEATURES 44
int asdm_est_features(const asdm_cs *cs, uint32_t nsub, const uint64_t *masks, float *x, uint32_t *adj_off,
                      uint32_t *adj, uint64_t adj_capacity, uint32_t *node_graph, uint64_t *n_nodes, uint64_t *n_adj);
/* A plan chosen with learned cardinalities: the planner's greedy search, with
 * every prefix of 3..max_subset vertices (0 = 6) estimated by the model, all
 * starts of all given queries searched in lockstep (one forward pass per
 * step).  plans[i] is freed with asdm_plan_free. */
int asdm_plan_create_learned(uint32_t nq, asdm_cs *const *cs, asdm_estimator *e, uint32_t max_subset,
                             asdm_plan **plans);

#ifdef __cplusplus
}
#endif
#endif /* ASDM_H */
