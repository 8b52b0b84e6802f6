/* C ABI of the B200 KGraph library (libkgraph_b200.so).
 *
 * Plain pointers and sizes only.  Every call returns 0 on success and a
 * non-zero KG_E_* code on failure; kg_last_error(ctx) then holds the message.
 * The C++ API (kgraph.h) and the Python module are thin layers over these
 * entry points, and a foreign binding (ctypes, cgo, JNI ...) can call them
 * directly.  Each entry point names the reference interface it replaces.
 *
 * Pointers to rows, queries and outputs may be host or device (CUDA)
 * memory; the library detects which and copies host buffers through pinned
 * staging on the context's stream.  A context is bound to one GPU; calls on
 * one context are serialised by an internal lock, so concurrent callers (the
 * reference calls KGraph::search from many OpenMP threads,
 * python-api.cpp:292-301) are safe.
 */
#ifndef KGRAPH_B200_H
#define KGRAPH_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct kg_ctx kg_ctx;

enum { KG_METRIC_EUCLIDEAN = 0, KG_METRIC_ANGULAR = 1, KG_METRIC_L2SQR = 2 };
enum {
    KG_OK = 0,
    KG_E_INVALID = 1,   /* kgraph::invalid_argument */
    KG_E_RUNTIME = 2,   /* kgraph::runtime_error / std::runtime_error */
    KG_E_IO = 3,        /* kgraph::io_error */
    KG_E_CUDA = 4,      /* CUDA failure (allocation, launch) */
    KG_E_DEVICE = 5     /* a kernel reported an error (lock spin limit, bad id) */
};

/* KGraph::IndexParams, kgraph.h:94-110 (same fields, same defaults). */
typedef struct {
    unsigned iterations, L, K, S, R, controls, seed;
    float delta, recall;
    unsigned prune;
    int reverse;
} kg_index_params;

/* KGraph::IndexInfo, kgraph.h:135-147. stop_condition: 0 ITERATION, 1 DELTA, 2 RECALL. */
typedef struct {
    int stop_condition;
    unsigned iterations;
    float cost, recall, accuracy, delta, M;
} kg_index_info;

/* KGraph::SearchParams, kgraph.h:113-126. */
typedef struct {
    unsigned K, M, P, S, T;
    float epsilon;
    unsigned seed, init;
} kg_search_params;

/* Fills the reference's defaults (kgraph.h:14-37, 108, 124). */
void kg_index_params_default(kg_index_params *p);
void kg_search_params_default(kg_search_params *p);

/* Creates a context on CUDA device `device` (KGraph::create, kgraph.h:199). */
int kg_ctx_create(int device, kg_ctx **out);
void kg_ctx_destroy(kg_ctx *ctx);
const char *kg_last_error(kg_ctx *ctx);
/* KGraph::version, kgraph.h:201. */
const char *kg_version(void);
/* kgraph::verbosity (kgraph.h:42): > 0 prints the per-iteration build log
 * line of kgraph.cpp:952-962 to stderr. */
void kg_set_verbosity(unsigned v);

/* Binds the dataset: n rows of d floats, `stride_bytes` apart, copied into
 * HBM with 64-byte aligned, zero-padded rows.  metric is KG_METRIC_*:
 *   EUCLIDEAN  the Python oracle, half squared L2 (python-api.cpp:51-59)
 *   ANGULAR    the Python oracle, -cos          (python-api.cpp:61-69)
 *   L2SQR      MatrixOracle<.., metric::l2sqr>   (kgraph-data.h:38-61, 302-331)
 * Replaces the dataset the reference's oracle wraps (NDArrayOracle ctor,
 * python-api.cpp:110-114; MatrixProxy, kgraph-data.h:221-231). */
int kg_set_data(kg_ctx *ctx, const float *rows, size_t n, size_t d, size_t stride_bytes, int metric);

/* KGraph::build (kgraph.h:168; KGraphConstructor, kgraph.cpp:886-999).
 * info may be NULL. */
int kg_build(kg_ctx *ctx, const kg_index_params *params, kg_index_info *info);

/* Graph size for export: n nodes, E edges. */
int kg_graph_size(kg_ctx *ctx, size_t *n, size_t *E);
/* Copies the graph out as CSR: offsets[n+1], ids[E], dists[E] (may be NULL),
 * M[n].  Backs KGraph::save / get_nn (kgraph.cpp:333-373, 566-582). */
int kg_graph_export(kg_ctx *ctx, uint64_t *offsets, uint32_t *ids, float *dists, uint32_t *M);
/* Installs a CSR graph (KGraph::load, kgraph.cpp:291-331).  dists may be NULL
 * (FORMAT_NO_DIST); no_dist then marks distances unavailable. */
int kg_graph_import(kg_ctx *ctx, size_t n, const uint64_t *offsets, const uint32_t *ids, const float *dists,
                    const uint32_t *M);

/* Batched KGraph::search (kgraph.h:197; KGraphImpl::search, kgraph.cpp:423-564)
 * for nq queries of d floats, `q_stride_bytes` apart, in one launch.
 * K_per_q / P_per_q (may be NULL) override params->K / params->P per query.
 * Outputs are rows of out_ld entries (out_ld >= every K): ids[nq*out_ld],
 * dists (may be NULL), counts[nq] (results returned, <= K), costs (may be
 * NULL; SearchInfo.cost).  When params->init > 0, ids is also the input of the
 * starting points (doc/params.md "User-Provided Starting Points").
 * Without a graph every query takes the brute-force path
 * (SearchOracle::search, kgraph.cpp:231-252; python-api.cpp:303-314). */
int kg_search_batch(kg_ctx *ctx, const float *queries, size_t nq, size_t q_stride_bytes,
                    const kg_search_params *params, const uint32_t *K_per_q, const uint32_t *P_per_q,
                    size_t out_ld, uint32_t *ids, float *dists, uint32_t *counts, float *costs);

/* Launch shape of the batched search kernel.  No counterpart in the reference
 * (its search is one OpenMP thread per query, python-api.cpp:292-301): every
 * shape walks exactly as the reference and returns the same bits; only the
 * speed differs.
 *   split            D-split: lanes of a warp per distance (2, 4 or 8); one
 *                    warp evaluates 32/split candidates per pass
 *   warps_per_block  query tile: queries (one warp each) per block, 1/2/4/8;
 *                    0 = as many as fit 200 KB of shared memory, at most 8
 *   prefetch         neighbour batches whose rows are prefetched into L2 ahead
 *                    of the walk (0 or 2)
 *   regs             registers per thread the kernel is compiled for: 64
 *                    (0 = 64), 80 (FP32 walk only: fewer spills where
 *                    large pools limit residency anyway) or 56 (the FP32
 *                    walk with compact entries, blocks of at most 4 warps:
 *                    36 resident warps per SM instead of 32)
 *   compact          1: 8-byte pool entries instead of 12 (the id in the
 *                    bits N needs, the expansion progress in batches of S in
 *                    the rest of 31 bits; M read again when an entry is
 *                    expanded), so more queries fit on an SM where the pool's
 *                    shared memory limits residency (large P).  Used by the
 *                    FP32 walk where the graph allows it (S >= 1, every
 *                    node's min(max(M, params M), degree) <= (2^(31 - id
 *                    bits) - 1) S); elsewhere the 12-byte entry runs.
 *                    A new context starts with split 4, warps_per_block 0,
 *                    prefetch 2, regs 64, compact 1.
 * ms / default_ms / variants are filled by kg_search_autotune. */
typedef struct {
    unsigned split, warps_per_block, prefetch;
    float ms, default_ms;
    unsigned variants;
    unsigned regs;
    unsigned compact;
} kg_search_tuning;
/* Times every shape on `queries` (a representative sample), checks that all
 * of them return identical ids, distances, counts and costs, and keeps the
 * fastest for the context's later searches.  With params->init > 0 the
 * starting points are init_ids, nq rows of init_ld (else both are ignored).
 * best may be NULL. */
int kg_search_autotune(kg_ctx *ctx, const float *queries, size_t nq, size_t q_stride_bytes,
                       const kg_search_params *params, const uint32_t *K_per_q, const uint32_t *P_per_q,
                       const uint32_t *init_ids, size_t init_ld, kg_search_tuning *best);
/* Sets / reads the context's search shape (split, warps_per_block, prefetch, regs, compact). */
int kg_set_search_tuning(kg_ctx *ctx, const kg_search_tuning *t);
int kg_get_search_tuning(kg_ctx *ctx, kg_search_tuning *t);
/* The shape the last kg_search_batch actually launched: warps_per_block as
 * chosen (0 when every query went to the tensor-core brute force), compact = 1
 * only if the compact pool entry ran, ms its device time. */
int kg_last_search_shape(kg_ctx *ctx, kg_search_tuning *t);

/* Distance filter of the search.  No counterpart in the reference (its walk
 * evaluates every candidate in FP32, kgraph.cpp:495-513).  With BF16 or FP8
 * (E4M3 with a per-row scale), the walk first evaluates each candidate against
 * a compressed copy of its row and derives a rigorous lower bound of its
 * canonical FP32 distance (FP32 accumulation, the copy's per-row error bound and
 * the FP32 rounding bounds of both computations).  Once the pool is full, a
 * candidate whose bound is at or beyond the pool's last entry -- one the
 * reference would drop into the spare slot -- is not evaluated in FP32; every
 * other candidate is, exactly as without the filter.  Results (ids,
 * distances, counts, costs) are identical in every mode.  The copy is built on
 * the call (and again after kg_set_data), n * round_up(d, 16) * 2 (BF16) or
 * * 1 (FP8) bytes plus 16 bytes per row. */
enum { KG_SEARCH_FP32 = 0, KG_SEARCH_BF16 = 1, KG_SEARCH_FP8 = 2 };
int kg_set_search_precision(kg_ctx *ctx, int mode);
/* The filter's work in the last kg_search_batch and its copy's quantisation
 * error: approx = candidates evaluated on the compressed rows, skipped = of
 * those, the ones the bound excluded (FP32 evaluations saved); max / mean over
 * rows of ||x - y|| / ||x||, y the reconstructed row. */
typedef struct {
    int mode;
    unsigned long long approx, skipped;
    double max_rel_row_error, mean_rel_row_error;
} kg_search_filter_stats;
int kg_last_search_filter(kg_ctx *ctx, kg_search_filter_stats *out);
/* Check of the filter's arithmetic: for each of nq queries and each of its
 * per_query dataset rows (ids, nq rows of per_query), the lower bound the
 * filter derives from the compressed row (lb) and the canonical FP32 distance
 * (dist); lb <= dist must hold for every pair.  Needs a BF16 or FP8 search
 * precision and d <= 256.  Pointers may be host or device memory. */
int kg_filter_bounds(kg_ctx *ctx, const float *queries, size_t nq, size_t q_stride_bytes, const uint32_t *ids,
                     size_t per_query, float *lb, float *dist);

/* Brute-force path of kg_search_batch (every query of a batch with P >= N, or
 * no graph: SearchOracle::search, kgraph.cpp:231-252; the Python module's
 * blas=True, python-api.cpp:131-205).  Results are identical in every mode.
 *   KG_BRUTEFORCE_AUTO    the tensor-core path where it applies (K <= 128,
 *                         d <= 256, at least 1024 rows), else the CUDA cores;
 *   KG_BRUTEFORCE_SCAN    one warp per query scans every row in id order on the
 *                         CUDA cores (the reference's loop);
 *   KG_BRUTEFORCE_TENSOR  the tensor-core path where it applies: rows and
 *                         queries centred and rounded to BF16, their products on
 *                         tcgen05 (FP32 accumulation) give an approximate
 *                         distance; a rigorous margin of its error selects, per
 *                         query, every row that can be among the K nearest, and
 *                         those are evaluated with the canonical FP32 distance.
 *                         No counterpart in the reference.  Memory: a BF16 copy
 *                         of the dataset (n * round_up(d, 16) * 2 bytes), built on
 *                         first use. */
enum { KG_BRUTEFORCE_AUTO = 0, KG_BRUTEFORCE_SCAN = 1, KG_BRUTEFORCE_TENSOR = 2 };
int kg_set_bruteforce_mode(kg_ctx *ctx, int mode);
/* The last brute-force batch: tensor = 1 when it ran on the tensor cores;
 * candidates = rows evaluated in FP32 over all queries; full_scans = queries
 * whose candidates exceeded the per-query capacity (max(1024, 8 K)) and were
 * scanned in full instead. */
typedef struct {
    int tensor;
    unsigned long long candidates, full_scans;
} kg_bruteforce_stats;
int kg_last_bruteforce_stats(kg_ctx *ctx, kg_bruteforce_stats *out);

/* KGraphImpl::reverse (kgraph.cpp:667-702) on the current graph. */
int kg_reverse(kg_ctx *ctx, int rev_k);
/* KGraph::prune (kgraph.h:180; kgraph.cpp:584-665) on the current graph. */
int kg_prune(kg_ctx *ctx, unsigned level);

/* kg_search_batch without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot call cudaMalloc while serving
 * -- a latency-critical thread that must not block on the allocator, or an
 * application that owns all GPU memory through its own pool.  Queries and
 * outputs must be DEVICE buffers (queries: 16-byte aligned rows of the
 * context's padded width, q_stride_bytes = 4 * round_up(d, 16)); dataset and
 * graph are the context's.  One K and P for the whole batch, P <= 4096.
 * Scratch (counters, seed table, visited sets) is a static device array of
 * KG_NOALLOC_SCRATCH_BYTES per GPU, held until the process exits; a batch
 * whose seeds, per-query index and one SM's worth of visited sets do not fit
 * is rejected with KG_E_INVALID.  The first call through a context looks up
 * the array's device address on the context's device and keeps it in the
 * context, so make that call before any stream capture; create contexts anew
 * after a device reset (the old ones' buffers are gone with it).  Every call
 * shares the array: calls whose kernels overlap on the GPU race; serialise
 * them.  Results are those of kg_search_batch.  Speed: it reuses the search-
 * side copy of the graph and the distance filter's compressed rows when an
 * earlier kg_search_batch on the context has built them; otherwise it walks
 * the CSR graph in FP32 (same results, lower throughput), since building
 * either would allocate. */
#define KG_NOALLOC_SCRATCH_BYTES ((size_t)64 << 20)
int kg_search_batch_noalloc(kg_ctx *ctx, const float *queries, size_t nq, size_t q_stride_bytes,
                            const kg_search_params *params, size_t out_ld, uint32_t *ids, float *dists,
                            uint32_t *counts, float *costs);
/* Size of that static scratch array in bytes. */
size_t kg_noalloc_scratch_bytes(void);

/* Learned entry router.  No counterpart in the reference: it predicts, per
 * query, starting points for the walk, which the search takes through the
 * reference's own user-provided starting points (params->init > 0 with the
 * seeds in ids, doc/params.md "User-Provided Starting Points").  Training
 * (on the GPU): k-means of the dataset into `clusters` entry clusters (entry
 * node = the member nearest the centroid); labels = the cluster of the best
 * node the plain search (P = label_P) finds for each training query (then
 * refined, see `refine`); MLP
 * d -> hidden -> hidden -> clusters (ReLU), BF16 weights with FP32 masters and
 * accumulation, softmax cross-entropy, Adam. */
typedef struct {
    unsigned clusters, hidden, kmeans_iters, label_P, epochs, batch;
    float lr;
    unsigned seed;
    unsigned entries;   /* fine clusters (entry nodes) per cluster, 1..16 */
    unsigned probe;     /* clusters whose entry nodes are ranked per query, 1..32 */
    unsigned refine;    /* refinement rounds (0..8): each relabels a training query with the node the
                           router-seeded walk (P = refine_P) finds when it is closer than its label,
                           then trains `epochs` more */
    unsigned refine_P;
} kg_router_params;
typedef struct {
    unsigned steps;
    float final_loss, train_accuracy;
    unsigned empty_clusters;     /* clusters without an entry node */
    unsigned entries;            /* entry nodes over all clusters */
    unsigned component_entries;  /* of which added for graph components no fine cluster reached */
    unsigned relabelled;         /* training labels changed by the refinement */
    float label_s;               /* wall seconds: plain-search labels of the training queries */
    float cluster_s;             /* normalisation, k-means, entry nodes, graph components */
    float mlp_s;                 /* MLP epochs (all rounds) */
    float refine_s;              /* refinement searches and regrouping */
} kg_router_info;
void kg_router_params_default(kg_router_params *p);
/* Trains the router on the context's dataset and graph. */
int kg_router_train(kg_ctx *ctx, const kg_router_params *p, const float *train_queries, size_t ntrain,
                    size_t q_stride_bytes, kg_router_info *info);
/* Seeds of each query: the entry nodes of its `probe` most likely clusters,
 * ranked by exact FP32 distance to the query, the m nearest first (rows of
 * out_ld); pass them to kg_search_batch as ids with params->init = m (m < K). */
int kg_router_seeds(kg_ctx *ctx, const float *queries, size_t nq, size_t q_stride_bytes, unsigned m, uint32_t *seeds,
                    size_t out_ld);
/* kg_router_seeds followed by kg_search_batch in one call: the queries cross
 * to the GPU once and the seeds never leave it.  params->init is the number of
 * router seeds per query (0 < init < K); ids is output only.  Results equal
 * kg_router_seeds + kg_search_batch(init) on the same queries. */
int kg_router_search(kg_ctx *ctx, const float *queries, size_t nq, size_t q_stride_bytes,
                     const kg_search_params *params, size_t out_ld, uint32_t *ids, float *dists, uint32_t *counts,
                     float *costs);
/* Mean loss and gradients (W1|b1|W2|b2|W3|b3, FP32, row-major in x out) of the
 * MLP on n <= 4096 labelled rows, with `weights` (same layout, may be NULL to
 * keep the current ones) and identity input normalisation: the check of the
 * training kernels against an independent implementation. */
int kg_router_gradients(kg_ctx *ctx, unsigned d, unsigned hidden, unsigned clusters, const float *weights,
                        const float *x, const int32_t *labels, unsigned n, float *loss, float *grads);
/* Milliseconds of the last kg_router_seeds device work (CUDA events on the
 * context's stream). */
int kg_last_router_timing(kg_ctx *ctx, float *seeds_ms);
/* Checks of the router's tensor-core products on caller data (no counterpart
 * in the reference).  Operands are BF16 bit patterns (uint16), host or device
 * memory; outputs are copied back to the caller's buffers.
 * kg_tc_gemm_check: C[M,N] = op(A)[M,K] op(B)[K,N] (+ beta C) (+ bias[N])
 * (ReLU when relu != 0) with FP32 accumulation, exactly the product the MLP's
 * forward and backward passes run; op(A) = A (M x K, row stride lda) or, with
 * ta, A^T (A stored K x M); likewise B / tb.  C has row stride ldc >= N and is
 * read when beta != 0.
 * kg_tc_assign_check: the fused k-means assignment, lab[r] = argmin over c of
 * cn[c] - 2 F[r].cent[c] (ties: smaller c), best[r] that value (may be NULL);
 * F is n x D, cent C x D, row-major, D <= 256. */
int kg_tc_gemm_check(kg_ctx *ctx, int M, int N, int K, const uint16_t *A, int lda, int ta, const uint16_t *B,
                     int ldb, int tb, const float *bias, int relu, float beta, float *C, int ldc);
int kg_tc_assign_check(kg_ctx *ctx, const uint16_t *F, int n, int D, const uint16_t *cent, int C, const float *cn,
                       int32_t *lab, float *best);

/* Precision of the NN-descent local join.  No counterpart in the reference
 * (its join evaluates every pair in FP32, kgraph.cpp:740-751, 797-815).
 *   KG_JOIN_FP32  every pair's canonical FP32 distance on the CUDA cores;
 *   KG_JOIN_BF16  the pairs' Gram block on the tensor cores (BF16 operands
 *                 centred on the node, FP32 accumulation); a pair is skipped
 *                 only when its BF16 distance minus a rigorous error margin is
 *                 above both endpoints' radius, every other pair is recomputed
 *                 in FP32 and inserted exactly as in KG_JOIN_FP32;
 *                 The BF16 filter runs in the iterations that start with at
 *                 least half of the pools full (before that every pair passes
 *                 the radius test and the FP32 join is the cheaper path);
 *   KG_JOIN_BF16_ALWAYS  the BF16 filter in every iteration;
 *   KG_JOIN_FP8 / KG_JOIN_FP8_ALWAYS  the same filter with FP8 E4M3 tiles and a
 *                 scale per row (max |x_u - x_n| / 448); the margin adds each
 *                 row's exact quantisation error ||v - scale q|| (FP64) relative
 *                 to ||v||; needs d padded to a multiple of 32;
 *   KG_JOIN_AUTO  (default) the faster path measured for the build's own
 *                 workloads: KG_JOIN_FP32 (the join is bound by the locked
 *                 pool inserts, which the filter does not reduce). */
enum { KG_JOIN_AUTO = 0, KG_JOIN_FP32 = 1, KG_JOIN_BF16 = 2, KG_JOIN_BF16_ALWAYS = 3, KG_JOIN_FP8 = 4,
       KG_JOIN_FP8_ALWAYS = 5 };
int kg_set_join_precision(kg_ctx *ctx, int mode);

/* How the FP32 local join applies its inserts (Nhood::parallel_try_insert,
 * kgraph.cpp:723-736).  No counterpart in the reference, whose threads insert
 * under a per-node lock as they go.
 *   KG_INSERTS_LOCKED    the same: one warp takes the target's lock per offer;
 *   KG_INSERTS_DEFERRED  the join records every offer that passes the unlocked
 *                        radius test; the offers are then grouped by target and
 *                        each pool takes its own in one merge, in ascending
 *                        (distance, id) order (inserts into different pools
 *                        touch disjoint state: a pool's outcome depends only on
 *                        the order of its own offers, which the reference's
 *                        threads leave arbitrary), with the same duplicate,
 *                        radius and L rules, and `found` as the inserts set it
 *                        in the offers' arrival order; offers
 *                        beyond the record buffer's capacity (sized from free
 *                        device memory, at most 20 GB; a join that needs more
 *                        runs in rounds of consecutive nodes) are inserted under
 *                        the lock during the join;
 *   KG_INSERTS_AUTO      (default) KG_INSERTS_DEFERRED.
 * The tensor-core joins (KG_JOIN_BF16 / KG_JOIN_FP8 iterations) always lock. */
enum { KG_INSERTS_AUTO = 0, KG_INSERTS_LOCKED = 1, KG_INSERTS_DEFERRED = 2 };
int kg_set_join_inserts(kg_ctx *ctx, int mode);
/* Bound on the deferred inserts' record buffers, in offers (32 bytes of device
 * memory each; 0 = automatic: 30 % of free memory, at most 20 GB).  A join
 * whose first-iteration offers (at most 2 x C(2S, 2) per node) exceed it runs
 * in rounds of consecutive nodes, each with its own merge; offers beyond it
 * within a round are inserted under the lock.  No counterpart in the
 * reference. */
int kg_set_join_offer_capacity(kg_ctx *ctx, size_t offers);
/* Check entry point of the deferred inserts' merge, on caller data: n pools of
 * L+1 entries (rows of L+1: distances, ids with the new-flag in bit 31), their
 * list lengths and radii (updated in place), and n_off offers (target pool,
 * candidate id, distance, source node with bit 31 set for a pair's x <- y
 * offer); found[source] is set to 1 where such an offer lands below K (other
 * entries 0).  A pool's offers are merged in ascending (distance, id) order in
 * passes of at most 512; `found` follows the serial inserts in the caller's
 * order of each pool's offers (their arrival order).  No counterpart in the
 * reference. */
int kg_join_merge_check(kg_ctx *ctx, unsigned n, unsigned L, unsigned K, float *pool_d, uint32_t *pool_i,
                        uint32_t *nodeL, float *radius, size_t n_off, const uint32_t *target, const uint32_t *cand,
                        const float *dist, const uint32_t *src, uint32_t *found);
/* Counters of the last kg_build's join.  mode: KG_JOIN_BF16 or KG_JOIN_FP8 when
 * any iteration ran the tensor-core filter (tc_iterations of them).  pairs: join
 * pairs (IndexInfo.cost * N(N-1)/2 summed over iterations); rechecked: pairs
 * recomputed in FP32 after the BF16 filter.  On a sample of nodes every pair
 * is also evaluated in FP64: sampled pairs, the BF16 tile distance's absolute
 * and relative error against FP64 (max, mean) and the error as a fraction of
 * the margin (max, mean; < 1 means the filter was safe); violations = sampled
 * or rechecked pairs whose error exceeded the margin. */
typedef struct {
    int mode;
    unsigned long long pairs, rechecked, sampled, violations;
    double max_abs_err, mean_abs_err, max_rel_err, mean_rel_err, max_err_over_margin, mean_err_over_margin;
    unsigned tc_iterations;
} kg_join_stats;
int kg_last_join_stats(kg_ctx *ctx, kg_join_stats *out);

/* Milliseconds of the last kg_build / kg_search_batch device work, measured
 * with CUDA events on the context's stream (for profiling and benchmarks). */
int kg_last_timing(kg_ctx *ctx, float *build_ms, float *search_ms);
/* CUDA graph launches of the last kg_build's iterations.  No counterpart in
 * the reference: each NN-descent iteration (update, join, statistics) is
 * captured once and replayed as one graph launch (two with the statistics
 * split off when the join runs on the tensor cores, three with its update). */
int kg_last_build_graphs(kg_ctx *ctx, unsigned *graph_launches);
/* Work of the last kg_build's local joins, summed over its iterations: pairs
 * evaluated (the reference's IndexInfo.cost * N(N-1)/2 counter,
 * kgraph.cpp:797-815, 928), list entries (|new| + |old| over all nodes: the
 * dataset rows the joins read) and the iterations run.  Any pointer may be
 * NULL. */
int kg_last_build_work(kg_ctx *ctx, uint64_t *pairs, uint64_t *list_entries, unsigned *iterations);
/* The same per NN-descent iteration of the last kg_build (the reference's
 * per-iteration log line, kgraph.cpp:952-962, has no counterpart for these):
 * join pairs, join list entries, locked insert attempts (offers that passed the
 * unlocked radius test, kgraph.cpp:724), inserts that entered a list (not a
 * duplicate), the iteration's device milliseconds (its launches: the previous
 * iteration's update, the join, the statistics) and whether its join ran on
 * the tensor cores.  Fills min(cap, iterations) entries; *n = iterations. */
typedef struct {
    unsigned long long pairs, list_entries, insert_attempts, inserts_landed;
    float ms;
    unsigned tensor_core;
} kg_build_iteration;
int kg_last_build_iterations(kg_ctx *ctx, kg_build_iteration *out, unsigned cap, unsigned *n);
/* Work of the last kg_search_batch: distance evaluations (seeds included;
 * the sum of SearchInfo.cost * N plus the seeds) and adjacency entries read. */
int kg_last_search_work(kg_ctx *ctx, uint64_t *evaluations, uint64_t *adjacency_reads);

#ifdef __cplusplus
}
#endif
#endif
