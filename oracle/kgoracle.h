/* CPU restatement of KGraph's hot paths -- TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker the tests, smoke() and bench.py's cpu_baseline
 * compare the CUDA path against.  The product never links, loads or calls it.
 * Every function restates one piece of the reference (file:line given with
 * each declaration) in scalar C++, single threaded and deterministic.
 *
 * Parity pin: tests/test_oracle_pin.py checks this restatement against the
 * reference itself, compiled from its own sources into oracle/_ref (distances,
 * brute force, search on a reference-built index, and a single-thread build
 * graph bit for bit), and against the committed fixtures in tests/golden/.
 *
 * Metrics (the three dense oracles the reference ships):
 *   KGO_EUCLIDEAN = 0  python-api.cpp:51-59   d = (n_i + n_j) - x.y, n = |x|^2/2
 *   KGO_ANGULAR   = 1  python-api.cpp:61-69   d = -x.y / (n_i*n_j + FLT_EPSILON), n = |x|
 *   KGO_L2SQR     = 2  kgraph-data.h:38-61    d = sum (x-y)^2
 * All sums follow the reference's AVX-512 xsimd order (kgraph-data.h:41-103)
 * as its -O3 build evaluates them (measured bit for bit against oracle/_ref):
 * 16 lanes, lane l accumulates elements l, l+16, ... as a rounded product
 * then a rounded add (the vector intrinsics are not contracted); then the
 * xsimd avx512f reduce_add tree; then the scalar tail (D % 16 elements),
 * added in order: when the tail has 8 or more elements GCC vectorises the
 * first 8 products (rounded products, in-order adds); every other tail
 * element is a FUSED multiply-add (GCC contracts the scalar `acc += a*b`).
 * The angular denominator n_i*n_j + FLT_EPSILON is fused the same way.
 */
#ifndef KGORACLE_H
#define KGORACLE_H
#include <stdint.h>
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

enum { KGO_EUCLIDEAN = 0, KGO_ANGULAR = 1, KGO_L2SQR = 2 };

/* kgraph-data.h:65-83 (dot), 87-103 (norm2), 38-61 (l2sqr::apply) */
float kgo_dot(const float *a, const float *b, unsigned d);
float kgo_norm2(const float *a, unsigned d);
float kgo_l2sqr(const float *a, const float *b, unsigned d);

/* NDArrayOracle ctor, python-api.cpp:110-114: per-row norm term. */
void kgo_norms(const float *X, unsigned n, unsigned d, int metric, float *norms);
/* python-api.cpp:123-125 / kgraph-data.h:325-327: distance between rows i, j. */
float kgo_pair(const float *X, const float *norms, unsigned d, int metric, unsigned i, unsigned j);
/* python-api.cpp:105-107 / kgraph-data.h:315-317: distance query -> row i. */
float kgo_query_dist(const float *X, const float *norms, unsigned d, int metric,
                     const float *q, float qnorm, unsigned i);
float kgo_query_norm(const float *q, unsigned d, int metric);

/* SearchOracle::search, kgraph.cpp:231-252 (brute force with epsilon).
 * Returns the number of results (<= K). */
unsigned kgo_bruteforce(const float *X, const float *norms, unsigned n, unsigned d, int metric,
                        const float *q, unsigned K, float epsilon, uint32_t *ids, float *dists);

/* LinearSearch, kgraph.cpp:212-229: exact K-NN of row i, skipping i. */
void kgo_linear_search(const float *X, const float *norms, unsigned n, unsigned d, int metric,
                       unsigned i, unsigned K, uint32_t *ids, float *dists);

/* GenRandom, kgraph.cpp:44-65, driven by std::mt19937(seed); `skip` draws of
 * whole GenRandom(size) calls are made first (to reach trial t of a search). */
void kgo_genrandom(unsigned seed, unsigned size, unsigned N, unsigned calls, uint32_t *out);

/* KGraphImpl::search, kgraph.cpp:423-564, on a CSR graph (offsets[n+1],
 * nbr[E]) with per-node M.  ids is also the input when init > 0.
 * Returns the number of results; *cost = SearchInfo.cost.  Returns
 * 0xFFFFFFFF on a reference exception (bad init), message in kgo_last_error. */
unsigned kgo_search(const float *X, const float *norms, unsigned n, unsigned d, int metric,
                    const uint64_t *offsets, const uint32_t *nbr, const uint32_t *M,
                    const float *q, unsigned K, unsigned P, unsigned Mp, unsigned S, unsigned T,
                    float epsilon, unsigned seed, unsigned init,
                    uint32_t *ids, float *dists, float *cost);

/* KGraphConstructor, kgraph.cpp:705-1001, exactly as the reference runs it on
 * ONE OpenMP thread (thread 0 rng = mt19937(seed ^ 0); random_shuffle on the
 * C library rand(), reseeded here with srand(rand_seed) first).
 * Output CSR graph: call with offsets == NULL to get the edge count in *E
 * after the build; the graph is kept until the next call of kgo_build.
 * info[7] = stop_condition, iterations, cost, recall, accuracy, delta, M.
 * log (may be NULL) receives one row of 9 floats per iteration: iteration,
 * recall, accuracy, cost, M, delta, one-recall, one-ratio, 0. */
int kgo_build(const float *X, const float *norms, unsigned n, unsigned d, int metric,
              unsigned iterations, unsigned L, unsigned K, unsigned S, unsigned R,
              unsigned controls, unsigned seed, float delta, float recall,
              unsigned prune, int reverse, unsigned rand_seed,
              uint64_t *E, float *info, float *log, unsigned log_cap);
/* Copies the graph made by the last kgo_build (offsets[n+1], ids, dists, M). */
void kgo_build_result(uint64_t *offsets, uint32_t *ids, float *dists, uint32_t *M);

/* KGraphImpl::reverse, kgraph.cpp:667-702, on a CSR graph with distances.
 * Output into the same result store as kgo_build (fetch with kgo_build_result
 * after kgo_reverse returns the new edge count). */
uint64_t kgo_reverse(unsigned n, const uint64_t *offsets, const uint32_t *ids, const float *dists,
                     const uint32_t *M, int rev_k);

/* KGraphImpl::prune1 / prune2, kgraph.cpp:584-665.  Same result store. */
uint64_t kgo_prune(unsigned n, const uint64_t *offsets, const uint32_t *ids, const float *dists,
                   const uint32_t *M, unsigned level);

/* Nhood::parallel_try_insert (kgraph.cpp:723-736) of n_off offers (cand[k],
 * dist[k]) in the given order into one pool of Lp = L+1 entries (ids with the
 * new-flag in bit 31), its list length *L and *radius; r_out[k] = the
 * reference's return value (pool.size() for a radius rejection, L+1 for a
 * duplicate, else the insert position). */
void kgo_serial_inserts(unsigned Lp, float *pool_d, uint32_t *pool_i, unsigned *L, float *radius, unsigned n_off,
                        const uint32_t *cand, const float *dist, uint32_t *r_out);

/* libstdc++ std::sort by dist on (dist, id) pairs -- what the reference's
 * sort(pool) / sort(knn) calls do (kgraph.cpp:476, 697, 793). */
void kgo_std_sort_pairs(float *dists, uint32_t *ids, unsigned n);

const char *kgo_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
