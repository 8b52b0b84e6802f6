// NN-descent state in HBM and the kernels that advance it (kg_build.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "kg_common.cuh"

namespace kgb {

// Pool entries: structure of arrays, row stride PS (= L+1 rounded up to 8).
// Slot L of each row is the reference's overflow slot (pool.back()).  An
// unset slot holds UNSET_ID (flag clear) and +FLT_MAX.
constexpr uint32_t UNSET_ID = 0x7FFFFFFFu;

struct BuildState {
    DataView D;
    float *pool_d;
    uint32_t *pool_i;           // id | FLAG_BIT
    uint32_t PS, L, Lp, K, S, R;
    uint32_t *nodeL, *nodeM;
    float *radius, *radiusM;
    uint32_t *found, *lock;
    uint32_t *nn_new, *cnt_new, NEWCAP;
    uint32_t *nn_old, *cnt_old, OLDCAP;
    uint32_t *rcnt_new, *rcnt_old;       // reverse-sample counts, then cursors
    uint64_t *roff_new, *roff_old;       // exclusive scans of the counts (N+1)
    uint32_t *rbuf_new, *rbuf_old;       // reverse samples, CSR by target
    unsigned long long *n_comps;         // join pair counter
    unsigned long long *stat;            // [0] flagged-in-top-K count, [1] sum of M, [2] full pools
    unsigned long long *list_entries;    // join list entries (|new| + |old| summed over nodes and iterations)
    unsigned long long *inserts;         // [0] locked insert attempts, [1] of those landed (both cumulative)
    uint32_t *err;
    uint32_t *work;                      // dynamic work counter
    uint64_t seed;
    uint32_t *iter;                      // iteration number, advanced on the device
                                         // so that one captured graph serves every iteration
    struct JoinTcStats *tc;              // tensor-core join counters (kg_join_tc.cu)
    // Deferred inserts of the FP32 join (null off_lin: every insert is locked).
    // The join appends each offer that passes the unlocked radius test to
    // off_lin ({target, candidate, distance bits, source node | OFFER_UU}) while
    // off_cursor stays below off_cap (the excess takes the locked path) and
    // counts it in off_cnt[target]; the offers are then grouped by target into
    // off_grp (off_pos: exclusive scan of off_cnt; off_fill: cursors) and each
    // pool takes its offers in one merge (offer_merge_kernel).
    uint4 *off_lin, *off_grp;
    unsigned long long *off_cursor, off_cap;
    uint32_t *off_cnt, *off_fill, *mg_work;
    uint64_t *off_pos;
    uint32_t mg_warp_bytes;              // shared memory per merging warp
    uint32_t jt_rows;                    // rows the shared-memory join stages per node (0: join_kernel)
    uint32_t node_lo, node_hi;           // the join's nodes in this round (deferred joins go in rounds
                                         // whose offers fit the record buffer)
};
// Source-node word of a deferred offer: set when the offer is the pair's
// x <- y insert, whose position decides the source node's `found`.
constexpr uint32_t OFFER_UU = 0x80000000u;

// Counters of the tensor-core join, accumulated over a build.  Errors are of
// the BF16 tile distance against an FP64 evaluation of the same pair, on a
// sample of nodes; `violations` counts pairs whose tile error exceeded the
// recheck margin (sampled pairs and rechecked pairs).
struct JoinTcStats {
    unsigned long long pairs, rechecked, sampled, violations, rel_count;
    double sum_abs, sum_ratio, sum_rel;
    unsigned int max_abs_bits, max_ratio_bits, max_rel_bits, pad;
};

// Candidate pairs between the two phases of a tensor-core join round.  A
// round covers the nodes [bounds[r], bounds[r+1]), chosen from prefix sums of
// each node's worst-case pair count so that the round's pairs fit the queue.
struct JoinQueue {
    uint32_t *x, *y, *n;
    unsigned long long *tail;
    uint32_t *work;      // claim counter within a round
    uint32_t *bounds;    // round boundaries (node ids)
};
constexpr int JOIN_TC_MAX_CTAS_PER_SM = 3;
// Fraction of full pools (finite radii) from which an iteration's join runs
// on the tensor cores.
constexpr double JOIN_TC_MIN_FULL = 0.5;

// One round of the tensor-core local join (kg_join_tc.cu): the filter over the
// round's nodes (prec 0: BF16 tiles; 1: E4M3 tiles with per-row scales), then
// the inserts of the queued pairs.
cudaError_t launch_join_tc(int num_sms, int grid_insert, cudaStream_t st, const BuildState &s, JoinQueue jq,
                           uint32_t round, int prec);
// worst[n] = node n's largest pair count (n < N), worst[N] = 0.
cudaError_t join_tc_worst(cudaStream_t st, const BuildState &s, uint64_t *worst);
// bounds[0..R] from the exclusive prefix `pre` of worst (R rounds of <= slab).
cudaError_t join_tc_bounds(cudaStream_t st, const uint64_t *pre, uint32_t N, uint64_t slab, uint32_t R,
                           uint32_t *bounds);
// Whether the tensor-core join supports this state (shared memory fits).
bool join_tc_supported(const BuildState &s, int prec);
// Largest number of join pairs one node can produce.
uint64_t join_tc_node_max(const BuildState &s);

}  // namespace kgb
