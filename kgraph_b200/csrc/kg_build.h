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
    unsigned long long *stat;            // [0] flagged-in-top-K count, [1] sum of M
    uint32_t *err;
    uint32_t *work;                      // dynamic work counter
    uint64_t seed;
    uint32_t iteration;
};

}  // namespace kgb
