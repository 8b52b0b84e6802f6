// Exact brute-force k-NN on the tensor cores (kg_bruteforce.cu).
#pragma once
#include <cstdint>
#include <cstddef>

struct kg_ctx;

namespace kgb {

constexpr uint32_t BF_MAX_K = 128;   // K the tensor-core path keeps per query (larger K: the CUDA-core scan)

// Whether the tensor-core path serves K on this context's dataset (shared memory fits).
bool bruteforce_tc_supported(const kg_ctx *ctx, uint32_t K);
size_t bruteforce_tc_smem(uint32_t ld, uint32_t K);
// The dataset's BF16 rows and row terms (once per dataset version).
int bruteforce_prepare(kg_ctx *ctx);
// SearchOracle::search (kgraph.cpp:231-252) for nq device queries (rows of q_ld
// floats): enqueues the sweeps and the FP32 recheck on the context's stream;
// outputs are device rows of out_ld.  work[0] receives the FP32 evaluations.
int bruteforce_tc(kg_ctx *ctx, const float *Q, uint32_t q_ld, uint32_t nq, uint32_t K, float epsilon,
                  uint32_t *out_ids, float *out_d, uint32_t *out_cnt, float *out_cost, uint32_t out_ld,
                  unsigned long long *work);

}  // namespace kgb
