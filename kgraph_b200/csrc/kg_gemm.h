// Tensor-core GEMM for the router (kg_gemm.cu).
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

namespace kgb {

// C[M,N] = op(A)[M,K] * op(B)[K,N] (+ beta * C) (+ bias[N]) (ReLU) on tcgen05:
// BF16 operands, FP32 accumulation in TMEM, FP32 C and optional BF16 copy Cb
// (same ldc).  ta / tb: A / B stored transposed (K x M / N x K row-major).  A
// tensor-core wait that runs out sets ERR_TC_TIMEOUT in *err.  ws (ws_bytes,
// may be null) is device scratch for the K-split partial tiles; with less than
// tc_gemm_workspace_bytes(M, N, K) the product is split less (or not at all).
void tc_gemm(cudaStream_t st, int M, int N, int K, const __nv_bfloat16 *A, int lda, int ta, const __nv_bfloat16 *B,
             int ldb, int tb, float *C, int ldc, __nv_bfloat16 *Cb, const float *bias, int relu, float beta, float *ws,
             size_t ws_bytes, uint32_t *err);
// Scratch bytes tc_gemm uses for its K split of an M x N x K product (0: not split).
size_t tc_gemm_workspace_bytes(int M, int N, int K);

// k-means assignment on tcgen05: lab[r] = argmin_c cn[c] - 2 F[r].cent[c]
// (ties: smaller c), best[r] that value; F is n x D, cent C x D (BF16,
// row-major), D <= 256.  false when the shape is not supported (the caller then
// uses tc_gemm and a separate argmin).
bool tc_assign(cudaStream_t st, int n, int D, const __nv_bfloat16 *F, const __nv_bfloat16 *cent, int C, const float *cn,
               int32_t *lab, float *best, uint32_t *err);

}  // namespace kgb
