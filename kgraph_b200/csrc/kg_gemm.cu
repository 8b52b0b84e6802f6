// BF16 x BF16 -> FP32 GEMM on the fifth-generation tensor cores (tcgen05),
// for the learned router: k-means assignment against the centroids and the
// MLP's forward and backward products (kg_router.cu).
//
// C[M,N] = op(A)[M,K] * op(B)[K,N] (+ beta * C) (+ bias[N]) (ReLU), FP32 out,
// optional BF16 copy.  op(A) = A (row-major, lda) or A^T (A is K x M); same for
// B.  One CTA of 4 warps owns a 128 x 128 tile of C: its accumulator lives in
// 128 TMEM columns.  K advances in chunks of 64: the threads stage the A and B
// chunks into shared memory in the K-major core-matrix layout (kg_tc.cuh),
// transposing where op() asks for it and zero-filling past M, N and K; one
// elected thread issues the four K=16 MMAs of the chunk and commits them to an
// mbarrier that every thread waits on (bounded: a wait that runs out sets
// ERR_TC_TIMEOUT in the error word and the CTA stops accumulating).  The
// epilogue reads the tile back with tcgen05.ld, warp w holding rows 32w..32w+31.
#include <cuda_bf16.h>
#include "kg_common.cuh"
#include "kg_gemm.h"
#include "kg_tc.cuh"

namespace kgb {
namespace {

constexpr int GM = 128, GN = 128, GKC = 64;
constexpr int G_THREADS = 128;
constexpr long long G_WAIT_CYCLES = 2000000000ll;   // ~1 s at 2 GHz

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// Stages rows [r0, r0 + 128) x K [k0, k0 + 64) of op(X) (rows x K, element
// (r, k) = t ? X[k * ld + r] : X[r * ld + k]) into `tile`, zero outside.
__device__ __forceinline__ void stage_tile(uint8_t *tile, const __nv_bfloat16 *X, int ld, int t, int rows, int K,
                                           int r0, int k0, int tid) {
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
    for (int e = tid; e < GM * (GKC / 8); e += G_THREADS) {
        const int r = e / (GKC / 8), k8 = e % (GKC / 8);
        const int gr = r0 + r;
        __nv_bfloat16 v[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int gk = k0 + 8 * k8 + i;
            v[i] = (gr < rows && gk < K) ? (t ? X[(size_t)gk * ld + gr] : X[(size_t)gr * ld + gk]) : zero;
        }
        uint4 pk;
        pk.x = pack2(v[0], v[1]); pk.y = pack2(v[2], v[3]);
        pk.z = pack2(v[4], v[5]); pk.w = pack2(v[6], v[7]);
        *reinterpret_cast<uint4 *>(tile + tc::kmajor_off(r, 8 * k8, GKC)) = pk;
    }
}

__global__ void __launch_bounds__(G_THREADS) tc_gemm_kernel(int M, int N, int K, const __nv_bfloat16 *A, int lda,
                                                            int ta, const __nv_bfloat16 *B, int ldb, int tb, float *C,
                                                            int ldc, __nv_bfloat16 *Cb, const float *bias, int relu,
                                                            float beta, uint32_t *err) {
    __shared__ __align__(1024) uint8_t sA[GM * GKC * 2];
    __shared__ __align__(1024) uint8_t sB[GN * GKC * 2];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * GM, n0 = blockIdx.x * GN;
    if (warp == 0) tc::tmem_alloc(&tmem_base, GN);
    if (tid == 0) tc::mbar_init(&mbar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    uint32_t phase = 0;
    bool ok = true;
    for (int k0 = 0; k0 < K && ok; k0 += GKC) {
        stage_tile(sA, A, lda, ta, M, K, m0, k0, tid);
        stage_tile(sB, B, ldb, !tb, N, K, n0, k0, tid);   // rows of op(B)^T: (n, k) = op(B)[k][n]
        tc::fence_async_shared();   // the generic-proxy stores, visible to the MMA
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t idesc = tc::idesc_bf16_f32(GM, GN);
            const uint32_t aa = tc::smem_addr(sA), ba = tc::smem_addr(sB);
#pragma unroll
            for (int kk = 0; kk < GKC / 16; ++kk)
                tc::mma_bf16(tmem, tc::smem_desc(aa + kk * 256, 128, GKC * 16), tc::smem_desc(ba + kk * 256, 128, GKC * 16),
                             idesc, (k0 > 0 || kk > 0) ? 1u : 0u);
            tc::mma_commit(&mbar);
        }
        const bool done = tc::mbar_wait(&mbar, phase, G_WAIT_CYCLES);
        ok = !__syncthreads_or(!done);   // the shared tiles are rewritten only after the MMAs read them
        phase ^= 1;
        tc::fence_after_sync();
    }
    if (!ok) {
        if (tid == 0) raise_error(err, ERR_TC_TIMEOUT);
    } else if (K > 0) {
        const int row = m0 + 32 * warp + lane;
        for (int part = 0; part < GN / 32; ++part) {
            if (n0 + 32 * part >= N) break;   // uniform over the CTA
            float v[32];
            tc::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + 32 * part, v);
            if (row < M) {
#pragma unroll
                for (int c = 0; c < 32; ++c) {
                    const int col = n0 + 32 * part + c;
                    if (col >= N) break;
                    float x = v[c];
                    if (beta != 0.f) x += beta * C[(size_t)row * ldc + col];
                    if (bias) x += bias[col];
                    if (relu) x = fmaxf(x, 0.f);
                    C[(size_t)row * ldc + col] = x;
                    if (Cb) Cb[(size_t)row * ldc + col] = __float2bfloat16_rn(x);
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tmem, GN);
}

}  // namespace

void tc_gemm(cudaStream_t st, int M, int N, int K, const __nv_bfloat16 *A, int lda, int ta, const __nv_bfloat16 *B,
             int ldb, int tb, float *C, int ldc, __nv_bfloat16 *Cb, const float *bias, int relu, float beta,
             uint32_t *err) {
    if (M <= 0 || N <= 0) return;
    const dim3 grid((N + GN - 1) / GN, (M + GM - 1) / GM);
    tc_gemm_kernel<<<grid, G_THREADS, 0, st>>>(M, N, K, A, lda, ta, B, ldb, tb, C, ldc, Cb, bias, relu, beta, err);
}

}  // namespace kgb
