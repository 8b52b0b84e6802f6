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

// Stages rows [r0, r0 + 128) x K [k0, k0 + KC) of op(X) (rows x K, element
// (r, k) = t ? X[k * ld + r] : X[r * ld + k]) into `tile` (K-major layout of
// KC columns), zero outside.  Untransposed rows whose 8 elements are in range
// and 16-byte aligned are read as one 16-byte load.
template <int KC, int NT>
__device__ __forceinline__ void stage_tile(uint8_t *tile, const __nv_bfloat16 *X, int ld, int t, int rows, int K,
                                           int r0, int k0, int tid) {
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
    const bool vec = !t && (ld & 7) == 0 && (reinterpret_cast<uintptr_t>(X) & 15) == 0;
    for (int e = tid; e < GM * (KC / 8); e += NT) {
        const int r = e / (KC / 8), k8 = e % (KC / 8);
        const int gr = r0 + r;
        if (vec) {
            const int gk = k0 + 8 * k8;
            uint4 pk = make_uint4(0u, 0u, 0u, 0u);
            if (gr < rows && gk + 8 <= K) {
                pk = *reinterpret_cast<const uint4 *>(X + (size_t)gr * ld + gk);
                *reinterpret_cast<uint4 *>(tile + tc::kmajor_off(r, 8 * k8, KC)) = pk;
                continue;
            }
        }
        __nv_bfloat16 v[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int gk = k0 + 8 * k8 + i;
            v[i] = (gr < rows && gk < K) ? (t ? X[(size_t)gk * ld + gr] : X[(size_t)gr * ld + gk]) : zero;
        }
        uint4 pk;
        pk.x = pack2(v[0], v[1]); pk.y = pack2(v[2], v[3]);
        pk.z = pack2(v[4], v[5]); pk.w = pack2(v[6], v[7]);
        *reinterpret_cast<uint4 *>(tile + tc::kmajor_off(r, 8 * k8, KC)) = pk;
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
        stage_tile<GKC, G_THREADS>(sA, A, lda, ta, M, K, m0, k0, tid);
        stage_tile<GKC, G_THREADS>(sB, B, ldb, !tb, N, K, n0, k0, tid);   // rows of op(B)^T: (n, k) = op(B)[k][n]
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

// k-means assignment: for 128 rows of F per CTA, the centroid c minimising
// cn[c] - 2 f.c over all C centroids (ties: smaller c).  The rows' tile stays
// in shared memory; centroid tiles of 128 stream through a second buffer, each
// tile's products land in TMEM and the epilogue folds them into a running
// minimum per row (thread = row): no product matrix is written.  D <= 256.
constexpr int A_THREADS = 128;
__global__ void __launch_bounds__(A_THREADS) tc_assign_kernel(const __nv_bfloat16 *F, int n, int D,
                                                              const __nv_bfloat16 *cent, int C, const float *cn,
                                                              int32_t *lab, float *best, uint32_t *err) {
    extern __shared__ __align__(1024) uint8_t asmem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Dp = (D + 15) / 16 * 16;
    uint8_t *sA = asmem, *sB = asmem + GM * Dp * 2;
    // rows of 16-byte multiples: every 8-element piece inside the row is one 16-byte load, the
    // padding past D (when D is not a multiple of 16) is zero
    const bool vec = (D & 7) == 0 && (reinterpret_cast<uintptr_t>(F) & 15) == 0 &&
                     (reinterpret_cast<uintptr_t>(cent) & 15) == 0;
    const int m0 = blockIdx.x * GM;
    if (warp == 0) tc::tmem_alloc(&tmem_base, GN);
    if (tid == 0) tc::mbar_init(&mbar, 1);
    // the rows' tile, once (K-major over the whole padded width)
    for (int kc = 0; kc < Dp; kc += 16) {
        // stage_tile works in KC-column layouts; the rows tile uses Dp columns, filled 16 at a time
        for (int e = tid; e < GM * 2; e += A_THREADS) {
            const int r = e >> 1, k8 = kc / 8 + (e & 1);
            const int gr = m0 + r;
            uint4 pk = make_uint4(0u, 0u, 0u, 0u);
            if (vec) {
                if (gr < n && 8 * k8 < D) pk = *reinterpret_cast<const uint4 *>(F + (size_t)gr * D + 8 * k8);
            } else if (gr < n) {
                __nv_bfloat16 v[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int gk = 8 * k8 + i;
                    v[i] = gk < D ? F[(size_t)gr * D + gk] : __float2bfloat16_rn(0.f);
                }
                pk.x = pack2(v[0], v[1]); pk.y = pack2(v[2], v[3]);
                pk.z = pack2(v[4], v[5]); pk.w = pack2(v[6], v[7]);
            }
            *reinterpret_cast<uint4 *>(sA + tc::kmajor_off(r, 8 * k8, Dp)) = pk;
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    uint32_t phase = 0;
    bool ok = true;
    float bv = INFINITY;
    int bi = 0;
    const int row = m0 + 32 * warp + lane;
    for (int c0 = 0; c0 < C && ok; c0 += GN) {
        for (int e = tid; e < GN * (Dp / 8); e += A_THREADS) {
            const int r = e / (Dp / 8), k8 = e % (Dp / 8);
            const int gc = c0 + r;
            uint4 pk = make_uint4(0u, 0u, 0u, 0u);
            if (vec) {
                if (gc < C && 8 * k8 < D) pk = *reinterpret_cast<const uint4 *>(cent + (size_t)gc * D + 8 * k8);
            } else if (gc < C) {
                __nv_bfloat16 v[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int gk = 8 * k8 + i;
                    v[i] = gk < D ? cent[(size_t)gc * D + gk] : __float2bfloat16_rn(0.f);
                }
                pk.x = pack2(v[0], v[1]); pk.y = pack2(v[2], v[3]);
                pk.z = pack2(v[4], v[5]); pk.w = pack2(v[6], v[7]);
            }
            *reinterpret_cast<uint4 *>(sB + tc::kmajor_off(r, 8 * k8, Dp)) = pk;
        }
        tc::fence_async_shared();
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            const uint32_t idesc = tc::idesc_bf16_f32(GM, GN);
            const uint32_t aa = tc::smem_addr(sA), ba = tc::smem_addr(sB);
            for (int kk = 0; kk < Dp / 16; ++kk)
                tc::mma_bf16(tmem, tc::smem_desc(aa + kk * 256, 128, Dp * 16), tc::smem_desc(ba + kk * 256, 128, Dp * 16),
                             idesc, kk > 0 ? 1u : 0u);
            tc::mma_commit(&mbar);
        }
        const bool done = tc::mbar_wait(&mbar, phase, G_WAIT_CYCLES);
        ok = !__syncthreads_or(!done);
        phase ^= 1;
        tc::fence_after_sync();
        if (!ok) break;
        for (int part = 0; part < GN / 32; ++part) {
            if (c0 + 32 * part >= C) break;   // uniform
            float v[32];
            tc::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + 32 * part, v);
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const int c = c0 + 32 * part + j;
                if (c < C) {
                    const float d = cn[c] - 2.f * v[j];
                    if (d < bv) { bv = d; bi = c; }
                }
            }
        }
        tc::fence_before_sync();
        __syncthreads();   // the TMEM tile and the centroid buffer are reused by the next tile
        tc::fence_after_sync();
    }
    if (!ok) {
        if (tid == 0) raise_error(err, ERR_TC_TIMEOUT);
    } else if (row < n) {
        lab[row] = bi;
        if (best) best[row] = bv;
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_free(tmem, GN);
}

}  // namespace

bool tc_assign(cudaStream_t st, int n, int D, const __nv_bfloat16 *F, const __nv_bfloat16 *cent, int C, const float *cn,
               int32_t *lab, float *best, uint32_t *err) {
    if (D > 256 || n <= 0) return false;
    const int Dp = (D + 15) / 16 * 16;
    const size_t smem = (size_t)2 * GM * Dp * 2;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(tc_assign_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return false;
    tc_assign_kernel<<<(n + GM - 1) / GM, A_THREADS, smem, st>>>(F, n, D, cent, C, cn, lab, best, err);
    return cudaGetLastError() == cudaSuccess;
}

void tc_gemm(cudaStream_t st, int M, int N, int K, const __nv_bfloat16 *A, int lda, int ta, const __nv_bfloat16 *B,
             int ldb, int tb, float *C, int ldc, __nv_bfloat16 *Cb, const float *bias, int relu, float beta,
             uint32_t *err) {
    if (M <= 0 || N <= 0) return;
    const dim3 grid((N + GN - 1) / GN, (M + GM - 1) / GM);
    tc_gemm_kernel<<<grid, G_THREADS, 0, st>>>(M, N, K, A, lda, ta, B, ldb, tb, C, ldc, Cb, bias, relu, beta, err);
}

}  // namespace kgb
