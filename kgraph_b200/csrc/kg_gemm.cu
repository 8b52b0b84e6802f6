// BF16 x BF16 -> FP32 GEMM on the fifth-generation tensor cores (tcgen05),
// for the learned router: k-means assignment against the centroids and the
// MLP's forward and backward products (kg_router.cu).
//
// C[M,N] = op(A)[M,K] * op(B)[K,N] (+ beta * C) (+ bias[N]) (ReLU), FP32 out,
// optional BF16 copy.  op(A) = A (row-major, lda) or A^T (A is K x M); same for
// B.  A CTA owns a 128 x 128 tile of C; its accumulator lives in 128 TMEM
// columns and the epilogue reads it back with tcgen05.ld, warp w (mod 4)
// holding rows 32w..32w+31.
//
// Main path (operands 16-byte aligned with row pitches of 16-byte multiples,
// which every router shape has): TMA.  One thread loads 64-wide K chunks of A
// and B into a ring of four shared-memory stages with cp.async.bulk.tensor
// (128-byte swizzle; an operand stored transposed is loaded as it lies and
// described MN-major to the MMA, so nothing is transposed by hand; the tensor
// map's bounds zero-fill past M, N and K), another thread issues the MMAs of a
// stage as soon as its bytes have landed and releases the stage through
// tcgen05.commit, so loads run ahead of the tensor core by up to four chunks.
// Products with few output tiles and a long K (the weight gradients: K = the
// batch) are split along K over more CTAs; each writes its partial tile to a
// workspace and a second kernel sums the partials in a fixed order (the
// result does not depend on scheduling).
//
// Fallback (any other alignment): the threads stage the A and B chunks into
// shared memory in the K-major core-matrix layout (kg_tc.cuh), transposing
// where op() asks for it and zero-filling past M, N and K, and one elected
// thread issues the chunk's MMAs.
//
// Every wait is bounded: one that runs out sets ERR_TC_TIMEOUT in the error
// word, the CTA stops issuing work, waits (bounded) for what it has in flight,
// frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>
#include <algorithm>
#include <atomic>
#include <mutex>
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

__global__ void __launch_bounds__(G_THREADS) staged_gemm_kernel(int M, int N, int K, const __nv_bfloat16 *A, int lda,
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
__global__ void __launch_bounds__(A_THREADS) staged_assign_kernel(const __nv_bfloat16 *F, int n, int D,
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


// ---------------------------------------------------------------------------
// TMA-fed kernels.  Warps 0-3: epilogue (TMEM lane quadrant = warp); warp 4,
// lane 0: TMA producer; warp 5: TMEM owner, lane 0 issues the MMAs.
constexpr int T_BK = 64;                      // K per stage: 64 BF16 = one 128-byte swizzle row
constexpr int T_ST = 4;                       // stages in the ring
constexpr int T_THREADS = 192;
constexpr uint32_t T_BOX = 128 * 128;         // bytes of one 128-row (or 2 x 64-column) operand box set
constexpr size_t T_SMEM = (size_t)T_ST * 2 * T_BOX + 1024;   // + alignment slack

__device__ __forceinline__ uint8_t *align1024(uint8_t *p) {
    return reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(p) + 1023) & ~(uintptr_t)1023);
}

// Descriptor of the K = 16 step kk of a 128 x 64 operand tile at saddr (layouts in kg_tc.cuh).
__device__ __forceinline__ uint64_t tile_desc(uint32_t saddr, int mn_major, int kk) {
    return mn_major ? tc::smem_desc_sw128(saddr + kk * 2048, 8192, 1024) : tc::smem_desc_sw128(saddr + kk * 32, 16, 1024);
}

// Loads the 128 x 64 tile of an operand whose rows of op() start at r0 and
// whose K chunk starts at k: K-major, one 64 x 128 box at (k, r0); MN-major,
// two 64 x 64 boxes at (r0, k) and (r0 + 64, k).
__device__ __forceinline__ void load_tile(uint8_t *dst, const CUtensorMap *map, int mn_major, int r0, int k,
                                          uint64_t *bar) {
    if (mn_major) {
        tc::tma_load_2d(dst, map, r0, k, bar);
        tc::tma_load_2d(dst + 8192, map, r0 + 64, k, bar);
    } else {
        tc::tma_load_2d(dst, map, k, r0, bar);
    }
}

// Bounded wait for the last phase armed on each stage that the producer issued.
__device__ void drain_stages(uint64_t *full, int issued, int stages) {
    for (int s = 0; s < stages && s < issued; ++s) {
        const int last = s + (issued - 1 - s) / stages * stages;
        tc::mbar_wait(&full[s], (uint32_t)(last / stages) & 1u, G_WAIT_CYCLES);
    }
}

__device__ __forceinline__ float gemm_epilogue(float x, const float *C, size_t at, const float *bias, int col, int relu,
                                               float beta) {
    if (beta != 0.f) x += beta * C[at];
    if (bias) x += bias[col];
    if (relu) x = fmaxf(x, 0.f);
    return x;
}

// grid (N tiles, M tiles, K splits); blockIdx.z covers K chunks [z * kc_per, min(nkc, (z + 1) * kc_per)), at
// least one.  ws == null: the full product with the epilogue; else the raw partial tile into ws[z][M][N].
__global__ void __launch_bounds__(T_THREADS, 1)
    tma_gemm_kernel(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tB, int M, int N, int K,
                    int a_mn, int b_mn, int kc_per, float *C, int ldc, __nv_bfloat16 *Cb, const float *bias, int relu,
                    float beta, float *ws, uint32_t *err) {
    extern __shared__ uint8_t tg_raw[];
    uint8_t *sm = align1024(tg_raw);
    __shared__ __align__(8) uint64_t full[T_ST], empty[T_ST], done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile uint32_t fail;
    __shared__ int issued;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * GM, n0 = blockIdx.x * GN;
    const int nkc = (K + T_BK - 1) / T_BK;
    const int kc0 = blockIdx.z * kc_per, iters = min(nkc, kc0 + kc_per) - kc0;
    if (warp == 5) tc::tmem_alloc(&tmem_base, GN);
    if (tid == 0) {
        for (int s = 0; s < T_ST; ++s) { tc::mbar_init(&full[s], 1); tc::mbar_init(&empty[s], 1); }
        tc::mbar_init(&done, 1);
        fail = 0;
        issued = 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    if (warp == 4 && lane == 0) {
        int i = 0;
        for (; i < iters && !fail; ++i) {
            const int s = i % T_ST;
            if (i >= T_ST && !tc::mbar_wait(&empty[s], ((uint32_t)(i / T_ST) & 1u) ^ 1u, G_WAIT_CYCLES)) {
                fail = 1;
                break;
            }
            uint8_t *a = sm + (size_t)s * 2 * T_BOX, *b = a + T_BOX;
            tc::mbar_expect_tx(&full[s], 2 * T_BOX);
            const int k = (kc0 + i) * T_BK;
            load_tile(a, &tA, a_mn, m0, k, &full[s]);
            load_tile(b, &tB, b_mn, n0, k, &full[s]);
        }
        issued = i;
    } else if (warp == 5 && lane == 0) {
        const uint32_t idesc = tc::idesc_bf16_f32_major(GM, GN, (uint32_t)a_mn, (uint32_t)b_mn);
        for (int i = 0; i < iters; ++i) {
            const int s = i % T_ST;
            if (fail || !tc::mbar_wait(&full[s], (uint32_t)(i / T_ST) & 1u, G_WAIT_CYCLES)) {
                fail = 1;
                break;
            }
            tc::fence_after_sync();
            const uint32_t a = tc::smem_addr(sm + (size_t)s * 2 * T_BOX), b = a + T_BOX;
#pragma unroll
            for (int kk = 0; kk < T_BK / 16; ++kk)
                tc::mma_bf16(tmem, tile_desc(a, a_mn, kk), tile_desc(b, b_mn, kk), idesc, (i > 0 || kk > 0) ? 1u : 0u);
            tc::mma_commit(&empty[s]);
        }
        tc::mma_commit(&done);   // arrives when every MMA issued above has completed
    }
    __syncthreads();   // the producer and the MMA issuer are done issuing: `fail` and `issued` are final
    const bool mma_done = tc::mbar_wait(&done, 0, G_WAIT_CYCLES);
    tc::fence_after_sync();
    const bool ok = mma_done && !fail;
    if (warp < 4 && ok) {
        const int row = m0 + 32 * warp + lane;
        for (int part = 0; part < GN / 32; ++part) {
            const int c0 = n0 + 32 * part;
            if (c0 >= N) break;   // uniform over the CTA
            float v[32];
            tc::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + 32 * part, v);
            if (row >= M) continue;
            const int nc = min(32, N - c0);
            if (ws) {
                float *w = ws + ((size_t)blockIdx.z * M + row) * N + c0;
#pragma unroll
                for (int c = 0; c < 32; ++c)
                    if (c < nc) w[c] = v[c];
            } else {
#pragma unroll
                for (int c = 0; c < 32; ++c) {
                    if (c >= nc) break;
                    const size_t at = (size_t)row * ldc + c0 + c;
                    const float x = gemm_epilogue(v[c], C, at, bias, c0 + c, relu, beta);
                    C[at] = x;
                    if (Cb) Cb[at] = __float2bfloat16_rn(x);
                }
            }
        }
    }
    if (!ok && tid == 0) raise_error(err, ERR_TC_TIMEOUT);
    if (fail && warp == 4 && lane == 0) drain_stages(full, issued, T_ST);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 5) tc::tmem_free(tmem, GN);
}

// C = sum over z of ws[z] (in order z = 0, 1, ...), then the epilogue.
__global__ void splitk_reduce_kernel(const float *ws, int S, int M, int N, float *C, int ldc, __nv_bfloat16 *Cb,
                                     const float *bias, int relu, float beta) {
    const size_t total = (size_t)M * N;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        float x = ws[e];
        for (int z = 1; z < S; ++z) x += ws[(size_t)z * total + e];
        const int row = (int)(e / N), col = (int)(e % N);
        const size_t at = (size_t)row * ldc + col;
        x = gemm_epilogue(x, C, at, bias, col, relu, beta);
        C[at] = x;
        if (Cb) Cb[at] = __float2bfloat16_rn(x);
    }
}

// k-means assignment with TMA: the CTA's 128 rows (D <= 256 as up to four
// 64-column boxes) stay resident; the centroid tiles stream through two
// stages; two TMEM accumulators let the epilogue fold tile t into the running
// argmin while the MMAs of tile t + 1 run.
constexpr int AS_ST = 2;
__global__ void __launch_bounds__(T_THREADS, 1)
    tma_assign_kernel(const __grid_constant__ CUtensorMap tF, const __grid_constant__ CUtensorMap tC, int n, int D,
                      int C, const float *cn, int32_t *lab, float *best, uint32_t *err) {
    extern __shared__ uint8_t ta_raw[];
    uint8_t *sm = align1024(ta_raw);
    __shared__ __align__(8) uint64_t fullA, full[AS_ST], empty[AS_ST], acc_full[2], acc_empty[2], done;
    __shared__ uint32_t tmem_base;
    __shared__ volatile uint32_t fail;
    __shared__ int issued;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nb = (D + 63) / 64;                 // 64-column boxes per row
    const int ksteps = (D + 15) / 16;             // K = 16 steps (zero columns past D beyond that are skipped)
    const uint32_t tile_bytes = (uint32_t)nb * T_BOX;
    uint8_t *sA = sm, *sB = sm + tile_bytes;      // sB: AS_ST stages of tile_bytes
    const int m0 = blockIdx.x * GM;
    const int ntiles = (C + GN - 1) / GN;
    if (warp == 5) tc::tmem_alloc(&tmem_base, 2 * GN);
    if (tid == 0) {
        tc::mbar_init(&fullA, 1);
        for (int s = 0; s < AS_ST; ++s) { tc::mbar_init(&full[s], 1); tc::mbar_init(&empty[s], 1); }
        for (int s = 0; s < 2; ++s) { tc::mbar_init(&acc_full[s], 1); tc::mbar_init(&acc_empty[s], 4); }
        tc::mbar_init(&done, 1);
        fail = 0;
        issued = 0;
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    float bv = INFINITY;
    int bi = 0;
    bool a_loaded = false;
    if (warp == 4 && lane == 0) {
        tc::mbar_expect_tx(&fullA, tile_bytes);
        for (int j = 0; j < nb; ++j) tc::tma_load_2d(sA + (size_t)j * T_BOX, &tF, 64 * j, m0, &fullA);
        a_loaded = true;
        int t = 0;
        for (; t < ntiles && !fail; ++t) {
            const int s = t % AS_ST;
            if (t >= AS_ST && !tc::mbar_wait(&empty[s], ((uint32_t)(t / AS_ST) & 1u) ^ 1u, G_WAIT_CYCLES)) {
                fail = 1;
                break;
            }
            uint8_t *b = sB + (size_t)s * tile_bytes;
            tc::mbar_expect_tx(&full[s], tile_bytes);
            for (int j = 0; j < nb; ++j) tc::tma_load_2d(b + (size_t)j * T_BOX, &tC, 64 * j, GN * t, &full[s]);
        }
        issued = t;
    } else if (warp == 5 && lane == 0) {
        const uint32_t idesc = tc::idesc_bf16_f32(GM, GN);
        bool go = tc::mbar_wait(&fullA, 0, G_WAIT_CYCLES);
        if (!go) fail = 1;
        const uint32_t a = tc::smem_addr(sA);
        for (int t = 0; t < ntiles && go; ++t) {
            const int s = t % AS_ST, acc = t & 1;
            if (fail || !tc::mbar_wait(&full[s], (uint32_t)(t / AS_ST) & 1u, G_WAIT_CYCLES) ||
                (t >= 2 && !tc::mbar_wait(&acc_empty[acc], ((uint32_t)(t / 2) & 1u) ^ 1u, G_WAIT_CYCLES))) {
                fail = 1;
                break;
            }
            tc::fence_after_sync();
            const uint32_t b = tc::smem_addr(sB + (size_t)s * tile_bytes);
            for (int kk = 0; kk < ksteps; ++kk) {
                const uint32_t off = (uint32_t)(kk >> 2) * T_BOX + (uint32_t)(kk & 3) * 32;
                tc::mma_bf16(tmem + (uint32_t)(acc * GN), tc::smem_desc_sw128(a + off, 16, 1024),
                             tc::smem_desc_sw128(b + off, 16, 1024), idesc, kk > 0 ? 1u : 0u);
            }
            tc::mma_commit(&empty[s]);
            tc::mma_commit(&acc_full[acc]);
        }
        tc::mma_commit(&done);
    } else if (warp < 4) {
        for (int t = 0; t < ntiles; ++t) {
            const int acc = t & 1;
            // bounded in slices, so that an MMA issuer that gave up (it sets `fail`) is noticed early
            bool got = false;
            for (long long spent = 0; !got && !fail && spent < G_WAIT_CYCLES; spent += 1000000)
                got = tc::mbar_wait(&acc_full[acc], (uint32_t)(t / 2) & 1u, 1000000);
            if (!got) { fail = 1; break; }
            tc::fence_after_sync();
            const int c0 = GN * t;
            for (int part = 0; part < GN / 32; ++part) {
                if (c0 + 32 * part >= C) break;   // uniform
                float v[32];
                tc::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(acc * GN + 32 * part), v);
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
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(&acc_empty[acc]);
        }
    }
    __syncthreads();
    const bool mma_done = tc::mbar_wait(&done, 0, G_WAIT_CYCLES);
    tc::fence_after_sync();
    const bool ok = mma_done && !fail;
    const int row = m0 + 32 * warp + lane;
    if (warp < 4 && ok && row < n) {
        lab[row] = bi;
        if (best) best[row] = bv;
    }
    if (!ok && tid == 0) raise_error(err, ERR_TC_TIMEOUT);
    if (fail && warp == 4 && lane == 0) {
        if (a_loaded) tc::mbar_wait(&fullA, 0, G_WAIT_CYCLES);
        drain_stages(full, issued, AS_ST);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 5) tc::tmem_free(tmem, 2 * GN);
}

// ---------------------------------------------------------------------------
// Host side.

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Tensor map of a row-major BF16 matrix (outer rows of `inner` elements, `ld`
// apart) with a box of box_inner x box_outer and the 128-byte swizzle.  False
// when TMA cannot address it (alignment) or the driver refuses it.
bool bf16_map(CUtensorMap *m, const void *base, uint64_t inner, uint64_t outer, uint64_t ld, uint32_t box_inner,
              uint32_t box_outer) {
    PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn || (reinterpret_cast<uintptr_t>(base) & 15) || (ld * 2) % 16 || inner == 0 || outer == 0) return false;
    const cuuint64_t dims[2] = {inner, outer};
    const cuuint64_t strides[1] = {ld * 2};
    const cuuint32_t box[2] = {box_inner, box_outer};
    const cuuint32_t es[2] = {1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Map of an operand as the TMA kernel reads it: K-major (op() rows x K, K
// contiguous) -> boxes of 64 (K) x 128 rows; MN-major (stored K x MN) -> boxes
// of 64 (MN) x 64 (K).
bool operand_map(CUtensorMap *m, const void *X, int ld, int mn_major, int rows, int K) {
    return mn_major ? bf16_map(m, X, (uint64_t)rows, (uint64_t)K, (uint64_t)ld, 64, 64)
                    : bf16_map(m, X, (uint64_t)K, (uint64_t)rows, (uint64_t)ld, 64, 128);
}

// Opts a kernel into more than 48 KB of dynamic shared memory, once per device,
// at the largest size any of its launches asks for.
bool allow_smem(const void *kernel, size_t bytes, std::atomic<uint32_t> &done_mask) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    const uint32_t bit = 1u << (dev & 31);
    if (done_mask.load() & bit) return true;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
        return false;
    done_mask.fetch_or(bit);
    return true;
}
std::atomic<uint32_t> g_gemm_smem{0}, g_assign_smem{0};

// K splits for a product: enough CTAs to cover the SMs when the output has few
// tiles, at least two K chunks per split.
int gemm_splits(int M, int N, int K) {
    const int tiles = ((M + GM - 1) / GM) * ((N + GN - 1) / GN);
    const int nkc = (K + T_BK - 1) / T_BK;
    int S = std::min(148 / std::max(tiles, 1), nkc / 2);
    return std::max(S, 1);
}

}  // namespace

size_t tc_gemm_workspace_bytes(int M, int N, int K) {
    if (M <= 0 || N <= 0 || K <= 0) return 0;
    const int S = gemm_splits(M, N, K);
    return S > 1 ? (size_t)S * M * N * sizeof(float) : 0;
}

bool tc_assign(cudaStream_t st, int n, int D, const __nv_bfloat16 *F, const __nv_bfloat16 *cent, int C, const float *cn,
               int32_t *lab, float *best, uint32_t *err) {
    if (D > 256 || n <= 0 || C <= 0) return false;
    CUtensorMap mF, mC;
    if (operand_map(&mF, F, D, 0, n, D) && operand_map(&mC, cent, D, 0, C, D)) {
        const size_t smem = (size_t)(1 + AS_ST) * ((D + 63) / 64) * T_BOX + 1024;
        if (allow_smem(reinterpret_cast<const void *>(tma_assign_kernel), (size_t)(1 + AS_ST) * 4 * T_BOX + 1024,
                       g_assign_smem)) {
            tma_assign_kernel<<<(n + GM - 1) / GM, T_THREADS, smem, st>>>(mF, mC, n, D, C, cn, lab, best, err);
            return cudaGetLastError() == cudaSuccess;
        }
    }
    const int Dp = (D + 15) / 16 * 16;
    const size_t smem = (size_t)2 * GM * Dp * 2;
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(staged_assign_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return false;
    staged_assign_kernel<<<(n + GM - 1) / GM, A_THREADS, smem, st>>>(F, n, D, cent, C, cn, lab, best, err);
    return cudaGetLastError() == cudaSuccess;
}

void tc_gemm(cudaStream_t st, int M, int N, int K, const __nv_bfloat16 *A, int lda, int ta, const __nv_bfloat16 *B,
             int ldb, int tb, float *C, int ldc, __nv_bfloat16 *Cb, const float *bias, int relu, float beta, float *ws,
             size_t ws_bytes, uint32_t *err) {
    if (M <= 0 || N <= 0) return;
    // op(A) rows are M (A K-major unless stored transposed); op(B)^T rows are N (B K-major when stored transposed)
    const int a_mn = ta ? 1 : 0, b_mn = tb ? 0 : 1;
    CUtensorMap mA, mB;
    if (K > 0 && operand_map(&mA, A, lda, a_mn, M, K) && operand_map(&mB, B, ldb, b_mn, N, K) &&
        allow_smem(reinterpret_cast<const void *>(tma_gemm_kernel), T_SMEM, g_gemm_smem)) {
        const int nkc = (K + T_BK - 1) / T_BK;
        int S = gemm_splits(M, N, K);
        if (S > 1 && (!ws || ws_bytes < (size_t)S * M * N * sizeof(float)))
            S = ws ? (int)std::min<size_t>(S, ws_bytes / ((size_t)M * N * sizeof(float))) : 1;
        if (S < 1) S = 1;
        const int kc_per = (nkc + S - 1) / S;
        S = (nkc + kc_per - 1) / kc_per;   // every split has at least one chunk
        const dim3 grid((N + GN - 1) / GN, (M + GM - 1) / GM, S);
        tma_gemm_kernel<<<grid, T_THREADS, T_SMEM, st>>>(mA, mB, M, N, K, a_mn, b_mn, kc_per, C, ldc, Cb, bias, relu,
                                                          beta, S > 1 ? ws : nullptr, err);
        if (S > 1) {
            const size_t total = (size_t)M * N;
            const int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 8);
            splitk_reduce_kernel<<<blocks, 256, 0, st>>>(ws, S, M, N, C, ldc, Cb, bias, relu, beta);
        }
        return;
    }
    const dim3 grid((N + GN - 1) / GN, (M + GM - 1) / GM);
    staged_gemm_kernel<<<grid, G_THREADS, 0, st>>>(M, N, K, A, lda, ta, B, ldb, tb, C, ldc, Cb, bias, relu, beta, err);
}

}  // namespace kgb
