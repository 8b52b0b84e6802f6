// Check entry points of the router's tensor-core products (kg_gemm.cu): the
// tcgen05 GEMM and the fused k-means assignment, run on caller data so tests
// can compare them with an independent FP64 evaluation at any shape (the
// router's own training shapes included).  No counterpart in the reference.
#include <cuda_bf16.h>
#include "kg_ctx.h"
#include "kg_gemm.h"

using namespace kgb;

namespace {
struct Guard {
    kg_ctx *c;
    explicit Guard(kg_ctx *ctx) : c(ctx) { c->mu.lock(); cudaSetDevice(c->device); }
    ~Guard() { c->mu.unlock(); }
};
// Device copies of the check's operands, freed on scope exit.
struct Tmp {
    void *p = nullptr;
    cudaError_t alloc(size_t b) { return cudaMalloc(&p, b < 16 ? 16 : b); }
    ~Tmp() { if (p) cudaFree(p); }
};
}  // namespace

extern "C" int kg_tc_gemm_check(kg_ctx *ctx, int M, int N, int K, const uint16_t *A, int lda, int ta,
                                const uint16_t *B, int ldb, int tb, const float *bias, int relu, float beta, float *C,
                                int ldc) {
    if (!ctx) return KG_E_INVALID;
    Guard g(ctx);
    if (M <= 0 || N <= 0 || K < 0 || !A || !B || !C || lda <= 0 || ldb <= 0 || ldc < N)
        return set_error(ctx, KG_E_INVALID, "bad GEMM shape");
    const size_t a_el = (size_t)(ta ? K : M) * lda, b_el = (size_t)(tb ? N : K) * ldb, c_el = (size_t)M * ldc;
    Tmp dA, dB, dC, dbias, dws;
    const size_t wsb = tc_gemm_workspace_bytes(M, N, K);
    cudaError_t e;
    if ((e = dA.alloc(a_el * 2)) != cudaSuccess || (e = dB.alloc(b_el * 2)) != cudaSuccess ||
        (e = dC.alloc(c_el * 4)) != cudaSuccess || (bias && (e = dbias.alloc((size_t)N * 4)) != cudaSuccess) ||
        (wsb && (e = dws.alloc(wsb)) != cudaSuccess))
        return cuda_fail(ctx, e, "alloc");
    cudaStream_t st = ctx->stream;
    cudaMemcpyAsync(dA.p, A, a_el * 2, cudaMemcpyDefault, st);
    cudaMemcpyAsync(dB.p, B, b_el * 2, cudaMemcpyDefault, st);
    cudaMemcpyAsync(dC.p, C, c_el * 4, cudaMemcpyDefault, st);
    if (bias) cudaMemcpyAsync(dbias.p, bias, (size_t)N * 4, cudaMemcpyDefault, st);
    tc_gemm(st, M, N, K, static_cast<const __nv_bfloat16 *>(dA.p), lda, ta, static_cast<const __nv_bfloat16 *>(dB.p),
            ldb, tb, static_cast<float *>(dC.p), ldc, nullptr, bias ? static_cast<const float *>(dbias.p) : nullptr,
            relu, beta, static_cast<float *>(dws.p), wsb, ctx->errw.as<uint32_t>());
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "tc_gemm launch");
    cudaMemcpyAsync(C, dC.p, c_el * 4, cudaMemcpyDefault, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "tc_gemm");
    return check_device_error(ctx, "tc_gemm");
}

extern "C" int kg_tc_assign_check(kg_ctx *ctx, const uint16_t *F, int n, int D, const uint16_t *cent, int C,
                                  const float *cn, int32_t *lab, float *best) {
    if (!ctx) return KG_E_INVALID;
    Guard g(ctx);
    if (n <= 0 || D <= 0 || D > 256 || C <= 0 || !F || !cent || !cn || !lab)
        return set_error(ctx, KG_E_INVALID, "bad assignment shape (D <= 256)");
    Tmp dF, dc, dcn, dl, db;
    cudaError_t e;
    if ((e = dF.alloc((size_t)n * D * 2)) != cudaSuccess || (e = dc.alloc((size_t)C * D * 2)) != cudaSuccess ||
        (e = dcn.alloc((size_t)C * 4)) != cudaSuccess || (e = dl.alloc((size_t)n * 4)) != cudaSuccess ||
        (e = db.alloc((size_t)n * 4)) != cudaSuccess)
        return cuda_fail(ctx, e, "alloc");
    cudaStream_t st = ctx->stream;
    cudaMemcpyAsync(dF.p, F, (size_t)n * D * 2, cudaMemcpyDefault, st);
    cudaMemcpyAsync(dc.p, cent, (size_t)C * D * 2, cudaMemcpyDefault, st);
    cudaMemcpyAsync(dcn.p, cn, (size_t)C * 4, cudaMemcpyDefault, st);
    if (!tc_assign(st, n, D, static_cast<const __nv_bfloat16 *>(dF.p), static_cast<const __nv_bfloat16 *>(dc.p), C,
                   static_cast<const float *>(dcn.p), static_cast<int32_t *>(dl.p), static_cast<float *>(db.p),
                   ctx->errw.as<uint32_t>()))
        return set_error(ctx, KG_E_INVALID, "tc_assign: shape not supported");
    cudaMemcpyAsync(lab, dl.p, (size_t)n * 4, cudaMemcpyDefault, st);
    if (best) cudaMemcpyAsync(best, db.p, (size_t)n * 4, cudaMemcpyDefault, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "tc_assign");
    return check_device_error(ctx, "tc_assign");
}
