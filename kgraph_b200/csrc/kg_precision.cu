// Reduced-precision copies of the dataset for the search's distance filter.
//
// No counterpart in the reference (its search evaluates every candidate in
// FP32, kgraph.cpp:495-513).  With a filter precision set, the walk first
// evaluates each candidate against a compressed copy of its row -- BF16, or
// FP8 E4M3 with a per-row scale -- and turns that into a rigorous lower bound
// of the candidate's canonical FP32 distance (kg_search.cu).  Once the pool is
// full, a candidate whose bound is at or beyond the pool's last entry would
// land in the spare slot (kgraph.cpp:503-506) and is skipped; every other
// candidate is evaluated in FP32 exactly as without the filter.  Results are
// therefore identical to the FP32 walk; the filter only saves row reads.
//
// Per row the copy stores {e, scale, norm term, 0} (float4), where e bounds
// || x - y ||_2 for y the values the filter reconstructs in FP32:
//   BF16      y_i = bf16_rn(x_i) (exact in FP32);
//   FP8 E4M3  scale = max|x| / 448, q_i = e4m3_satfinite(x_i / scale),
//             y_i = fl32(q_i * scale).
// e is accumulated in FP64 (every y_i and x_i is exact there) and rounded up.
#include <cuda_bf16.h>
#include <cuda_fp8.h>
#include <cstring>
#include <vector>
#include "kg_ctx.h"

namespace kgb {
namespace {

__device__ __forceinline__ unsigned long long ordered_bits(double v) {
    unsigned long long u = (unsigned long long)__double_as_longlong(v);
    return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}

// One warp per row.  stats: [0] max relative error e / ||x|| (ordered bits),
// [1] sum of relative errors (double bits, atomicAdd), [2] rows with ||x|| > 0.
template <int PREC>
__global__ void quantize_kernel(DataView D, void *Xc, float4 *meta, unsigned long long *stats) {
    const int lane = threadIdx.x & 31;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; row < D.n; row += warps) {
        const float *x = D.X + (size_t)row * D.ld;
        float scale = 1.f;
        if (PREC == 2) {
            float mx = 0.f;
            for (uint32_t j = lane; j < D.d; j += 32) mx = fmaxf(mx, fabsf(x[j]));
            for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xFFFFFFFFu, mx, o));
            scale = mx > 0.f ? __fdiv_rn(mx, 448.f) : 1.f;
        }
        double e2 = 0.0, n2 = 0.0;
        for (uint32_t j = lane; j < D.ld; j += 32) {
            const float v = j < D.d ? x[j] : 0.f;
            float y;
            if (PREC == 1) {
                const __nv_bfloat16 b = __float2bfloat16_rn(v);
                reinterpret_cast<__nv_bfloat16 *>(Xc)[(size_t)row * D.ld + j] = b;
                y = __bfloat162float(b);
            } else {
                const __nv_fp8_storage_t q = __nv_cvt_float_to_fp8(__fdiv_rn(v, scale), __NV_SATFINITE, __NV_E4M3);
                reinterpret_cast<__nv_fp8_storage_t *>(Xc)[(size_t)row * D.ld + j] = q;
                const __half_raw h = __nv_cvt_fp8_to_halfraw(q, __NV_E4M3);
                y = __fmul_rn(__half2float(__half(h)), scale);
            }
            const double df = (double)v - (double)y;
            e2 += df * df;
            n2 += (double)v * (double)v;
        }
        for (int o = 16; o; o >>= 1) {
            e2 += __shfl_xor_sync(0xFFFFFFFFu, e2, o);
            n2 += __shfl_xor_sync(0xFFFFFFFFu, n2, o);
        }
        if (lane == 0) {
            // sqrt in FP64 is correctly rounded: one relative step of slack, then round up to FP32
            const float e = e2 > 0.0 ? __double2float_ru(sqrt(e2) * (1.0 + 1e-12)) : 0.f;
            meta[row] = make_float4(e, scale, D.norms[row], 0.f);
            if (n2 > 0.0) {
                const double rel = sqrt(e2 / n2);
                atomicMax(stats, ordered_bits(rel));
                atomicAdd(reinterpret_cast<double *>(stats + 1), rel);
                atomicAdd(stats + 2, 1ull);
            }
        }
    }
}

}  // namespace

// (Re)builds the compressed copy for ctx->search_prec when the data changed.
int ensure_search_precision(kg_ctx *ctx) {
    const int prec = ctx->search_prec;
    if (prec == KG_SEARCH_FP32 || (ctx->prec_built == prec && ctx->prec_data_version == ctx->data_version))
        return KG_OK;
    const size_t elem = prec == KG_SEARCH_BF16 ? 2 : 1;
    cudaError_t e;
    if ((e = ctx->Xc.reserve((size_t)ctx->n * ctx->ld * elem)) != cudaSuccess ||
        (e = ctx->cmeta.reserve((size_t)ctx->n * sizeof(float4))) != cudaSuccess ||
        (e = ctx->cstats.reserve(64)) != cudaSuccess)
        return cuda_fail(ctx, e, "alloc compressed rows");
    cudaStream_t st = ctx->stream;
    cudaMemsetAsync(ctx->cstats.p, 0, 64, st);
    const DataView D{ctx->X.as<float>(), ctx->norms.as<float>(), ctx->n, ctx->d, ctx->ld, ctx->metric};
    const int grid = ctx->num_sms * 8;
    auto *stats = ctx->cstats.as<unsigned long long>();
    if (prec == KG_SEARCH_BF16)
        quantize_kernel<1><<<grid, 256, 0, st>>>(D, ctx->Xc.p, ctx->cmeta.as<float4>(), stats);
    else
        quantize_kernel<2><<<grid, 256, 0, st>>>(D, ctx->Xc.p, ctx->cmeta.as<float4>(), stats);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "quantize");
    unsigned long long h[3] = {0, 0, 0};
    cudaMemcpyAsync(h, stats, sizeof(h), cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "quantize");
    const unsigned long long mb = (h[0] & 0x8000000000000000ull) ? (h[0] & ~0x8000000000000000ull) : ~h[0];
    double mx, sum;
    std::memcpy(&mx, &mb, 8);
    std::memcpy(&sum, &h[1], 8);
    ctx->prec_max_rel = h[2] ? mx : 0.0;
    ctx->prec_mean_rel = h[2] ? sum / (double)h[2] : 0.0;
    ctx->prec_built = prec;
    ctx->prec_data_version = ctx->data_version;
    return KG_OK;
}

}  // namespace kgb

using namespace kgb;

extern "C" int kg_set_search_precision(kg_ctx *ctx, int mode) {
    if (!ctx) return KG_E_INVALID;
    std::lock_guard<std::mutex> guard(ctx->mu);
    cudaSetDevice(ctx->device);
    if (mode < KG_SEARCH_FP32 || mode > KG_SEARCH_FP8) return set_error(ctx, KG_E_INVALID, "bad search precision");
    if (!ctx->has_data && mode != KG_SEARCH_FP32) return set_error(ctx, KG_E_RUNTIME, "no dataset");
    ctx->search_prec = mode;
    return ensure_search_precision(ctx);
}

extern "C" int kg_last_search_filter(kg_ctx *ctx, kg_search_filter_stats *out) {
    if (!ctx || !out) return KG_E_INVALID;
    std::lock_guard<std::mutex> guard(ctx->mu);
    *out = kg_search_filter_stats{};
    out->mode = ctx->search_prec;
    out->approx = ctx->last_work[2];
    out->skipped = ctx->last_work[3];
    out->max_rel_row_error = ctx->search_prec ? ctx->prec_max_rel : 0.0;
    out->mean_rel_row_error = ctx->search_prec ? ctx->prec_mean_rel : 0.0;
    return KG_OK;
}

extern "C" int kg_filter_bounds(kg_ctx *ctx, const float *queries, size_t nq, size_t q_stride_bytes,
                                const uint32_t *ids, size_t per_query, float *lb, float *dist) {
    if (!ctx) return KG_E_INVALID;
    std::lock_guard<std::mutex> guard(ctx->mu);
    cudaSetDevice(ctx->device);
    if (!ctx->has_data || ctx->search_prec == KG_SEARCH_FP32)
        return set_error(ctx, KG_E_RUNTIME, "kg_filter_bounds needs a dataset and a BF16 or FP8 search precision");
    if (!queries || !ids || !lb || !dist || nq == 0 || per_query == 0 || q_stride_bytes < ctx->d * 4 ||
        ctx->ld > 256)
        return set_error(ctx, KG_E_INVALID, "bad arguments (d <= 256)");
    int r = ensure_search_precision(ctx);
    if (r != KG_OK) return r;
    const size_t np = nq * per_query;
    std::vector<uint32_t> hid(np);
    cudaMemcpy(hid.data(), ids, np * 4, cudaMemcpyDefault);
    for (uint32_t v : hid)
        if (v >= ctx->n) return set_error(ctx, KG_E_INVALID, "id out of range");
    DevBuf q, dev;
    cudaError_t e;
    if ((e = q.reserve(nq * ctx->ld * 4)) != cudaSuccess || (e = dev.reserve(np * 12)) != cudaSuccess) {
        q.release();
        return cuda_fail(ctx, e, "alloc");
    }
    cudaStream_t st = ctx->stream;
    cudaMemsetAsync(q.p, 0, nq * ctx->ld * 4, st);
    cudaMemcpy2DAsync(q.p, ctx->ld * 4, queries, q_stride_bytes, ctx->d * 4, nq, cudaMemcpyDefault, st);
    uint32_t *did = dev.as<uint32_t>();
    float *dlb = reinterpret_cast<float *>(did + np), *dd = dlb + np;
    cudaMemcpyAsync(did, hid.data(), np * 4, cudaMemcpyHostToDevice, st);
    SearchArgs a{};
    a.D = DataView{ctx->X.as<float>(), ctx->norms.as<float>(), ctx->n, ctx->d, ctx->ld, ctx->metric};
    a.Q = q.as<float>();
    a.q_ld = ctx->ld;
    a.nq = (uint32_t)nq;
    a.prec = (uint32_t)ctx->search_prec;
    a.Xc = ctx->Xc.p;
    a.cmeta = ctx->cmeta.as<float4>();
    e = launch_filter_bounds(a, did, (uint32_t)per_query, dlb, dd, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(lb, dlb, np * 4, cudaMemcpyDefault, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dist, dd, np * 4, cudaMemcpyDefault, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    q.release();
    dev.release();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "filter bounds");
    return KG_OK;
}
