// Learned entry router: predicts, for a query, the graph regions its walk
// should start from, and hands them to the search as the reference's own
// user-provided starting points (SearchParams::init with ids as input,
// kgraph.cpp:461-467; doc/params.md "User-Provided Starting Points").
//
// Why.  The reference seeds every query with the same P random nodes
// (kgraph.cpp:444-453).  On clustered data the k-NN graph splits into one
// component per cluster, so plain search needs P large enough that some seed
// falls in the query's cluster (P ~ 1000 for 256 clusters at 1M points).  A
// seed inside the right cluster reaches the same neighbours with a pool of
// P ~ 50..100.
//
// What runs on the GPU, all in this file:
//   * entry clusters, two levels: k-means of the dataset into C x E fine
//     clusters (assignment by a BF16 x BF16 -> FP32 tiled GEMM against the
//     centroids plus an argmin, update by atomics), the member nearest each fine
//     centroid being a fine entry node; then k-means of the fine centroids into
//     the C clusters the MLP predicts, each owning the entry nodes of its fine
//     clusters;
//   * the MLP  D -> H -> H -> C  (ReLU), BF16 weights with FP32 master copies,
//     FP32 accumulation: forward, softmax cross-entropy, backward and Adam, every
//     step by the kernels below;
//   * training pairs: (query, cluster of the best node the plain search finds);
//   * inference: the `probe` most likely clusters per query, their fine entry
//     nodes ranked by exact FP32 distance to the query, the m nearest are the
//     seeds.  The second level lets C logits address more regions than C: a
//     mixture with more components than clusters still gets a seed in the
//     query's own component.
#include <cuda_bf16.h>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <mutex>
#include <numeric>
#include <random>
#include <vector>
#include "kg_ctx.h"
#include "kg_gemm.h"
#include "kg_warp.cuh"

namespace kgb {

namespace {

__global__ void to_bf16_kernel(const float *x, __nv_bfloat16 *y, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        y[i] = __float2bfloat16_rn(x[i]);
}

// Rows of the dataset (ld-strided) -> normalised BF16 features (x - mean) * inv_std.
__global__ void features_kernel(const float *X, uint32_t ld, const uint32_t *rows, uint32_t n, uint32_t d,
                                const float *mean, const float *inv_std, __nv_bfloat16 *out) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)n * d;
         i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)(i / d), c = (uint32_t)(i % d);
        const uint32_t row = rows ? rows[r] : r;
        out[i] = __float2bfloat16_rn((X[(size_t)row * ld + c] - mean[c]) * inv_std[c]);
    }
}

// Per-dimension partial sums of a row block, in FP64 and a fixed order: block
// b sums rows [b R, (b + 1) R) of x (pass 1) or of (x - mu)^2 (mu non-null),
// into part[b * d + j].  The host adds the partials in block order, so the
// result does not depend on scheduling.
__global__ void colsum_kernel(const float *X, uint32_t ld, uint32_t n, uint32_t d, uint32_t R, const double *mu,
                              double *part) {
    const uint32_t r0 = blockIdx.x * R, r1 = min(n, r0 + R);
    for (uint32_t j = threadIdx.x; j < d; j += blockDim.x) {
        double s = 0.0;
        const double m = mu ? mu[j] : 0.0;
        for (uint32_t r = r0; r < r1; ++r) {
            const double v = (double)X[(size_t)r * ld + j];
            s += mu ? (v - m) * (v - m) : v;
        }
        part[(size_t)blockIdx.x * d + j] = s;
    }
}

// Labels of a training batch: lab[i] = y[order[i]].
__global__ void gather_labels_kernel(const int32_t *y, const uint32_t *order, uint32_t n, int32_t *lab) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) lab[i] = y[order[i]];
}

// Softmax cross-entropy, one warp per row: loss (summed into *loss), argmax
// hits (summed into *hits), and dZ = (softmax - onehot) / B as FP32 and BF16.
__global__ void softmax_ce_kernel(const float *Z, const int32_t *y, int B, int C, float *dZ, __nv_bfloat16 *dZb,
                                  float *loss, unsigned *hits) {
    const int lane = threadIdx.x & 31;
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (row >= B) return;
    const float *z = Z + (size_t)row * C;
    float mx = -INFINITY;
    int am = 0;
    for (int c = lane; c < C; c += 32)
        if (z[c] > mx) { mx = z[c]; am = c; }
    for (int o = 16; o; o >>= 1) {
        const float om = __shfl_xor_sync(0xFFFFFFFFu, mx, o);
        const int oa = __shfl_xor_sync(0xFFFFFFFFu, am, o);
        if (om > mx || (om == mx && oa < am)) { mx = om; am = oa; }
    }
    float s = 0.f;
    for (int c = lane; c < C; c += 32) s += expf(z[c] - mx);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    const int t = y[row];
    if (lane == 0) {
        atomicAdd(loss, logf(s) + mx - z[t]);
        if (am == t) atomicAdd(hits, 1u);
    }
    if (dZ) {
        const float inv = 1.f / s, sc = 1.f / B;
        for (int c = lane; c < C; c += 32) {
            const float g = (expf(z[c] - mx) * inv - (c == t ? 1.f : 0.f)) * sc;
            dZ[(size_t)row * C + c] = g;
            dZb[(size_t)row * C + c] = __float2bfloat16_rn(g);
        }
    }
}

// dH *= (H > 0): the ReLU derivative, FP32 in place plus the BF16 copy.
__global__ void relu_grad_kernel(float *dH, const float *H, __nv_bfloat16 *dHb, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float g = H[i] > 0.f ? dH[i] : 0.f;
        dH[i] = g;
        dHb[i] = __float2bfloat16_rn(g);
    }
}

// db[c] = sum over rows of dZ[r, c].
__global__ void colsum_kernel(const float *dZ, int B, int C, float *db) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    float s = 0.f;
    for (int r = 0; r < B; ++r) s += dZ[(size_t)r * C + c];
    db[c] = s;
}

// Adam (Kingma & Ba 2015) on FP32 master weights, then the BF16 copy.
__global__ void adam_kernel(float *w, const float *g, float *m, float *v, __nv_bfloat16 *wb, size_t n, float lr,
                            float b1, float b2, float c1, float c2, float eps) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16_rn(wi);
    }
}

// k-means assignment from the GEMM's X.C^T block: argmin_c |c|^2 - 2 x.c.
__global__ void argmin_kernel(const float *G, const float *cn, int rows, int C, int32_t *lab, float *best) {
    const int lane = threadIdx.x & 31;
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= rows) return;
    float bv = INFINITY;
    int bi = 0;
    for (int c = lane; c < C; c += 32) {
        const float v = cn[c] - 2.f * G[(size_t)r * C + c];
        if (v < bv) { bv = v; bi = c; }
    }
    for (int o = 16; o; o >>= 1) {
        const float ov = __shfl_xor_sync(0xFFFFFFFFu, bv, o);
        const int oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
        if (ov < bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    if (lane == 0) { lab[r] = bi; if (best) best[r] = bv; }
}

// Sums the members of every cluster (features as FP32) and counts them.
__global__ void kmeans_accumulate_kernel(const __nv_bfloat16 *F, const int32_t *lab, uint32_t n, uint32_t d,
                                         float *sum, uint32_t *cnt) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)n * d;
         i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)(i / d), c = (uint32_t)(i % d);
        atomicAdd(sum + (size_t)lab[r] * d + c, __bfloat162float(F[i]));
        if (c == 0) atomicAdd(cnt + lab[r], 1u);
    }
}

// New centroids = means; an empty cluster keeps its old centroid.  Also |c|^2.
__global__ void kmeans_update_kernel(float *cent, const float *sum, const uint32_t *cnt, uint32_t C, uint32_t d,
                                     __nv_bfloat16 *centb, float *cn) {
    const uint32_t c = blockIdx.x;
    if (c >= C) return;
    __shared__ float red[32];
    float s2 = 0.f;
    for (uint32_t j = threadIdx.x; j < d; j += blockDim.x) {
        float v = cent[(size_t)c * d + j];
        if (cnt[c]) v = sum[(size_t)c * d + j] / cnt[c];
        const __nv_bfloat16 b = __float2bfloat16_rn(v);
        cent[(size_t)c * d + j] = v;
        centb[(size_t)c * d + j] = b;
        const float bf = __bfloat162float(b);
        s2 += bf * bf;
    }
    for (int o = 16; o; o >>= 1) s2 += __shfl_xor_sync(0xFFFFFFFFu, s2, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s2;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (uint32_t w = 0; w < blockDim.x / 32; ++w) t += red[w];
        cn[c] = t;
    }
}

// Entry node of every cluster: the member nearest its centroid, smallest id on ties.
__global__ void entry_kernel(const int32_t *lab, const float *best, uint32_t n, unsigned long long *key) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        float b = best[r];
        uint32_t u = __float_as_uint(b);
        u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);   // order-preserving float key
        atomicMin(key + lab[r], ((unsigned long long)u << 32) | r);
    }
}

// Top-m logits of every row -> entry nodes, in descending logit order.
__global__ void topm_kernel(const float *Z, int rows, int C, int m, const uint32_t *entry, uint32_t *out, int out_ld) {
    const int lane = threadIdx.x & 31;
    const int r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= rows) return;
    const float *z = Z + (size_t)r * C;
    unsigned long long taken[4] = {0, 0, 0, 0};   // bitset over lanes' slots: C <= 32 * 64
    for (int t = 0; t < m; ++t) {
        float bv = -INFINITY;
        int bi = -1;
        for (int c = lane, s = 0; c < C; c += 32, ++s) {
            if ((taken[s >> 6] >> (s & 63)) & 1ull) continue;
            if (z[c] > bv) { bv = z[c]; bi = c; }
        }
        for (int o = 16; o; o >>= 1) {
            const float ov = __shfl_xor_sync(0xFFFFFFFFu, bv, o);
            const int oi = __shfl_xor_sync(0xFFFFFFFFu, bi, o);
            if (ov > bv || (ov == bv && oi >= 0 && (bi < 0 || oi < bi))) { bv = ov; bi = oi; }
        }
        if (bi < 0) bi = 0;
        if ((bi & 31) == lane) { const int s = bi >> 5; taken[s >> 6] |= 1ull << (s & 63); }
        if (lane == 0) out[(size_t)r * out_ld + t] = entry ? entry[bi] : (uint32_t)bi;
    }
}

// FP32 centroids from rows of the BF16 feature matrix.
__global__ void init_centroids_kernel(const __nv_bfloat16 *F, uint32_t D, const uint32_t *rows, uint32_t C,
                                      float *cent) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)C * D;
         i += (size_t)gridDim.x * blockDim.x)
        cent[i] = __bfloat162float(F[(size_t)rows[i / D] * D + i % D]);
}

constexpr int RANK_CAND = 256;   // fine entry nodes ranked per query, at most
constexpr int RANK_WARPS = 8;

// Seeds of one query per warp: the fine entry nodes of its `probe` most likely
// clusters (topc), their canonical FP32 distances to the query, and the m
// nearest (ties: earlier candidate first).  Fewer than m candidates repeat the
// nearest one.  Q holds the queries' FP32 rows of D.d floats.
__global__ void __launch_bounds__(RANK_WARPS * 32) seed_rank_kernel(DataView D, const float *Q, int rows,
                                                                   const uint32_t *topc, int probe,
                                                                   const uint32_t *eoff, const uint32_t *eids, int m,
                                                                   uint32_t *out, int out_ld) {
    extern __shared__ __align__(16) float rank_smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    float *q = rank_smem + (size_t)w * (D.ld + 2 * RANK_CAND);
    uint32_t *cid = reinterpret_cast<uint32_t *>(q + D.ld);
    float *cd = q + D.ld + RANK_CAND;
    for (int r = blockIdx.x * RANK_WARPS + w; r < rows; r += gridDim.x * RANK_WARPS) {
        for (uint32_t j = lane; j < D.ld; j += 32) q[j] = j < D.d ? Q[(size_t)r * D.d + j] : 0.f;
        // candidate ids, in cluster-rank order
        int n = 0;
        for (int t = 0; t < probe; ++t) {
            const uint32_t c = topc[(size_t)r * probe + t];
            const uint32_t a = eoff[c], b = eoff[c + 1];
            for (uint32_t k = a + lane; k < b; k += 32) {
                const int at = n + (int)(k - a);
                if (at < RANK_CAND) cid[at] = eids[k];
            }
            n = min(RANK_CAND, n + (int)(b - a));
        }
        __syncwarp();
        float qn = 0.f;
        if (D.metric != METRIC_L2SQR) qn = norm_term(group4_raw(q, q, D.d, METRIC_EUCLIDEAN, lane & 3, FULL), D.metric);
        const int g = lane >> 2, t = lane & 3;
        for (int base = 0; base < n; base += 8) {
            const int i = base + g;
            const float dd = query_dist(D, q, qn, i < n ? cid[i] : 0u, t, FULL);
            if (i < n && t == 0) cd[i] = dd;
        }
        __syncwarp();
        // m rounds of a warp argmin over the remaining candidates
        uint32_t taken = 0;   // bit s: this lane's candidate lane + 32 s is taken
        uint32_t first = 0;
        for (int k = 0; k < m; ++k) {
            float bv = INFINITY;
            int bi = -1;
            for (int i = lane, sl = 0; i < n; i += 32, ++sl) {
                if ((taken >> sl) & 1u) continue;
                if (cd[i] < bv) { bv = cd[i]; bi = i; }
            }
            for (int o = 16; o; o >>= 1) {
                const float ov = __shfl_xor_sync(FULL, bv, o);
                const int oi = __shfl_xor_sync(FULL, bi, o);
                if (oi >= 0 && (bi < 0 || ov < bv || (ov == bv && oi < bi))) { bv = ov; bi = oi; }
            }
            uint32_t pick;
            if (bi < 0) pick = first;   // candidates exhausted
            else {
                pick = cid[bi];
                if ((bi & 31) == lane) taken |= 1u << (bi >> 5);
            }
            if (k == 0) first = pick;
            if (lane == 0) out[(size_t)r * out_ld + k] = pick;
        }
        __syncwarp();
    }
}

// Every product of the router runs on the tensor cores (kg_gemm.cu); ws (may
// be null) is the scratch of the K-split products.
void gemm(cudaStream_t st, uint32_t *err, const DevBuf *ws, int M, int N, int K, const __nv_bfloat16 *A, int lda,
          int ta, const __nv_bfloat16 *B, int ldb, int tb, float *C, int ldc, __nv_bfloat16 *Cb, const float *bias,
          int relu, float beta = 0.f) {
    tc_gemm(st, M, N, K, A, lda, ta, B, ldb, tb, C, ldc, Cb, bias, relu, beta, ws ? ws->as<float>() : nullptr,
            ws ? ws->bytes : 0, err);
}

int blocks_for(size_t n, int per = 256) { return (int)std::min<size_t>((n + per - 1) / per, 148 * 32); }

}  // namespace

// ---------------------------------------------------------------------------
// Router state (device): weights, Adam moments, activations for one batch.
struct RouterState {
    uint32_t D = 0, H = 0, C = 0, batch = 0, probe = 1;
    uint32_t *err = nullptr;                     // the context's device error word
    uint32_t entries_total = 0, component_entries = 0;   // entry nodes; of which added for uncovered components
    bool trained = false;
    DevBuf mean, inv_std;                        // normalisation
    DevBuf eoff, eids;                           // per cluster: its fine entry nodes (CSR)
    DevBuf w[3], b[3], wb[3], gw[3], gb[3], mw[3], vw[3], mb[3], vb[3];
    DevBuf X, H1, H1b, H2, H2b, Z, dZ, dZb, dH, dHb, lab, scal, topc;
    DevBuf gws;                                  // K-split scratch of the backward products
    DevBuf tq, tyo;                              // training: the queries (FP32 rows), their labels and order
    void release() {
        DevBuf *all[] = {&mean, &inv_std, &eoff, &eids, &X, &H1, &H1b, &H2, &H2b, &Z, &dZ, &dZb, &dH, &dHb, &lab,
                         &scal, &topc, &tq, &tyo, &gws};
        for (DevBuf *p : all) p->release();
        for (int l = 0; l < 3; ++l) {
            DevBuf *ps[] = {&w[l], &b[l], &wb[l], &gw[l], &gb[l], &mw[l], &vw[l], &mb[l], &vb[l]};
            for (DevBuf *p : ps) p->release();
        }
    }
};

void router_release(RouterState *r) {
    if (r) { r->release(); delete r; }
}

namespace {

cudaError_t alloc_router(RouterState &r, uint32_t batch) {
    const uint32_t in[3] = {r.D, r.H, r.H}, out[3] = {r.H, r.H, r.C};
    cudaError_t e;
    for (int l = 0; l < 3; ++l) {
        const size_t nw = (size_t)in[l] * out[l];
        DevBuf *f32[] = {&r.w[l], &r.gw[l], &r.mw[l], &r.vw[l]};
        for (DevBuf *p : f32)
            if ((e = p->reserve(nw * 4)) != cudaSuccess) return e;
        if ((e = r.wb[l].reserve(nw * 2)) != cudaSuccess) return e;
        DevBuf *bs[] = {&r.b[l], &r.gb[l], &r.mb[l], &r.vb[l]};
        for (DevBuf *p : bs)
            if ((e = p->reserve(out[l] * 4)) != cudaSuccess) return e;
    }
    const size_t B = batch;
    if ((e = r.X.reserve(B * r.D * 2)) != cudaSuccess || (e = r.H1.reserve(B * r.H * 4)) != cudaSuccess ||
        (e = r.H1b.reserve(B * r.H * 2)) != cudaSuccess || (e = r.H2.reserve(B * r.H * 4)) != cudaSuccess ||
        (e = r.H2b.reserve(B * r.H * 2)) != cudaSuccess || (e = r.Z.reserve(B * r.C * 4)) != cudaSuccess ||
        (e = r.dZ.reserve(B * std::max(r.C, r.H) * 4)) != cudaSuccess || (e = r.dZb.reserve(B * r.C * 2)) != cudaSuccess ||
        (e = r.dH.reserve(B * r.H * 4)) != cudaSuccess || (e = r.dHb.reserve(B * r.H * 2)) != cudaSuccess ||
        (e = r.lab.reserve(B * 4)) != cudaSuccess || (e = r.scal.reserve(64)) != cudaSuccess)
        return e;
    // the backward products' K splits (the forward ones are not split at these shapes)
    const int Bi = (int)batch, D = (int)r.D, H = (int)r.H, C = (int)r.C;
    const size_t wsb = std::max({tc_gemm_workspace_bytes(H, C, Bi), tc_gemm_workspace_bytes(Bi, H, C),
                                 tc_gemm_workspace_bytes(H, H, Bi), tc_gemm_workspace_bytes(Bi, H, H),
                                 tc_gemm_workspace_bytes(D, H, Bi), tc_gemm_workspace_bytes(Bi, H, D),
                                 tc_gemm_workspace_bytes(Bi, C, H)});
    if (wsb && (e = r.gws.reserve(wsb)) != cudaSuccess) return e;
    r.batch = batch;
    return cudaSuccess;
}

// Forward of B rows already in r.X (BF16 features): H1, H2, Z.
void forward(cudaStream_t st, RouterState &r, int B) {
    gemm(st, r.err, &r.gws, B, r.H, r.D, r.X.as<__nv_bfloat16>(), r.D, 0, r.wb[0].as<__nv_bfloat16>(), r.H, 0, r.H1.as<float>(), r.H,
         r.H1b.as<__nv_bfloat16>(), r.b[0].as<float>(), 1);
    gemm(st, r.err, &r.gws, B, r.H, r.H, r.H1b.as<__nv_bfloat16>(), r.H, 0, r.wb[1].as<__nv_bfloat16>(), r.H, 0, r.H2.as<float>(), r.H,
         r.H2b.as<__nv_bfloat16>(), r.b[1].as<float>(), 1);
    gemm(st, r.err, &r.gws, B, r.C, r.H, r.H2b.as<__nv_bfloat16>(), r.H, 0, r.wb[2].as<__nv_bfloat16>(), r.C, 0, r.Z.as<float>(), r.C,
         nullptr, r.b[2].as<float>(), 0);
}

// Loss and gradients of B rows with labels in r.lab (after forward).
void backward(cudaStream_t st, RouterState &r, int B) {
    float *loss = r.scal.as<float>();
    unsigned *hits = reinterpret_cast<unsigned *>(r.scal.as<char>() + 4);
    softmax_ce_kernel<<<(B * 32 + 255) / 256, 256, 0, st>>>(r.Z.as<float>(), r.lab.as<int32_t>(), B, r.C,
                                                            r.dZ.as<float>(), r.dZb.as<__nv_bfloat16>(), loss, hits);
    // layer 3: dW3 = H2^T dZ, db3, dH2 = dZ W3^T
    gemm(st, r.err, &r.gws, r.H, r.C, B, r.H2b.as<__nv_bfloat16>(), r.H, 1, r.dZb.as<__nv_bfloat16>(), r.C, 0, r.gw[2].as<float>(), r.C,
         nullptr, nullptr, 0);
    colsum_kernel<<<(r.C + 255) / 256, 256, 0, st>>>(r.dZ.as<float>(), B, r.C, r.gb[2].as<float>());
    gemm(st, r.err, &r.gws, B, r.H, r.C, r.dZb.as<__nv_bfloat16>(), r.C, 0, r.wb[2].as<__nv_bfloat16>(), r.C, 1, r.dH.as<float>(), r.H,
         nullptr, nullptr, 0);
    relu_grad_kernel<<<blocks_for((size_t)B * r.H), 256, 0, st>>>(r.dH.as<float>(), r.H2.as<float>(),
                                                                  r.dHb.as<__nv_bfloat16>(), (size_t)B * r.H);
    // layer 2
    gemm(st, r.err, &r.gws, r.H, r.H, B, r.H1b.as<__nv_bfloat16>(), r.H, 1, r.dHb.as<__nv_bfloat16>(), r.H, 0, r.gw[1].as<float>(), r.H,
         nullptr, nullptr, 0);
    colsum_kernel<<<(r.H + 255) / 256, 256, 0, st>>>(r.dH.as<float>(), B, r.H, r.gb[1].as<float>());
    // dH1 = dH2 W2^T (into r.dZ as scratch: B x H fits), then the ReLU mask
    gemm(st, r.err, &r.gws, B, r.H, r.H, r.dHb.as<__nv_bfloat16>(), r.H, 0, r.wb[1].as<__nv_bfloat16>(), r.H, 1, r.dZ.as<float>(), r.H,
         nullptr, nullptr, 0);
    relu_grad_kernel<<<blocks_for((size_t)B * r.H), 256, 0, st>>>(r.dZ.as<float>(), r.H1.as<float>(),
                                                                  r.dHb.as<__nv_bfloat16>(), (size_t)B * r.H);
    // layer 1
    gemm(st, r.err, &r.gws, r.D, r.H, B, r.X.as<__nv_bfloat16>(), r.D, 1, r.dHb.as<__nv_bfloat16>(), r.H, 0, r.gw[0].as<float>(), r.H,
         nullptr, nullptr, 0);
    colsum_kernel<<<(r.H + 255) / 256, 256, 0, st>>>(r.dZ.as<float>(), B, r.H, r.gb[0].as<float>());
}

// Weakly connected components of the CSR graph by minimum-label propagation:
// every edge pulls both endpoints' labels down to the smaller one, then labels
// jump to their label's label; repeated until nothing changes.  The label of a
// component is its smallest node id.
__global__ void cc_hook_kernel(uint32_t N, const uint64_t *off, const uint32_t *nbr, uint32_t *lab, uint32_t *changed) {
    const int lane = threadIdx.x & 31;
    for (uint32_t u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; u < N; u += (gridDim.x * blockDim.x) >> 5) {
        const uint64_t a = off[u], b = off[u + 1];
        bool ch = false;
        for (uint64_t k = a + lane; k < b; k += 32) {
            const uint32_t v = nbr[k];
            if (v >= N) continue;
            const uint32_t lu = lab[u], lv = lab[v];
            if (lu < lv) ch |= atomicMin(lab + v, lu) > lu;
            else if (lv < lu) ch |= atomicMin(lab + u, lv) > lv;
        }
        if (__any_sync(0xFFFFFFFFu, ch) && lane == 0) *changed = 1u;
    }
}

__global__ void cc_jump_kernel(uint32_t N, uint32_t *lab) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < N; v += gridDim.x * blockDim.x) {
        uint32_t l = lab[v];
        while (lab[l] < l) l = lab[l];   // labels only point down, so this ends
        lab[v] = l;
    }
}

__global__ void iota_kernel(uint32_t N, uint32_t *lab) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < N; v += gridDim.x * blockDim.x) lab[v] = v;
}

// Scratch of one k-means run, released on scope exit.
struct KMeansBufs {
    DevBuf work, rows;
    ~KMeansBufs() { work.release(); rows.release(); }
};

// Lloyd's k-means of n BF16 rows F (n x D) into C centroids started at the rows
// `seed_rows`: `iters` updates, then a final assignment into lab[n] / best[n]
// (|c|^2 - 2 f.c of the chosen centroid).  The BF16 centroids end in
// *centb_out (inside kb.work); `block` holds one block of F.C^T.
cudaError_t kmeans_run(cudaStream_t st, uint32_t *err, const __nv_bfloat16 *F, uint32_t n, uint32_t D, uint32_t C,
                       uint32_t iters, const std::vector<uint32_t> &seed_rows, KMeansBufs &kb, DevBuf &block,
                       int32_t *lab, float *best, __nv_bfloat16 **centb_out) {
    cudaError_t e;
    const uint32_t brows = (uint32_t)std::max<size_t>(1024, std::min<size_t>(65536, ((size_t)1 << 29) / C));
    if ((e = kb.work.reserve((size_t)C * D * 4 * 2 + (size_t)C * D * 2 + (size_t)C * 8 + 64)) != cudaSuccess ||
        (e = kb.rows.reserve((size_t)C * 4)) != cudaSuccess)
        return e;
    if (D > 256 && (e = block.reserve((size_t)brows * C * 4)) != cudaSuccess) return e;   // product + argmin path
    float *cent = kb.work.as<float>();
    float *csum = cent + (size_t)C * D;
    __nv_bfloat16 *centb = reinterpret_cast<__nv_bfloat16 *>(csum + (size_t)C * D);
    float *cn = reinterpret_cast<float *>(centb + (size_t)C * D);
    uint32_t *ccnt = reinterpret_cast<uint32_t *>(cn + C);
    cudaMemcpyAsync(kb.rows.p, seed_rows.data(), (size_t)C * 4, cudaMemcpyHostToDevice, st);
    init_centroids_kernel<<<blocks_for((size_t)C * D), 256, 0, st>>>(F, D, kb.rows.as<uint32_t>(), C, cent);
    cudaMemsetAsync(ccnt, 0, (size_t)C * 4, st);
    kmeans_update_kernel<<<C, 128, 0, st>>>(cent, csum, ccnt, C, D, centb, cn);
    for (uint32_t it = 0; it <= iters; ++it) {
        // assignment fused into the tensor-core product (no n x C matrix), or product + argmin for D > 256
        if (!tc_assign(st, (int)n, (int)D, F, centb, (int)C, cn, lab, best, err)) {
            for (uint32_t r0 = 0; r0 < n; r0 += brows) {
                const uint32_t rows = std::min<uint32_t>(brows, n - r0);
                gemm(st, err, nullptr, rows, C, D, F + (size_t)r0 * D, D, 0, centb, D, 1, block.as<float>(), C, nullptr, nullptr,
                     0);
                argmin_kernel<<<(rows * 32 + 255) / 256, 256, 0, st>>>(block.as<float>(), cn, rows, C, lab + r0,
                                                                       best + r0);
            }
        }
        if (it == iters) break;
        cudaMemsetAsync(csum, 0, (size_t)C * D * 4, st);
        cudaMemsetAsync(ccnt, 0, (size_t)C * 4, st);
        kmeans_accumulate_kernel<<<blocks_for((size_t)n * D), 256, 0, st>>>(F, lab, n, D, csum, ccnt);
        kmeans_update_kernel<<<C, 128, 0, st>>>(cent, csum, ccnt, C, D, centb, cn);
    }
    *centb_out = centb;
    return cudaGetLastError();
}

constexpr uint32_t MIN_COMPONENT = 8;
constexpr size_t LABEL_CHUNKS = 16;   // label searches, each with its own seeds
constexpr int REGROUP_TOP = 8;        // most likely clusters a fine cluster may move to

// Component label of every node of the context's graph (host copy in comp).
int graph_components(kg_ctx *ctx, DevBuf &buf, std::vector<uint32_t> &comp) {
    const uint32_t N = ctx->gn;
    cudaStream_t st = ctx->stream;
    cudaError_t e;
    if ((e = buf.reserve((size_t)N * 4 + 16)) != cudaSuccess) return cuda_fail(ctx, e, "router alloc");
    uint32_t *lab = buf.as<uint32_t>(), *changed = lab + N;
    iota_kernel<<<blocks_for(N), 256, 0, st>>>(N, lab);
    for (int it = 0; it < 1000; ++it) {
        uint32_t h = 0;
        cudaMemsetAsync(changed, 0, 4, st);
        cc_hook_kernel<<<blocks_for((size_t)N * 32), 256, 0, st>>>(N, ctx->offsets.as<uint64_t>(),
                                                                   ctx->nbr.as<uint32_t>(), lab, changed);
        cc_jump_kernel<<<blocks_for(N), 256, 0, st>>>(N, lab);
        cudaMemcpyAsync(&h, changed, 4, cudaMemcpyDeviceToHost, st);
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "graph components");
        if (!h) break;
    }
    comp.resize(N);
    cudaMemcpyAsync(comp.data(), lab, (size_t)N * 4, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "graph components");
    return KG_OK;
}

void init_weights(RouterState &r, uint64_t seed) {
    std::mt19937_64 rng(seed);
    const uint32_t in[3] = {r.D, r.H, r.H}, out[3] = {r.H, r.H, r.C};
    for (int l = 0; l < 3; ++l) {
        const size_t nw = (size_t)in[l] * out[l];
        std::normal_distribution<float> nd(0.f, std::sqrt(2.f / in[l]));   // He initialisation
        std::vector<float> h(nw);
        for (auto &x : h) x = nd(rng);
        cudaMemcpy(r.w[l].p, h.data(), nw * 4, cudaMemcpyHostToDevice);
        cudaMemset(r.b[l].p, 0, out[l] * 4);
        cudaMemset(r.mw[l].p, 0, nw * 4);
        cudaMemset(r.vw[l].p, 0, nw * 4);
        cudaMemset(r.mb[l].p, 0, out[l] * 4);
        cudaMemset(r.vb[l].p, 0, out[l] * 4);
        to_bf16_kernel<<<blocks_for(nw), 256>>>(r.w[l].as<float>(), r.wb[l].as<__nv_bfloat16>(), nw);
    }
}

}  // namespace
}  // namespace kgb

using namespace kgb;

namespace {
struct Guard {
    kg_ctx *c;
    explicit Guard(kg_ctx *ctx) : c(ctx) { c->mu.lock(); cudaSetDevice(c->device); }
    ~Guard() { c->mu.unlock(); }
};

// Normalised BF16 features of host/device query rows into r.X (n <= r.batch).
int stage_queries(kg_ctx *ctx, RouterState &r, const float *q, size_t n, size_t stride, DevBuf &tmp) {
    cudaError_t e;
    if ((e = tmp.reserve(n * r.D * 4)) != cudaSuccess) return cuda_fail(ctx, e, "router alloc");
    e = cudaMemcpy2DAsync(tmp.p, r.D * 4, q, stride, r.D * 4, n, is_device_ptr(q) ? cudaMemcpyDeviceToDevice
                                                                                   : cudaMemcpyHostToDevice,
                          ctx->stream);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "router queries");
    features_kernel<<<blocks_for(n * r.D), 256, 0, ctx->stream>>>(tmp.as<float>(), r.D, nullptr, (uint32_t)n, r.D,
                                                                    r.mean.as<float>(), r.inv_std.as<float>(),
                                                                    r.X.as<__nv_bfloat16>());
    return KG_OK;
}
}  // namespace

extern "C" int kg_last_router_timing(kg_ctx *ctx, float *seeds_ms) {
    if (!ctx) return KG_E_INVALID;
    if (seeds_ms) *seeds_ms = ctx->last_router_ms;
    return KG_OK;
}

extern "C" void kg_router_params_default(kg_router_params *p) {
    p->clusters = 1024;
    p->hidden = 256;
    p->kmeans_iters = 8;
    p->label_P = 1000;
    p->epochs = 4;
    p->batch = 1024;
    p->lr = 2e-3f;
    p->seed = 1998;
    p->entries = 8;
    p->probe = 8;
    p->refine = 2;
    p->refine_P = 50;
}

extern "C" int kg_router_train(kg_ctx *ctx, const kg_router_params *p, const float *train_queries, size_t ntrain,
                               size_t q_stride_bytes, kg_router_info *info) {
    if (!ctx) return KG_E_INVALID;
    if (!p || !train_queries || ntrain == 0) return set_error(ctx, KG_E_INVALID, "bad router arguments");
    {
        Guard g(ctx);
        if (!ctx->has_data || !ctx->has_graph) return set_error(ctx, KG_E_RUNTIME, "router needs a dataset and a graph");
        if (p->clusters < 2 || p->clusters > 2048 || p->hidden < 8 || p->batch < 1 || p->entries > 16 ||
            p->probe < 1 || p->probe > 32 || p->refine > 8)
            return set_error(ctx, KG_E_INVALID, "router sizes out of range (clusters 2..2048, entries 0..16, "
                                                "probe 1..32)");
    }
    using clk = std::chrono::steady_clock;
    auto secs = [](clk::time_point a, clk::time_point b) { return (float)std::chrono::duration<double>(b - a).count(); };
    const clk::time_point t_start = clk::now();
    float refine_s = 0.f, mlp_s = 0.f;
    // 1. labels: the best node the plain search finds for each training query.
    //    The plain search starts every query of a call from the same P seeds
    //    (kgraph.cpp:444-453), so a region without a seed is missed by every
    //    query of the call; the training queries are therefore searched in
    //    LABEL_CHUNKS calls with different seeds, which spreads those misses
    //    over different regions instead of repeating them.
    std::vector<uint32_t> top(ntrain), cnt(ntrain);
    std::vector<float> topd(ntrain);
    for (size_t c = 0; c < LABEL_CHUNKS; ++c) {
        const size_t a = ntrain * c / LABEL_CHUNKS, b = ntrain * (c + 1) / LABEL_CHUNKS;
        if (a == b) continue;
        kg_search_params sp;
        kg_search_params_default(&sp);
        sp.K = 1;
        sp.P = p->label_P;
        sp.seed = p->seed + 1 + (unsigned)c;
        const float *qa = reinterpret_cast<const float *>(reinterpret_cast<const char *>(train_queries) +
                                                          a * q_stride_bytes);
        int rc = kg_search_batch(ctx, qa, b - a, q_stride_bytes, &sp, nullptr, nullptr, 1, top.data() + a,
                                 topd.data() + a, cnt.data() + a, nullptr);
        if (rc != KG_OK) return rc;
    }
    const clk::time_point t_labels = clk::now();
    std::unique_lock<std::mutex> lk(ctx->mu);   // released around the refinement's searches
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    cudaError_t e;
    if (!ctx->router) ctx->router = new RouterState;
    RouterState &r = *ctx->router;
    r.err = ctx->errw.as<uint32_t>();
    r.trained = false;
    r.D = ctx->d;
    r.H = p->hidden;
    r.C = p->clusters;
    const uint32_t N = ctx->n, D = ctx->d, C = r.C;
    if ((e = alloc_router(r, std::max<uint32_t>(p->batch, 4096))) != cudaSuccess) return cuda_fail(ctx, e, "router alloc");
    DevBuf &s0 = ctx->build_scratch[20], &s1 = ctx->build_scratch[21], &s2 = ctx->build_scratch[22],
           &s3 = ctx->build_scratch[23];

    // 2. normalisation over the dataset (per-dimension mean and 1/std): FP64
    //    partial sums per row block on the device, added on the host in order
    std::vector<double> mu(D, 0.0), var(D, 0.0);
    {
        const uint32_t nb = std::max<uint32_t>(1u, std::min<uint32_t>(N, (uint32_t)ctx->num_sms * 8));
        const uint32_t R = (N + nb - 1) / nb;
        DevBuf part;
        if ((e = part.reserve(((size_t)nb * D + D) * sizeof(double))) != cudaSuccess)
            return cuda_fail(ctx, e, "router alloc");
        double *dpart = part.as<double>(), *dmu = dpart + (size_t)nb * D;
        std::vector<double> hpart((size_t)nb * D);
        for (int pass = 0; pass < 2; ++pass) {
            if (pass == 1) cudaMemcpyAsync(dmu, mu.data(), D * sizeof(double), cudaMemcpyHostToDevice, st);
            colsum_kernel<<<nb, 128, 0, st>>>(ctx->X.as<float>(), ctx->ld, N, D, R, pass ? dmu : nullptr, dpart);
            cudaMemcpyAsync(hpart.data(), dpart, hpart.size() * sizeof(double), cudaMemcpyDeviceToHost, st);
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess) { part.release(); return cuda_fail(ctx, e, "router stats"); }
            std::vector<double> &acc = pass ? var : mu;
            for (uint32_t b = 0; b < nb; ++b)
                for (uint32_t j = 0; j < D; ++j) acc[j] += hpart[(size_t)b * D + j];
            if (pass == 0)
                for (uint32_t j = 0; j < D; ++j) mu[j] /= N;
        }
        part.release();
    }
    std::vector<float> hm(D), hs(D);
    for (uint32_t j = 0; j < D; ++j) { hm[j] = (float)mu[j]; hs[j] = (float)(1.0 / std::sqrt(var[j] / N + 1e-6)); }
    if ((e = r.mean.reserve(D * 4)) != cudaSuccess || (e = r.inv_std.reserve(D * 4)) != cudaSuccess)
        return cuda_fail(ctx, e, "router alloc");
    cudaMemcpyAsync(r.mean.p, hm.data(), D * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(r.inv_std.p, hs.data(), D * 4, cudaMemcpyHostToDevice, st);

    // 3. entry clusters.  Fine level: k-means of the dataset features into
    //    Cf = C x E clusters, entry node = the member nearest each centroid.
    const uint32_t E = std::max(1u, p->entries), Cf = C * E;
    if ((e = s0.reserve((size_t)N * D * 2)) != cudaSuccess ||            // features (BF16)
        (e = s2.reserve((size_t)N * 4 * 2 + (size_t)Cf * 8)) != cudaSuccess)   // labels, best (+ fine level's)
        return cuda_fail(ctx, e, "router alloc");
    __nv_bfloat16 *F = s0.as<__nv_bfloat16>();
    int32_t *lab = s2.as<int32_t>();
    float *best = reinterpret_cast<float *>(lab + N);
    int32_t *labc = reinterpret_cast<int32_t *>(best + N);
    float *bestc = reinterpret_cast<float *>(labc + Cf);
    features_kernel<<<blocks_for((size_t)N * D), 256, 0, st>>>(ctx->X.as<float>(), ctx->ld, nullptr, N, D,
                                                                 r.mean.as<float>(), r.inv_std.as<float>(), F);
    KMeansBufs fine, coarse;
    __nv_bfloat16 *centf = nullptr, *centc = nullptr;
    std::mt19937 krng(p->seed);
    {
        std::vector<uint32_t> pick(Cf);
        for (uint32_t c = 0; c < Cf; ++c) pick[c] = krng() % N;
        if ((e = kmeans_run(st, r.err, F, N, D, Cf, p->kmeans_iters, pick, fine, s3, lab, best, &centf)) != cudaSuccess)
            return cuda_fail(ctx, e, "router kmeans");
    }
    unsigned long long *key = reinterpret_cast<unsigned long long *>(s1.p);
    if ((e = s1.reserve((size_t)Cf * 8)) != cudaSuccess) return cuda_fail(ctx, e, "router alloc");
    key = reinterpret_cast<unsigned long long *>(s1.p);
    cudaMemsetAsync(key, 0xFF, (size_t)Cf * 8, st);
    entry_kernel<<<blocks_for(N), 256, 0, st>>>(lab, best, N, key);
    // Coarse level: the fine centroids grouped into the C clusters of the MLP.
    if (E > 1) {
        std::vector<uint32_t> pick(C);
        for (uint32_t c = 0; c < C; ++c) pick[c] = krng() % Cf;
        if ((e = kmeans_run(st, r.err, centf, Cf, D, C, p->kmeans_iters, pick, coarse, s3, labc, bestc, &centc)) !=
            cudaSuccess)
            return cuda_fail(ctx, e, "router kmeans");
    }
    std::vector<unsigned long long> hkey(Cf);
    std::vector<int32_t> hlab(N), hlabc(Cf);
    cudaMemcpyAsync(hkey.data(), key, (size_t)Cf * 8, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hlab.data(), lab, (size_t)N * 4, cudaMemcpyDeviceToHost, st);
    if (E > 1) cudaMemcpyAsync(hlabc.data(), labc, (size_t)Cf * 4, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "router kmeans");
    if (E == 1)
        for (uint32_t f = 0; f < Cf; ++f) hlabc[f] = (int32_t)f;
    // Entry nodes per cluster: those of its non-empty fine clusters, plus one
    // node of every connected component of the graph (of at least
    // MIN_COMPONENT nodes) that holds no fine entry node: a walk never leaves
    // its component, so every component needs a way in.  Such a node joins the
    // cluster its own members are assigned to.
    const std::vector<int32_t> hfine(hlab.begin(), hlab.end());   // fine cluster of every node
    std::vector<uint32_t> comp_reps;
    {
        std::vector<uint32_t> comp;
        int rc = graph_components(ctx, s1, comp);
        if (rc != KG_OK) return rc;
        std::vector<uint32_t> size(N, 0);
        std::vector<uint8_t> covered(N, 0);
        for (uint32_t i = 0; i < ctx->gn; ++i) ++size[comp[i]];
        for (uint32_t f = 0; f < Cf; ++f)
            if (hkey[f] != ~0ull) covered[comp[(uint32_t)(hkey[f] & 0xFFFFFFFFu)]] = 1;
        for (uint32_t i = 0; i < ctx->gn; ++i)
            if (comp[i] == i && !covered[i] && size[i] >= MIN_COMPONENT) comp_reps.push_back(i);   // smallest id
    }
    uint32_t empty = 0;   // clusters without an entry node
    // (Re)derives every node's cluster from its fine cluster and installs the
    // clusters' entry nodes (CSR) for the seed ranking.
    auto install_entries = [&]() -> int {
        for (uint32_t i = 0; i < N; ++i) hlab[i] = hlabc[hfine[i]];
        std::vector<std::pair<uint32_t, uint32_t>> ent;   // (cluster, node)
        ent.reserve(Cf + comp_reps.size());
        for (uint32_t f = 0; f < Cf; ++f)
            if (hkey[f] != ~0ull) ent.emplace_back((uint32_t)hlabc[f], (uint32_t)(hkey[f] & 0xFFFFFFFFu));
        for (uint32_t rep : comp_reps) ent.emplace_back((uint32_t)hlab[rep], rep);
        std::stable_sort(ent.begin(), ent.end(),
                         [](const std::pair<uint32_t, uint32_t> &a, const std::pair<uint32_t, uint32_t> &b) {
                             return a.first < b.first;
                         });
        std::vector<uint32_t> heoff(C + 1, 0), heids(ent.size());
        for (size_t k = 0; k < ent.size(); ++k) { ++heoff[ent[k].first + 1]; heids[k] = ent[k].second; }
        for (uint32_t c = 0; c < C; ++c) heoff[c + 1] += heoff[c];
        empty = 0;
        for (uint32_t c = 0; c < C; ++c) empty += heoff[c + 1] == heoff[c];
        cudaError_t e2;
        if ((e2 = r.eoff.reserve((size_t)(C + 1) * 4)) != cudaSuccess ||
            (e2 = r.eids.reserve(std::max<size_t>(heids.size(), 1) * 4)) != cudaSuccess)
            return cuda_fail(ctx, e2, "router alloc");
        cudaMemcpyAsync(r.eoff.p, heoff.data(), (size_t)(C + 1) * 4, cudaMemcpyHostToDevice, st);
        if (!heids.empty()) cudaMemcpyAsync(r.eids.p, heids.data(), heids.size() * 4, cudaMemcpyHostToDevice, st);
        if ((e2 = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e2, "router entries");
        r.entries_total = (uint32_t)heids.size();
        r.component_entries = (uint32_t)comp_reps.size();
        return KG_OK;
    };
    {
        int rc = install_entries();
        if (rc != KG_OK) return rc;
    }
    r.probe = std::max(1u, std::min(p->probe, C));

    const clk::time_point t_clusters = clk::now();
    // 4. training set: the cluster of each query's best node.  The queries stay
    //    on the device as FP32 rows; each step gathers and normalises its batch
    //    there by the epoch's shuffled order, and nothing waits for the host
    //    until an epoch run ends.
    std::vector<int32_t> ylab(ntrain);
    for (size_t i = 0; i < ntrain; ++i) ylab[i] = cnt[i] ? hlab[top[i] < N ? top[i] : 0] : 0;
    init_weights(r, p->seed);
    const uint32_t B = p->batch;
    DevBuf &tq = r.tq, &tyo = r.tyo;
    if ((e = tq.reserve(ntrain * D * 4)) != cudaSuccess || (e = tyo.reserve(ntrain * 8)) != cudaSuccess)
        return cuda_fail(ctx, e, "router alloc");
    if ((e = cudaMemcpy2DAsync(tq.p, D * 4, train_queries, q_stride_bytes, D * 4, ntrain, cudaMemcpyDefault, st)) !=
        cudaSuccess)
        return cuda_fail(ctx, e, "router queries");
    int32_t *dy = tyo.as<int32_t>();                                          // labels of the training queries
    uint32_t *dorder = reinterpret_cast<uint32_t *>(dy + ntrain);             // the epoch's order
    std::vector<uint32_t> order(ntrain);
    for (size_t i = 0; i < ntrain; ++i) order[i] = (uint32_t)i;
    std::mt19937 rng(p->seed + 1);
    float last_loss = 0.f;
    unsigned step = 0;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const size_t full = ntrain < B ? ntrain : ntrain / B * B;   // the last partial batch is dropped
    auto run_epochs = [&](uint32_t epochs) -> int {
    const clk::time_point t0 = clk::now();
    // pageable sources: each copy has read its host buffer when it returns
    cudaMemcpyAsync(dy, ylab.data(), ntrain * 4, cudaMemcpyHostToDevice, st);
    uint32_t last_bs = 0;
    for (uint32_t ep = 0; ep < epochs; ++ep) {
        std::shuffle(order.begin(), order.end(), rng);
        cudaMemcpyAsync(dorder, order.data(), ntrain * 4, cudaMemcpyHostToDevice, st);
        for (size_t s0i = 0; s0i < full; s0i += B) {
            const uint32_t bs = (uint32_t)std::min<size_t>(B, full - s0i);
            features_kernel<<<blocks_for((size_t)bs * D), 256, 0, st>>>(tq.as<float>(), D, dorder + s0i, bs, D,
                                                                        r.mean.as<float>(), r.inv_std.as<float>(),
                                                                        r.X.as<__nv_bfloat16>());
            gather_labels_kernel<<<(bs + 255) / 256, 256, 0, st>>>(dy, dorder + s0i, bs, r.lab.as<int32_t>());
            cudaMemsetAsync(r.scal.p, 0, 8, st);
            forward(st, r, bs);
            backward(st, r, bs);
            ++step;
            const float c1 = 1.f - std::pow(b1, (float)step), c2 = 1.f - std::pow(b2, (float)step);
            const uint32_t in[3] = {r.D, r.H, r.H}, out[3] = {r.H, r.H, r.C};
            for (int l = 0; l < 3; ++l) {
                const size_t nw = (size_t)in[l] * out[l];
                adam_kernel<<<blocks_for(nw), 256, 0, st>>>(r.w[l].as<float>(), r.gw[l].as<float>(), r.mw[l].as<float>(),
                                                             r.vw[l].as<float>(), r.wb[l].as<__nv_bfloat16>(), nw, p->lr, b1,
                                                             b2, c1, c2, eps);
                adam_kernel<<<blocks_for(out[l]), 256, 0, st>>>(r.b[l].as<float>(), r.gb[l].as<float>(),
                                                                 r.mb[l].as<float>(), r.vb[l].as<float>(), nullptr,
                                                                 out[l], p->lr, b1, b2, c1, c2, eps);
            }
            last_bs = bs;
        }
    }
    float hl = 0.f;   // the last step's summed loss
    cudaMemcpyAsync(&hl, r.scal.p, 4, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "router train");
    if (last_bs) last_loss = hl / last_bs;
    mlp_s += secs(t0, clk::now());
    return KG_OK;
    };
    int rc0 = run_epochs(p->epochs);
    if (rc0 != KG_OK) return rc0;
    // 5. refinement: the router's own seeds, handed to the walk, may find a
    //    closer node than the plain search did for a training query; the closer
    //    of the two becomes its label and training continues.
    std::vector<uint32_t> sids, scnt;
    std::vector<float> sd;
    unsigned relabelled = 0;
    for (uint32_t round = 0; round < p->refine; ++round) {
        const clk::time_point tr = clk::now();
        r.trained = true;
        const unsigned m = 3, ld = m + 1;   // the reference requires init < K
        sids.assign(ntrain * ld, 0u);
        scnt.assign(ntrain, 0u);
        sd.assign(ntrain * ld, 0.f);
        lk.unlock();
        int rc = kg_router_seeds(ctx, train_queries, ntrain, q_stride_bytes, m, sids.data(), ld);
        if (rc == KG_OK) {
            kg_search_params sp;
            kg_search_params_default(&sp);
            sp.K = ld;
            sp.P = p->refine_P;
            sp.init = m;
            rc = kg_search_batch(ctx, train_queries, ntrain, q_stride_bytes, &sp, nullptr, nullptr, ld, sids.data(),
                                 sd.data(), scnt.data(), nullptr);
        }
        lk.lock();
        cudaSetDevice(ctx->device);
        if (rc != KG_OK) return rc;
        for (size_t i = 0; i < ntrain; ++i) {
            if (!scnt[i] || (cnt[i] && !(sd[i * ld] < topd[i]))) continue;
            const uint32_t node = sids[i * ld];
            if (node >= N) continue;
            if (!cnt[i] || hlab[node] != ylab[i]) ++relabelled;
            top[i] = node;
            topd[i] = sd[i * ld];
            cnt[i] = 1;
            ylab[i] = hlab[node];
        }
        // Regrouping: every fine cluster moves to the cluster the network
        // predicts for its centroid (the first of its REGROUP_TOP most likely
        // that is not full), so the clusters become groups the network can tell
        // apart; the labels follow and training continues.
        if (E > 1) {
            DevBuf dtop;
            cudaError_t e2 = dtop.reserve((size_t)Cf * REGROUP_TOP * 4);
            if (e2 != cudaSuccess) return cuda_fail(ctx, e2, "router alloc");
            for (uint32_t c0 = 0; c0 < Cf; c0 += r.batch) {
                const uint32_t bs = std::min<uint32_t>(r.batch, Cf - c0);
                cudaMemcpyAsync(r.X.p, centf + (size_t)c0 * D, (size_t)bs * D * 2, cudaMemcpyDeviceToDevice, st);
                forward(st, r, (int)bs);
                topm_kernel<<<((int)bs * 32 + 255) / 256, 256, 0, st>>>(r.Z.as<float>(), (int)bs, (int)C, REGROUP_TOP,
                                                                         nullptr, dtop.as<uint32_t>() + (size_t)c0 * REGROUP_TOP,
                                                                         REGROUP_TOP);
            }
            std::vector<uint32_t> htop((size_t)Cf * REGROUP_TOP);
            cudaMemcpyAsync(htop.data(), dtop.p, htop.size() * 4, cudaMemcpyDeviceToHost, st);
            e2 = cudaStreamSynchronize(st);
            dtop.release();
            if (e2 != cudaSuccess) return cuda_fail(ctx, e2, "router regroup");
            const uint32_t cap = (Cf + C - 1) / C * 3 / 2 + 1;
            std::vector<uint32_t> load(C, 0), forder(Cf);
            std::iota(forder.begin(), forder.end(), 0u);
            std::shuffle(forder.begin(), forder.end(), rng);
            std::vector<int32_t> nl(hlabc);
            for (uint32_t f : forder) {
                int pick = -1;
                for (int t = 0; t < REGROUP_TOP && pick < 0; ++t)
                    if (load[htop[(size_t)f * REGROUP_TOP + t]] < cap) pick = (int)htop[(size_t)f * REGROUP_TOP + t];
                if (pick < 0) pick = hlabc[f];
                nl[f] = pick;
                ++load[pick];
            }
            hlabc.swap(nl);
            if ((rc = install_entries()) != KG_OK) return rc;
            for (size_t i = 0; i < ntrain; ++i) ylab[i] = cnt[i] ? hlab[top[i] < N ? top[i] : 0] : 0;
        }
        refine_s += secs(tr, clk::now());
        if ((rc = run_epochs(p->epochs)) != KG_OK) return rc;
    }
    // accuracy of the final weights on the first min(ntrain, 4096) training rows
    float acc = 0.f;
    {
        const size_t n = std::min<size_t>(ntrain, 4096);
        unsigned hits_total = 0;
        cudaMemcpyAsync(dy, ylab.data(), n * 4, cudaMemcpyHostToDevice, st);
        for (size_t c0 = 0; c0 < n; c0 += r.batch) {
            const uint32_t bs = (uint32_t)std::min<size_t>(r.batch, n - c0);
            features_kernel<<<blocks_for((size_t)bs * D), 256, 0, st>>>(tq.as<float>() + c0 * D, D, nullptr, bs, D,
                                                                        r.mean.as<float>(), r.inv_std.as<float>(),
                                                                        r.X.as<__nv_bfloat16>());
            cudaMemcpyAsync(r.lab.p, dy + c0, bs * 4, cudaMemcpyDeviceToDevice, st);
            cudaMemsetAsync(r.scal.p, 0, 8, st);
            forward(st, r, bs);
            softmax_ce_kernel<<<(bs * 32 + 255) / 256, 256, 0, st>>>(r.Z.as<float>(), r.lab.as<int32_t>(), bs, r.C,
                                                                     nullptr, nullptr, r.scal.as<float>(),
                                                                     reinterpret_cast<unsigned *>(r.scal.as<char>() + 4));
            unsigned h = 0;
            cudaMemcpyAsync(&h, r.scal.as<char>() + 4, 4, cudaMemcpyDeviceToHost, st);
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "router eval");
            hits_total += h;
        }
        acc = n ? (float)hits_total / n : 0.f;
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "router train");
    r.trained = true;
    tq.release();    // the training set is not needed for seeding
    tyo.release();
    if (info) {
        info->steps = step;
        info->final_loss = last_loss;
        info->train_accuracy = acc;
        info->empty_clusters = empty;
        info->entries = r.entries_total;
        info->component_entries = r.component_entries;
        info->relabelled = relabelled;
        info->label_s = secs(t_start, t_labels);
        info->cluster_s = secs(t_labels, t_clusters);
        info->mlp_s = mlp_s;
        info->refine_s = refine_s;
    }
    return check_device_error(ctx, "router");
}

namespace {
// kg_router_seeds with the context lock held.
int router_seeds_locked(kg_ctx *ctx, const float *queries, size_t nq, size_t q_stride_bytes, unsigned m,
                        uint32_t *seeds, size_t out_ld) {
    if (!ctx->router || !ctx->router->trained) return set_error(ctx, KG_E_RUNTIME, "router not trained");
    RouterState &r = *ctx->router;
    r.err = ctx->errw.as<uint32_t>();
    if (m == 0 || m > r.C || m > out_ld || m > 64) return set_error(ctx, KG_E_INVALID, "bad number of router seeds");
    cudaStream_t st = ctx->stream;
    cudaError_t e;
    DevBuf &tq = ctx->build_scratch[19], &out = ctx->build_scratch[18];
    const bool sdev = is_device_ptr(seeds);
    if (!sdev && (e = out.reserve(nq * out_ld * 4)) != cudaSuccess) return cuda_fail(ctx, e, "router alloc");
    if ((e = r.topc.reserve((size_t)r.batch * r.probe * 4)) != cudaSuccess) return cuda_fail(ctx, e, "router alloc");
    {
        const size_t smem = (size_t)RANK_WARPS * (ctx->ld + 2 * RANK_CAND) * 4;
        if (smem > 48 * 1024 &&
            (e = cudaFuncSetAttribute(seed_rank_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
                cudaSuccess)
            return cuda_fail(ctx, e, "router seeds");
    }
    uint32_t *dst = sdev ? seeds : out.as<uint32_t>();
    if (!sdev) cudaMemcpyAsync(dst, seeds, nq * out_ld * 4, cudaMemcpyHostToDevice, st);
    const char *qb = reinterpret_cast<const char *>(queries);
    cudaEventRecord(ctx->ev0, st);
    for (size_t c0 = 0; c0 < nq; c0 += r.batch) {
        const size_t bs = std::min<size_t>(r.batch, nq - c0);
        int rc = stage_queries(ctx, r, reinterpret_cast<const float *>(qb + c0 * q_stride_bytes), bs, q_stride_bytes, tq);
        if (rc != KG_OK) return rc;
        forward(st, r, (int)bs);
        topm_kernel<<<((int)bs * 32 + 255) / 256, 256, 0, st>>>(r.Z.as<float>(), (int)bs, r.C, (int)r.probe, nullptr,
                                                                 r.topc.as<uint32_t>(), (int)r.probe);
        const DataView DV{ctx->X.as<float>(), ctx->norms.as<float>(), ctx->n, ctx->d, ctx->ld, ctx->metric};
        const size_t smem = (size_t)RANK_WARPS * (ctx->ld + 2 * RANK_CAND) * 4;
        const int grid = (int)std::min<size_t>((bs + RANK_WARPS - 1) / RANK_WARPS, (size_t)ctx->num_sms * 8);
        seed_rank_kernel<<<grid, RANK_WARPS * 32, smem, st>>>(DV, tq.as<float>(), (int)bs, r.topc.as<uint32_t>(),
                                                               (int)r.probe, r.eoff.as<uint32_t>(),
                                                               r.eids.as<uint32_t>(), (int)m, dst + c0 * out_ld,
                                                               (int)out_ld);
    }
    cudaEventRecord(ctx->ev1, st);
    if (!sdev) cudaMemcpyAsync(seeds, dst, nq * out_ld * 4, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "router seeds");
    cudaEventElapsedTime(&ctx->last_router_ms, ctx->ev0, ctx->ev1);
    return KG_OK;
}
}  // namespace

extern "C" int kg_router_seeds(kg_ctx *ctx, const float *queries, size_t nq, size_t q_stride_bytes, unsigned m,
                               uint32_t *seeds, size_t out_ld) {
    if (!ctx) return KG_E_INVALID;
    Guard g(ctx);
    return router_seeds_locked(ctx, queries, nq, q_stride_bytes, m, seeds, out_ld);
}

extern "C" int kg_router_search(kg_ctx *ctx, const float *queries, size_t nq, size_t q_stride_bytes,
                                const kg_search_params *params, size_t out_ld, uint32_t *ids, float *dists,
                                uint32_t *counts, float *costs) {
    if (!ctx) return KG_E_INVALID;
    Guard g(ctx);
    if (!params || !queries || !ids || !counts) return set_error(ctx, KG_E_INVALID, "bad arguments");
    if (nq == 0) return KG_OK;
    if (!ctx->router || !ctx->router->trained) return set_error(ctx, KG_E_RUNTIME, "router not trained");
    if (!ctx->has_graph) return set_error(ctx, KG_E_RUNTIME, "no index");
    if (params->init == 0 || !(params->init < params->K)) return set_error(ctx, KG_E_INVALID, "L < params.K");
    if (params->init > out_ld) return set_error(ctx, KG_E_INVALID, "init larger than out_ld");
    if (q_stride_bytes < ctx->d * sizeof(float)) return set_error(ctx, KG_E_INVALID, "bad query array");
    cudaStream_t st = ctx->stream;
    cudaError_t e;
    // queries once into device rows of the padded width, used by both stages in place
    const size_t ld = ctx->ld;
    if ((e = ctx->qbuf.reserve(nq * ld * 4)) != cudaSuccess || (e = ctx->rseeds.reserve(nq * params->init * 4)) !=
                                                                   cudaSuccess)
        return cuda_fail(ctx, e, "alloc queries");
    if (ld != ctx->d) cudaMemsetAsync(ctx->qbuf.p, 0, nq * ld * 4, st);
    e = cudaMemcpy2DAsync(ctx->qbuf.p, ld * 4, queries, q_stride_bytes, ctx->d * 4, nq,
                          is_device_ptr(queries) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "copy queries");
    int rc = router_seeds_locked(ctx, ctx->qbuf.as<float>(), nq, ld * 4, params->init, ctx->rseeds.as<uint32_t>(),
                                 params->init);
    if (rc != KG_OK) return rc;
    const float router_ms = ctx->last_router_ms;
    rc = search_locked(ctx, ctx->qbuf.as<float>(), nq, ld * 4, params, nullptr, nullptr, out_ld, ids, dists, counts,
                       costs, ctx->search_shape, ctx->rseeds.as<uint32_t>(), params->init);
    ctx->last_router_ms = router_ms;
    return rc;
}

// Loss and gradients of the current weights on n labelled rows (n <= 4096), for
// checking the kernels against an independent implementation.  weights: if not
// NULL, W1|b1|W2|b2|W3|b3 (FP32, row-major in x out) replace the router's.
extern "C" int kg_router_gradients(kg_ctx *ctx, unsigned d, unsigned hidden, unsigned clusters, const float *weights,
                                   const float *x, const int32_t *labels, unsigned n, float *loss, float *grads) {
    if (!ctx) return KG_E_INVALID;
    Guard g(ctx);
    if (n == 0 || n > 4096) return set_error(ctx, KG_E_INVALID, "n must be in 1..4096");
    if (!ctx->router) ctx->router = new RouterState;
    RouterState &r = *ctx->router;
    r.err = ctx->errw.as<uint32_t>();
    cudaStream_t st = ctx->stream;
    cudaError_t e;
    if (weights || r.D != d || r.H != hidden || r.C != clusters) {
        r.D = d; r.H = hidden; r.C = clusters;
        if ((e = alloc_router(r, 4096)) != cudaSuccess) return cuda_fail(ctx, e, "router alloc");
        if ((e = r.mean.reserve(d * 4)) != cudaSuccess || (e = r.inv_std.reserve(d * 4)) != cudaSuccess)
            return cuda_fail(ctx, e, "router alloc");
        std::vector<float> zero(d, 0.f), one(d, 1.f);
        cudaMemcpy(r.mean.p, zero.data(), d * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(r.inv_std.p, one.data(), d * 4, cudaMemcpyHostToDevice);
        r.trained = false;
    }
    const uint32_t in[3] = {d, hidden, hidden}, out[3] = {hidden, hidden, clusters};
    if (weights) {
        size_t off = 0;
        for (int l = 0; l < 3; ++l) {
            const size_t nw = (size_t)in[l] * out[l];
            cudaMemcpy(r.w[l].p, weights + off, nw * 4, cudaMemcpyHostToDevice);
            off += nw;
            cudaMemcpy(r.b[l].p, weights + off, out[l] * 4, cudaMemcpyHostToDevice);
            off += out[l];
            to_bf16_kernel<<<blocks_for(nw), 256, 0, st>>>(r.w[l].as<float>(), r.wb[l].as<__nv_bfloat16>(), nw);
        }
    }
    DevBuf &tq = ctx->build_scratch[19];
    int rc = stage_queries(ctx, r, x, n, (size_t)d * 4, tq);
    if (rc != KG_OK) return rc;
    cudaMemcpyAsync(r.lab.p, labels, n * 4, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(r.scal.p, 0, 8, st);
    forward(st, r, n);
    backward(st, r, n);
    float hl = 0.f;
    cudaMemcpyAsync(&hl, r.scal.p, 4, cudaMemcpyDeviceToHost, st);
    size_t off = 0;
    for (int l = 0; l < 3; ++l) {
        const size_t nw = (size_t)in[l] * out[l];
        if (grads) cudaMemcpyAsync(grads + off, r.gw[l].p, nw * 4, cudaMemcpyDeviceToHost, st);
        off += nw;
        if (grads) cudaMemcpyAsync(grads + off, r.gb[l].p, out[l] * 4, cudaMemcpyDeviceToHost, st);
        off += out[l];
    }
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "router gradients");
    if (loss) *loss = hl / n;
    return KG_OK;
}
