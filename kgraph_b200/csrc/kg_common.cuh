// Shared device code: dataset view, the canonical FP32 distance, error words.
//
// Canonical distance.  Every distance the library computes -- build join,
// init pool, controls, search, brute force -- goes through the functions
// below, so the same pair always gets the same FP32 bits.  That is what keeps
// the reference's list semantics intact on the GPU: UpdateKnnList detects a
// duplicate only among entries of EQUAL distance (kgraph.cpp:187-193), the
// reverse-sampling test relies on d(i,j) == d(j,i) (kgraph.cpp:852,860), and
// control recall matches by distance value (kgraph.cpp:96-128).
//
// The order is the one the reference's own -O3 AVX-512 build evaluates
// (kgraph-data.h:41-103 with xsimd avx512f reduce_add), measured bit for bit:
//   * 16 lanes; lane l accumulates elements l, l+16, ... as a rounded
//     product followed by a rounded add (no fusion);
//   * lanes reduce as t_k = (x_k + x_{k+4}) + (x_{k+8} + x_{k+12}),
//     result (t_0 + t_1) + (t_2 + t_3);
//   * the D % 16 tail elements follow in order: when there are 8 or more, the
//     first 8 as rounded product + rounded add (the reference's compiler
//     vectorises those products), every other one as a fused multiply-add;
//   * euclidean (python-api.cpp:51-59): (n_i + n_j) - dot, n = norm2 / 2;
//     angular (python-api.cpp:61-69): -dot / fma(n_i, n_j, FLT_EPSILON),
//     n = sqrt(norm2); l2sqr (kgraph-data.h:38-61): the same lanes over (a-b)^2.
// On the GPU a distance is computed by a group of 4 consecutive lanes: lane t
// of the group owns canonical lanes 4t..4t+3 and loads one float4 per
// 16-element chunk, which keeps the loads 64-byte coalesced per row.  All
// arithmetic uses the explicit _rn intrinsics, so nvcc cannot contract it.
#pragma once
#include <cstdint>
#include <cfloat>
#include <cuda_runtime.h>

namespace kgb {

enum Metric : int { METRIC_EUCLIDEAN = 0, METRIC_ANGULAR = 1, METRIC_L2SQR = 2 };

// Device error word bits (read back by the host after every call).
enum : uint32_t {
    ERR_LOCK_TIMEOUT = 1u << 0,   // a per-node lock spin ran out of iterations
    ERR_CAPACITY = 1u << 1,       // a list outgrew the capacity it was sized for
    ERR_BAD_ID = 1u << 2,         // an id >= n was met (corrupt graph / init ids)
    ERR_INIT_K = 1u << 3,         // init >= K for a query (reference: invalid_argument)
    ERR_STEP_LIMIT = 1u << 4,     // a search walk exceeded its step bound (never expected)
    ERR_TC_TIMEOUT = 1u << 5,     // a tensor-core completion wait ran out of cycles
};

constexpr uint32_t FLAG_BIT = 0x80000000u;
constexpr uint32_t ID_MASK = 0x7FFFFFFFu;
constexpr uint32_t NO_ID = 0xFFFFFFFFu;

// Dense dataset in HBM: n rows of `ld` floats (ld = d rounded up to 16, rows
// 64-byte aligned, zero padded), plus the per-row norm term of the metric.
struct DataView {
    const float *X;
    const float *norms;
    uint32_t n, d, ld;
    int metric;
};

__device__ __forceinline__ float4 ld4(const float *p) { return *reinterpret_cast<const float4 *>(p); }

__device__ __forceinline__ void lane_acc(float4 &acc, float4 x, float4 y, int metric) {
    if (metric == METRIC_L2SQR) {
        float a = __fsub_rn(x.x, y.x), b = __fsub_rn(x.y, y.y), c = __fsub_rn(x.z, y.z), e = __fsub_rn(x.w, y.w);
        acc.x = __fadd_rn(acc.x, __fmul_rn(a, a));
        acc.y = __fadd_rn(acc.y, __fmul_rn(b, b));
        acc.z = __fadd_rn(acc.z, __fmul_rn(c, c));
        acc.w = __fadd_rn(acc.w, __fmul_rn(e, e));
    } else {
        acc.x = __fadd_rn(acc.x, __fmul_rn(x.x, y.x));
        acc.y = __fadd_rn(acc.y, __fmul_rn(x.y, y.y));
        acc.z = __fadd_rn(acc.z, __fmul_rn(x.z, y.z));
        acc.w = __fadd_rn(acc.w, __fmul_rn(x.w, y.w));
    }
}

// Reduce the group's 16 canonical lanes; every lane of the group returns the sum.
__device__ __forceinline__ float group4_reduce(float4 acc, unsigned mask) {
    float4 o;
    o.x = __shfl_xor_sync(mask, acc.x, 1); o.y = __shfl_xor_sync(mask, acc.y, 1);
    o.z = __shfl_xor_sync(mask, acc.z, 1); o.w = __shfl_xor_sync(mask, acc.w, 1);
    acc.x = __fadd_rn(acc.x, o.x); acc.y = __fadd_rn(acc.y, o.y);
    acc.z = __fadd_rn(acc.z, o.z); acc.w = __fadd_rn(acc.w, o.w);
    o.x = __shfl_xor_sync(mask, acc.x, 2); o.y = __shfl_xor_sync(mask, acc.y, 2);
    o.z = __shfl_xor_sync(mask, acc.z, 2); o.w = __shfl_xor_sync(mask, acc.w, 2);
    acc.x = __fadd_rn(acc.x, o.x); acc.y = __fadd_rn(acc.y, o.y);
    acc.z = __fadd_rn(acc.z, o.z); acc.w = __fadd_rn(acc.w, o.w);
    return __fadd_rn(__fadd_rn(acc.x, acc.y), __fadd_rn(acc.z, acc.w));
}

// Raw canonical sum (dot for euclidean/angular, squared L2 for l2sqr) of
// rows a and b, computed by the 4-lane group containing this lane.  `t` is
// the lane's index in its group, `mask` the warp's active mask (all four
// lanes of every participating group must be in it).
__device__ __forceinline__ float group4_raw(const float *a, const float *b, int d, int metric, int t,
                                           unsigned mask) {
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    const int chunks = d >> 4;
    for (int c = 0; c < chunks; ++c) lane_acc(acc, ld4(a + 16 * c + 4 * t), ld4(b + 16 * c + 4 * t), metric);
    float r = group4_reduce(acc, mask);
    int i = chunks << 4;
    if (d - i >= 8) {   // the reference's compiler vectorises 8 tail products: rounded, added in order
        for (int e = i + 8; i < e; ++i) {
            float x = a[i], y = b[i];
            if (metric == METRIC_L2SQR) { x = __fsub_rn(x, y); y = x; }
            r = __fadd_rn(r, __fmul_rn(x, y));
        }
    }
    for (; i < d; ++i) {
        float x = a[i], y = b[i];
        if (metric == METRIC_L2SQR) { x = __fsub_rn(x, y); y = x; }
        r = __fmaf_rn(x, y, r);
    }
    return r;
}

// One canonical lane's step: acc += x*y (or (x-y)^2 for l2sqr), rounded product then rounded add.
__device__ __forceinline__ void acc1(float &acc, float x, float y, int metric) {
    if (metric == METRIC_L2SQR) { x = __fsub_rn(x, y); y = x; }
    acc = __fadd_rn(acc, __fmul_rn(x, y));
}

// The canonical raw sum computed by a group of G consecutive lanes (the
// "D-split"): lane t of the group owns canonical lanes (16/G)*t .. (16/G)*(t+1)-1,
// so one warp evaluates 32/G distances per pass.  G = 4 is group4_raw.  The
// lane sums are combined in exactly the canonical tree order, so every G gives
// the same bits:
//   G = 2  lane t holds lanes 8t..8t+7: a_j = x_j + x_{j+4} locally, the
//          partner's a_j added (t_j), then (t_0 + t_1) + (t_2 + t_3);
//   G = 8  lane t holds lanes 2t, 2t+1: + partner t^2 gives x_k + x_{k+4},
//          + partner t^4 gives t_k, then t_{2t} + t_{2t+1} locally and the
//          partner t^1 added.
template <int G>
__device__ __forceinline__ float groupG_raw(const float *a, const float *b, int d, int metric, int t, unsigned mask) {
    static_assert(G == 2 || G == 4 || G == 8, "D-split of 2, 4 or 8 lanes");
    if constexpr (G == 4) {
        return group4_raw(a, b, d, metric, t, mask);
    } else {
        constexpr int W = 16 / G;
        float acc[W];
#pragma unroll
        for (int j = 0; j < W; ++j) acc[j] = 0.f;
        const int chunks = d >> 4;
        for (int c = 0; c < chunks; ++c) {
            const float *pa = a + 16 * c + W * t, *pb = b + 16 * c + W * t;
            if constexpr (W == 8) {
                const float4 x0 = ld4(pa), x1 = ld4(pa + 4), y0 = ld4(pb), y1 = ld4(pb + 4);
                acc1(acc[0], x0.x, y0.x, metric); acc1(acc[1], x0.y, y0.y, metric);
                acc1(acc[2], x0.z, y0.z, metric); acc1(acc[3], x0.w, y0.w, metric);
                acc1(acc[4], x1.x, y1.x, metric); acc1(acc[5], x1.y, y1.y, metric);
                acc1(acc[6], x1.z, y1.z, metric); acc1(acc[7], x1.w, y1.w, metric);
            } else {
                const float2 x = *reinterpret_cast<const float2 *>(pa), y = *reinterpret_cast<const float2 *>(pb);
                acc1(acc[0], x.x, y.x, metric);
                acc1(acc[1], x.y, y.y, metric);
            }
        }
        float r;
        if constexpr (W == 8) {
            float tk[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float aj = __fadd_rn(acc[j], acc[j + 4]);
                tk[j] = __fadd_rn(aj, __shfl_xor_sync(mask, aj, 1));
            }
            r = __fadd_rn(__fadd_rn(tk[0], tk[1]), __fadd_rn(tk[2], tk[3]));
        } else {
            float u0 = __fadd_rn(acc[0], __shfl_xor_sync(mask, acc[0], 2));
            float u1 = __fadd_rn(acc[1], __shfl_xor_sync(mask, acc[1], 2));
            u0 = __fadd_rn(u0, __shfl_xor_sync(mask, u0, 4));
            u1 = __fadd_rn(u1, __shfl_xor_sync(mask, u1, 4));
            const float u = __fadd_rn(u0, u1);
            r = __fadd_rn(u, __shfl_xor_sync(mask, u, 1));
        }
        int i = chunks << 4;
        if (d - i >= 8) {   // as in group4_raw
            for (int e = i + 8; i < e; ++i) {
                float x = a[i], y = b[i];
                if (metric == METRIC_L2SQR) { x = __fsub_rn(x, y); y = x; }
                r = __fadd_rn(r, __fmul_rn(x, y));
            }
        }
        for (; i < d; ++i) {
            float x = a[i], y = b[i];
            if (metric == METRIC_L2SQR) { x = __fsub_rn(x, y); y = x; }
            r = __fmaf_rn(x, y, r);
        }
        return r;
    }
}

__device__ __forceinline__ float finish_metric(float raw, float n1, float n2, int metric) {
    if (metric == METRIC_EUCLIDEAN) return __fsub_rn(__fadd_rn(n1, n2), raw);
    if (metric == METRIC_ANGULAR) return __fdiv_rn(-raw, __fmaf_rn(n1, n2, FLT_EPSILON));
    return raw;
}

// Norm term of one row from its canonical norm2 (python-api.cpp:53-54, 63-64).
__device__ __forceinline__ float norm_term(float norm2, int metric) {
    if (metric == METRIC_EUCLIDEAN) return __fmul_rn(norm2, 0.5f);
    if (metric == METRIC_ANGULAR) return __fsqrt_rn(norm2);
    return 0.0f;
}

// Distance between dataset rows i and j (4-lane group).
__device__ __forceinline__ float pair_dist(const DataView &D, uint32_t i, uint32_t j, int t, unsigned mask) {
    float raw = group4_raw(D.X + (size_t)i * D.ld, D.X + (size_t)j * D.ld, D.d, D.metric, t, mask);
    if (D.metric == METRIC_L2SQR) return raw;
    return finish_metric(raw, D.norms[i], D.norms[j], D.metric);
}

// Distance between query q (norm term qn) and dataset row i (4-lane group).
// Argument order follows the reference: dist(dot(row, query), n_row, n_query).
__device__ __forceinline__ float query_dist(const DataView &D, const float *q, float qn, uint32_t i, int t,
                                            unsigned mask) {
    float raw = group4_raw(D.X + (size_t)i * D.ld, q, D.d, D.metric, t, mask);
    if (D.metric == METRIC_L2SQR) return raw;
    return finish_metric(raw, D.norms[i], qn, D.metric);
}

// query_dist with a D-split of G lanes (groupG_raw); the same bits for every G.
template <int G>
__device__ __forceinline__ float query_dist_g(const DataView &D, const float *q, float qn, uint32_t i, int t,
                                              unsigned mask) {
    float raw = groupG_raw<G>(D.X + (size_t)i * D.ld, q, D.d, D.metric, t, mask);
    if (D.metric == METRIC_L2SQR) return raw;
    return finish_metric(raw, D.norms[i], qn, D.metric);
}

__device__ __forceinline__ void raise_error(uint32_t *err, uint32_t bits) { atomicOr(err, bits); }

}  // namespace kgb
