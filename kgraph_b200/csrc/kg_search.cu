// Batched graph-walk search: KGraphImpl::search (kgraph.cpp:423-564) for a
// whole batch of queries in one persistent launch.
//
// Layout.  One warp owns one query at a time and pulls the next query index
// from a global counter, so queries with uneven K and P balance themselves.
// The warp keeps the query vector and its candidate pool (K+P+1 entries:
// dist, id|flag, m|M<<16 -- the reference's NeighborX) in shared memory, and
// a private N-bit visited set in global memory (the reference's
// dynamic_bitset, kgraph.cpp:438).  The compact pool (CP) packs an entry
// into 8 bytes -- dist, and id (the bits N needs) | expansion progress m/S
// (the remaining bits up to 31) | flag -- and reads M again from the node's
// {M, degree} when the entry is expanded, together with its first adjacency
// window: a third fewer bytes per entry, so more queries fit on an SM where
// the pool limits residency.
//
// Exactness.  The walk is the reference's, step for step: the same P seeds
// for every query (host mt19937(seed) + GenRandom, kgraph.cpp:444-453), the
// seed pool sorted by the GNU introsort (kgraph.cpp:476), neighbours visited
// in adjacency order S at a time, each inserted with UpdateKnnList
// semantics, k reset to the insert position (kgraph.cpp:478-514).  The
// distances of one batch of S neighbours are computed in parallel (they are
// pure), then inserted one by one in order, which is what the reference's
// interleaved loop produces.  With the canonical distance this reproduces
// the reference's ids, distances, result count and SearchInfo.cost exactly.
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <algorithm>
#include "kg_common.cuh"
#include "kg_warp.cuh"
#include "kg_sort.h"
#include "kg_search.h"

namespace kgb {

namespace {

template <bool HM>
struct PoolAcc {   // accessor for gnu_sort over the smem pool (with the m|M words when HM)
    float *d; uint32_t *i; uint32_t *m;
    struct Rec { float d; uint32_t i, m; };
    __device__ float key(int x) const { return d[x]; }
    __device__ void swap(int x, int y) const {
        float td = d[x]; d[x] = d[y]; d[y] = td;
        uint32_t ti = i[x]; i[x] = i[y]; i[y] = ti;
        if constexpr (HM) { uint32_t tm = m[x]; m[x] = m[y]; m[y] = tm; }
    }
    __device__ Rec get(int x) const { return Rec{d[x], i[x], HM ? m[x] : 0u}; }
    __device__ void put(int x, Rec r) const { d[x] = r.d; i[x] = r.i; if constexpr (HM) m[x] = r.m; }
    __device__ float rkey(Rec r) const { return r.d; }
};

struct WarpSmem {
    float *q;          // ld floats
    float *pd;         // cap
    uint32_t *pid;     // cap   id | FLAG_BIT
    uint32_t *pm;      // cap   m | (M << 16)
    float *rd;         // rcap  (T > 1 result merge)
    uint32_t *rid;     // rcap
    float *cd;         // 32    batch distances
    uint32_t *cid;     // 32    batch ids
    uint32_t *cM;      // 32    batch actual_M
};

template <int CP>
__device__ __forceinline__ WarpSmem carve(char *base, const SearchArgs &a) {
    WarpSmem s;
    char *p = base;
    s.q = reinterpret_cast<float *>(p); p += sizeof(float) * a.D.ld;
    s.pd = reinterpret_cast<float *>(p); p += sizeof(float) * a.cap;
    s.pid = reinterpret_cast<uint32_t *>(p); p += sizeof(uint32_t) * a.cap;
    s.pm = nullptr;
    if constexpr (!CP) { s.pm = reinterpret_cast<uint32_t *>(p); p += sizeof(uint32_t) * a.cap; }
    s.rd = reinterpret_cast<float *>(p); p += sizeof(float) * a.rcap;
    s.rid = reinterpret_cast<uint32_t *>(p); p += sizeof(uint32_t) * a.rcap;
    s.cd = reinterpret_cast<float *>(p); p += sizeof(float) * 32;
    s.cid = reinterpret_cast<uint32_t *>(p); p += sizeof(uint32_t) * 32;
    s.cM = reinterpret_cast<uint32_t *>(p);
    return s;
}

// actual_M (kgraph.cpp:284-286) as stored in NeighborX::M (uint16_t).
__device__ __forceinline__ uint32_t actual_M(const SearchArgs &a, uint32_t pM, uint32_t id) {
    uint32_t deg, M;
    if (a.meta) {
        uint2 md = a.meta[id];
        M = md.x;
        deg = md.y;
    } else {
        deg = (uint32_t)(a.offsets[id + 1] - a.offsets[id]);
        M = a.Mnode[id];
    }
    return min(max(M, pM), deg) & 0xFFFFu;
}

// Neighbour p of node: the ELL copy for p < ell_w, else the CSR.
__device__ __forceinline__ uint32_t neighbour(const SearchArgs &a, uint32_t node, uint32_t p) {
    if (a.ell && p < a.ell_w) return a.ell[(size_t)node * a.ell_w + p];
    return a.nbr[a.offsets[node] + p];
}

// Distances for cnt candidates cid[0..cnt) -> cd[], 32/G per pass (G-lane groups).
template <int G>
__device__ __forceinline__ void batch_dist(const SearchArgs &a, const WarpSmem &s, float qn, uint32_t cnt,
                                           int lane) {
    constexpr uint32_t PER = 32 / G;
    const int g = lane / G, t = lane % G;
    for (uint32_t base = 0; base < cnt; base += PER) {
        uint32_t c = base + g;
        uint32_t id = c < cnt ? s.cid[c] : 0u;
        float dd = query_dist_g<G>(a.D, s.q, qn, id, t, FULL);
        if (c < cnt && t == 0) s.cd[c] = dd;
    }
    __syncwarp();
}

// SearchOracle::search (kgraph.cpp:231-252) by one warp: every row in id
// order, epsilon filter, sorted insert into K slots (+1 overflow).
template <int G>
__device__ uint32_t warp_bruteforce(const SearchArgs &a, const WarpSmem &s, float qn, uint32_t K, int lane) {
    const uint32_t N = a.D.n;
    uint32_t L = 0;
    for (uint32_t base = 0; base < N; base += 32) {
        uint32_t cnt = min(32u, N - base);
        if (lane < (int)cnt) s.cid[lane] = base + lane;
        __syncwarp();
        batch_dist<G>(a, s, qn, cnt, lane);
        for (uint32_t c = 0; c < cnt; ++c) {
            float dd = s.cd[c];
            if (dd > a.epsilon) continue;
            if (L == K && (K == 0 || dd >= s.pd[K - 1])) continue;   // would land at slot K
            warp_update_knn(s.pd, s.pid, (uint32_t *)nullptr, L, dd, base + c, 0u, lane);
            if (L < K) ++L;
        }
        __syncwarp();
    }
    return L;
}

// Distances of the candidate lanes in `cm` (each holds its id), computed 32/G
// at a time by the G-lane groups; every candidate lane returns its own distance.
// The candidates' ids are compacted through the warp's 32-entry staging array
// (rank order), the distances come back by shuffle.
template <int G>
__device__ __forceinline__ float warp_cand_dist(const SearchArgs &a, const float *q, float qn, uint32_t *stage,
                                               unsigned cm, bool cand, uint32_t id, int lane) {
    constexpr uint32_t PER = 32 / G;
    const int g = lane / G, t = lane % G;
    const uint32_t n = __popc(cm);
    const uint32_t my = __popc(cm & ((1u << lane) - 1u));
    float mine = 0.f;
    if (cand) stage[my] = id;
    __syncwarp();
    for (uint32_t base = 0; base < n; base += PER) {
        const uint32_t i = base + g;
        const float dd = query_dist_g<G>(a.D, q, qn, i < n ? stage[i] : 0u, t, FULL);
        const float got = __shfl_sync(FULL, dd, (int)(G * (my % PER)));
        if (cand && my / PER == base / PER) mine = got;
    }
    __syncwarp();   // the staging array is reused by the next batch
    return mine;
}

// Hint: bring dataset row `id` into L2 (four 128-byte lines for D = 128).
__device__ __forceinline__ void prefetch_row(const DataView &D, uint32_t id) {
    const char *p = reinterpret_cast<const char *>(D.X + (size_t)id * D.ld);
    const uint32_t bytes = D.ld * 4;
    for (uint32_t o = 0; o < bytes; o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(p + o));
}

__device__ __forceinline__ bool visited_test_set(uint32_t *vis, uint32_t id) {
    uint32_t bit = 1u << (id & 31);
    uint32_t old = atomicOr(vis + (id >> 5), bit);
    return (old & bit) != 0;
}

// ---- the distance filter on compressed rows (kg_precision.cu) ----
constexpr float U32 = 5.9604645e-8f;   // unit roundoff of FP32, 2^-24

// The W reconstructed values of `row` at elements [off, off + W): BF16 values,
// or FP8 E4M3 values times the row's scale (rounded to FP32, as the error
// bound of the compressed row assumes).
template <int PREC, int W>
__device__ __forceinline__ void load_y(const void *Xc, uint32_t ld, uint32_t row, uint32_t off, float scale,
                                       float *y) {
    if constexpr (PREC == 1) {
        const uint16_t *p = reinterpret_cast<const uint16_t *>(Xc) + (size_t)row * ld + off;
        uint32_t w[W / 2];
        if constexpr (W == 8) { const uint4 v = *reinterpret_cast<const uint4 *>(p); w[0] = v.x; w[1] = v.y; w[2] = v.z; w[3] = v.w; }
        else if constexpr (W == 4) { const uint2 v = *reinterpret_cast<const uint2 *>(p); w[0] = v.x; w[1] = v.y; }
        else { w[0] = *reinterpret_cast<const uint32_t *>(p); }
#pragma unroll
        for (int j = 0; j < W / 2; ++j) {
            y[2 * j] = __uint_as_float(w[j] << 16);
            y[2 * j + 1] = __uint_as_float(w[j] & 0xFFFF0000u);
        }
    } else {
        const uint8_t *p = reinterpret_cast<const uint8_t *>(Xc) + (size_t)row * ld + off;
        uint16_t h[W / 2];
        if constexpr (W == 8) {
            const uint2 v = *reinterpret_cast<const uint2 *>(p);
            h[0] = (uint16_t)v.x; h[1] = (uint16_t)(v.x >> 16); h[2] = (uint16_t)v.y; h[3] = (uint16_t)(v.y >> 16);
        } else if constexpr (W == 4) {
            const uint32_t v = *reinterpret_cast<const uint32_t *>(p);
            h[0] = (uint16_t)v; h[1] = (uint16_t)(v >> 16);
        } else {
            h[0] = *reinterpret_cast<const uint16_t *>(p);
        }
#pragma unroll
        for (int j = 0; j < W / 2; ++j) {
            const __half2_raw r = __nv_cvt_fp8x2_to_halfraw2((__nv_fp8x2_storage_t)h[j], __NV_E4M3);
            const float2 f = __half22float2(__half2(r));
            y[2 * j] = __fmul_rn(f.x, scale);
            y[2 * j + 1] = __fmul_rn(f.y, scale);
        }
    }
}

// Sum over the row of (q - y)^2 (dot q.y for angular) with FP32 accumulation,
// by the G-lane group of this lane; every lane of the group gets the sum.
template <int PREC, int G>
__device__ __forceinline__ float approx_raw(const SearchArgs &a, const float *q, uint32_t row, int t, float scale) {
    constexpr int W = 16 / G;
    const bool dot = a.D.metric == METRIC_ANGULAR;
    float acc = 0.f;
    const uint32_t chunks = a.D.ld >> 4;
    for (uint32_t c = 0; c < chunks; ++c) {
        const uint32_t off = 16 * c + W * t;
        float y[W];
        load_y<PREC, W>(a.Xc, a.D.ld, row, off, scale, y);
#pragma unroll
        for (int j = 0; j < W; ++j) {
            const float qj = q[off + j];
            if (dot) acc = __fmaf_rn(qj, y[j], acc);
            else { const float df = __fsub_rn(qj, y[j]); acc = __fmaf_rn(df, df, acc); }
        }
    }
#pragma unroll
    for (int o = G / 2; o; o >>= 1) acc = __fadd_rn(acc, __shfl_xor_sync(FULL, acc, o));
    return acc;
}

// Rigorous lower bound of the canonical FP32 distance (kg_common.cuh) of a row
// x from `raw` (approx_raw over its reconstruction y, ||x - y|| <= e), the
// query's and the row's norm terms nq, nx.  gamma_k = k u bounds the relative
// error of a k-deep FP32 sum: ld + 8 deep for approx_raw, d/16 + 24 for the
// canonical distance (16 lanes, a 4-level tree, up to 15 tail terms).  Every
// step rounds towards the bound.
__device__ __forceinline__ float filter_lb(int metric, float raw, float e, float nq, float nx, uint32_t d,
                                           uint32_t ld) {
    const float ga = (float)(ld + 8) * U32 * 1.01f;
    const float gc = (float)(d / 16 + 24) * U32 * 1.01f;
    if (metric == METRIC_ANGULAR) {
        // -dot_c >= -dot' - ||q|| (e + ga ||y|| + gc ||x||);  ||q|| <= nq (1 + 2 gc), ||x|| <= nx (1 + 2 gc),
        // ||y|| <= ||x|| + e; the canonical denominator is recomputed bit for bit, and rounding is monotone
        const float qn = __fmul_ru(nq, 1.f + 2.f * gc);
        const float xn = __fmul_ru(nx, 1.f + 2.f * gc);
        const float yn = __fadd_ru(xn, e);
        const float B = __fmul_ru(qn, __fadd_ru(e, __fadd_ru(__fmul_ru(ga, yn), __fmul_ru(gc, xn))));
        const float num = __fsub_rd(-raw, B);
        return __fdiv_rd(num, __fmaf_rn(nx, nq, FLT_EPSILON));
    }
    // ||q - y||^2 >= raw (1 - ga) and ||q - x|| >= ||q - y|| - e
    const float r = __fsqrt_rd(fmaxf(__fmul_rd(raw, 1.f - ga), 0.f));
    const float b = fmaxf(__fsub_rd(r, e), 0.f);
    const float t2 = __fmul_rd(b, b);   // <= ||q - x||^2
    if (metric == METRIC_L2SQR) return __fmul_rd(t2, 1.f - 2.f * gc);   // canonical >= ||q-x||^2 (1 - gamma)
    // euclidean: canonical (n_q + n_x) - dot >= ||q - x||^2 / 2 - 2.2 gc (n_q + n_x)
    return __fsub_rd(__fmul_rd(t2, 0.5f), __fmul_ru(2.2f * gc, __fadd_ru(nq, nx)));
}

// Lower bounds of the candidate lanes in `cm` from their compressed rows,
// 32/G per pass; every candidate lane returns its own bound.
template <int PREC, int G>
__device__ __forceinline__ float warp_cand_lb(const SearchArgs &a, const float *q, float qn, unsigned cm, bool cand,
                                              uint32_t id, int lane) {
    constexpr uint32_t PER = 32 / G;
    const int g = lane / G, t = lane % G;
    const uint32_t n = __popc(cm);
    const uint32_t my = __popc(cm & ((1u << lane) - 1u));
    float mine = 0.f;
    for (uint32_t base = 0; base < n; base += PER) {
        const uint32_t i = base + g;
        const int src = i < n ? (int)__fns(cm, 0, i + 1) : 0;
        const uint32_t cid = __shfl_sync(FULL, id, src);
        const uint32_t row = i < n ? cid : 0u;
        const float4 md = a.cmeta[row];   // {error bound, scale, norm term, 0}
        const float raw = approx_raw<PREC, G>(a, q, row, t, md.y);
        const float lb = filter_lb(a.D.metric, raw, md.x, qn, md.z, a.D.d, a.D.ld);
        const float got = __shfl_sync(FULL, lb, (int)(G * (my % PER)));
        if (cand && my / PER == base / PER) mine = got;
    }
    return mine;
}

// L2 prefetch of a compressed row.
template <int PREC>
__device__ __forceinline__ void prefetch_crow(const SearchArgs &a, uint32_t id) {
    const uint32_t bytes = a.D.ld * (PREC == 1 ? 2u : 1u);
    const char *p = reinterpret_cast<const char *>(a.Xc) + (size_t)id * bytes;
    for (uint32_t o = 0; o < bytes; o += 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(p + o));
}

}  // namespace

// G: lanes per distance (the D-split, 32/G candidates per pass); PF: neighbour
// batches whose rows are prefetched into L2 ahead of the walk; PREC: 0, or the
// compressed rows (1 BF16, 2 FP8) that filter candidates once the pool is full.
// MB: resident blocks of 256 threads per SM the register allocation is sized
// for (4: 64 registers per thread; 3: 80, fewer spills for large pools, whose
// shared memory limits residency anyway), or 9: blocks of at most 128
// threads at 56 registers (36 warps per SM instead of 32).  CP: the compact 8-byte pool entry
// (the host selects it only when every node's expansion fits the progress
// field: a.cp_idbits id bits, 31 - a.cp_idbits progress bits).
template <int G, int PF, int PREC, int MB, int CP>
__global__ void __launch_bounds__(MB == 9 ? 128 : 256, MB) search_kernel(SearchArgs a) {
    extern __shared__ __align__(16) char smem[];
    const uint32_t IDM = CP ? (1u << a.cp_idbits) - 1u : ID_MASK;   // the id bits of a pool word
    const uint32_t PMASK = CP ? ID_MASK >> a.cp_idbits : 0u;        // the progress bits, shifted down
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const uint32_t slot = blockIdx.x * a.warps_per_block + wib;
    WarpSmem s = carve<CP>(smem + (size_t)wib * a.warp_smem_bytes, a);
    uint32_t *vis = a.visited + (size_t)slot * a.vwords;
    const uint32_t N = a.D.n;

    for (;;) {
        uint32_t qi = 0;
        if (lane == 0) qi = atomicAdd(a.qcounter, 1u);
        qi = __shfl_sync(FULL, qi, 0);
        if (qi >= a.nq) break;
        const uint32_t K = a.Kq ? a.Kq[qi] : a.K;
        const uint32_t P = a.Pq ? a.Pq[qi] : a.P;
        const uint32_t T = a.T;
        const uint32_t S = a.S;
        const uint32_t cap = K + P + 1;   // knn.size(), kgraph.cpp:434

        // query -> smem, and its norm term (SearchOracle ctor, python-api.cpp:98-101).  The padding
        // columns [d, ld) of a caller's row may hold anything; the smem copy holds zeros there, so the
        // compressed-row filter, which sums over whole 16-column chunks, sees (0 - 0)^2 terms.
        const float *qg = a.Q + (size_t)qi * a.q_ld;
        for (uint32_t x = lane * 4; x < a.D.ld; x += 128) {
            float4 v = ld4(qg + x);
            if (x + 4 > a.D.d) {
                if (x + 0 >= a.D.d) v.x = 0.f;
                if (x + 1 >= a.D.d) v.y = 0.f;
                if (x + 2 >= a.D.d) v.z = 0.f;
                if (x + 3 >= a.D.d) v.w = 0.f;
            }
            *reinterpret_cast<float4 *>(s.q + x) = v;
        }
        __syncwarp();
        float qn = 0.f;
        if (a.D.metric != METRIC_L2SQR) {
            float n2 = group4_raw(s.q, s.q, a.D.d, METRIC_EUCLIDEAN, lane & 3, FULL);
            qn = norm_term(n2, a.D.metric);
        }

        uint32_t count = 0;
        float cost = 0.f;
        uint32_t *out_i = a.out_ids + (size_t)qi * a.out_ld;
        float *out_d = a.out_dists ? a.out_dists + (size_t)qi * a.out_ld : nullptr;

        if (P >= N) {   // kgraph.cpp:427-433: brute force, cost 1
            count = warp_bruteforce<G>(a, s, qn, K, lane);
            for (uint32_t k = lane; k < count; k += 32) {
                out_i[k] = s.pid[k] & ID_MASK;
                if (out_d) out_d[k] = s.pd[k];
            }
            if (lane == 0) { a.out_count[qi] = count; if (a.out_cost) a.out_cost[qi] = 1.0f; }
            __syncwarp();
            continue;
        }
        if (a.init && !(a.init < K)) {   // kgraph.cpp:463
            if (lane == 0) { raise_error(a.err, ERR_INIT_K); a.out_count[qi] = 0; }
            __syncwarp();
            continue;
        }

        for (uint32_t w = lane * 4; w < a.vwords; w += 128)
            *reinterpret_cast<uint4 *>(vis + w) = make_uint4(0u, 0u, 0u, 0u);
        __syncwarp();

        uint32_t n_comps = 0, n_adj = 0, n_seed = 0, n_apx = 0, n_skip = 0;
        uint32_t rn = 0;          // results.size() - 1
        bool have_results = false;
        for (uint32_t trial = 0; trial < T; ++trial) {
            uint32_t L = 0;
            if (a.init == 0) {
                const uint32_t *seeds = a.seeds + a.seed_index[qi] + (size_t)trial * P;
                // kgraph.cpp:454-459: keep seeds not visited by an earlier trial
                for (uint32_t base = 0; base < P; base += 32) {
                    uint32_t j = base + lane;
                    uint32_t sid = j < P ? seeds[j] : 0u;
                    bool keep = j < P && !((__ldcg(vis + (sid >> 5)) >> (sid & 31)) & 1u);
                    unsigned m = __ballot_sync(FULL, keep);
                    if (keep) s.pid[L + __popc(m & ((1u << lane) - 1u))] = sid;
                    L += __popc(m);
                }
            } else {
                L = a.init;
                const uint32_t *init = a.init_ids + (size_t)qi * a.out_ld;
                for (uint32_t j = lane; j < L; j += 32) s.pid[j] = init[j];
            }
            __syncwarp();
            n_seed += L;
            // kgraph.cpp:468-475: mark, flag, distance, m = 0, M = actual_M
            for (uint32_t base = 0; base < L; base += 32) {
                uint32_t j = base + lane;
                uint32_t id = j < L ? s.pid[j] : 0u;
                bool bad = j < L && id >= N;
                if (__any_sync(FULL, bad)) {
                    if (lane == 0) raise_error(a.err, ERR_BAD_ID);
                }
                if (j < L && !bad) {
                    atomicOr(vis + (id >> 5), 1u << (id & 31));
                    if constexpr (!CP) s.pm[j] = actual_M(a, a.Mp, id) << 16;
                }
                __syncwarp();
                uint32_t cnt = min(32u, L - base);
                if (j < L) s.cid[lane] = bad ? 0u : id;
                __syncwarp();
                batch_dist<G>(a, s, qn, cnt, lane);
                // an out-of-range starting point (the error is raised above) enters as id 0,
                // unflagged: it is never expanded, so no adjacency row is read for it
                if (j < L) { s.pd[j] = s.cd[lane]; s.pid[j] = bad ? 0u : (id | FLAG_BIT); }
                __syncwarp();
            }
            // kgraph.cpp:476: std::sort by dist (GNU introsort order for ties)
            if (lane == 0) {
                PoolAcc<!CP> acc{s.pd, s.pid, s.pm};
                gnu_sort(acc, 0, (int)L);
            }
            __syncwarp();

            uint32_t k = 0;
            // Each expansion advances m or clears a flag of an entry that was inserted
            // once, so the walk ends; the bound only turns a defect into an error.
            const uint64_t step_limit = 64ull * (N + cap) + 4096;
            uint64_t steps = 0;
            // The expansion loop of kgraph.cpp:478-514.  The entry at k is expanded
            // batch after batch (S neighbours each) exactly as the reference's loop
            // does while no insert lands at or before k.  Its adjacency entries come
            // in windows of up to 128 (four per lane) with one round trip for the
            // ids and one for their visited bits (this warp's private set, so the
            // bits can only change by this walk); a batch's unvisited neighbours are
            // then confirmed with an atomic test-and-set (exact even when an id
            // recurs across chunks), their distances computed and inserted in one
            // merge.  When an insert lands at or before k the reference moves on to
            // another entry: so does this loop, and the window is dropped (it is
            // reloaded from m when the entry comes up again).
            while (true) {
                k = warp_next_flagged(s.pid, k, L, lane);
                if (k >= L) break;
                const uint32_t pk = s.pid[k];
                const uint32_t node = pk & IDM;
                uint32_t eM, m, bq = 0;
                uint32_t wid[4];
                bool pre = false;   // CP: wid holds the ELL ids of the window at m
                if constexpr (CP) {
                    // the node's {M, degree} and its first window's ELL ids in flight together
                    bq = (pk >> a.cp_idbits) & PMASK;
                    m = bq * S;
                    if (a.ell) {
#pragma unroll
                        for (int c = 0; c < 4; ++c) {
                            const uint32_t p = m + 32 * c + lane;
                            wid[c] = p < a.ell_w ? a.ell[(size_t)node * a.ell_w + p] : 0xFFFFFFFFu;
                        }
                        pre = true;
                    }
                    eM = actual_M(a, a.Mp, node);
                } else {
                    const uint32_t mM0 = s.pm[k];
                    eM = mM0 >> 16;
                    m = mM0 & 0xFFFFu;
                }
                uint32_t wlo = 0, whi = 0;   // loaded window [wlo, whi)
                bool wuv[4];
                bool moved = false;
                while (true) {
                    if (++steps > step_limit) {
                        if (lane == 0) raise_error(a.err, ERR_STEP_LIMIT);
                        k = L;
                        break;
                    }
                    // kgraph.cpp:485-491: the entry's next batch
                    const uint32_t beginM = m;
                    uint32_t endM = beginM + S;
                    const bool done = endM > eM;
                    if (done) endM = eM;
                    if (lane == 0) {
                        if constexpr (CP) {   // progress in batches of S: endM = (bq + 1) S unless done
                            s.pid[k] = done ? node : (node | FLAG_BIT | ((bq + 1) << a.cp_idbits));
                        } else {
                            if (done) s.pid[k] = s.pid[k] & ID_MASK;
                            s.pm[k] = (endM & 0xFFFFu) | (eM << 16);
                        }
                    }
                    __syncwarp();
                    n_adj += endM - beginM;
                    // kgraph.cpp:495-513.  A batch of at most 32 neighbours is one unit (lane j
                    // holds neighbour beginM + j, gathered from the window, which is reloaded
                    // when it does not hold the whole batch); a longer batch (S > 32) goes in
                    // pieces that stay inside one 32-entry chunk.
                    const bool whole = endM - beginM <= 32;   // warp-uniform
                    for (uint32_t p0 = beginM; p0 < endM;) {
                        if (whole ? (p0 < wlo || endM > whi) : (p0 < wlo || p0 >= whi)) {   // load the window at p0
                            wlo = p0;
                            whi = min(p0 + 128u, eM);
#pragma unroll
                            for (int c = 0; c < 4; ++c) {
                                const uint32_t p = wlo + 32 * c + lane;
                                const bool act = p < whi;
                                uint32_t id = 0xFFFFFFFFu;
                                if (act) id = (CP && pre && p < a.ell_w) ? wid[c] : neighbour(a, node, p);
                                const bool bad = act && id >= N;
                                if (__any_sync(FULL, bad)) { if (lane == 0) raise_error(a.err, ERR_BAD_ID); }
                                const bool ok = act && !bad;
                                const unsigned same = __match_any_sync(FULL, id);
                                const unsigned okm = __ballot_sync(FULL, ok);   // every lane votes
                                wid[c] = id;
                                wuv[c] = ok && ((__ffs(same & okm) - 1) == lane);
                            }
#pragma unroll
                            for (int c = 0; c < 4; ++c)   // first occurrences not yet visited
                                if (wuv[c]) wuv[c] = !((__ldcg(vis + (wid[c] >> 5)) >> (wid[c] & 31)) & 1u);
                            pre = false;
                        }
                        const uint32_t c = (p0 - wlo) >> 5;
                        uint32_t id = 0, p1;
                        bool cand;
                        if (whole) {
                            // the batch spans window chunks c and c + 1 at most
                            uint32_t idA = 0, idB = 0;
                            bool uvA = false, uvB = false;
#pragma unroll
                            for (int cc = 0; cc < 4; ++cc) {
                                if ((uint32_t)cc == c) { idA = wid[cc]; uvA = wuv[cc]; }
                                if ((uint32_t)cc == c + 1) { idB = wid[cc]; uvB = wuv[cc]; }
                            }
                            const uint32_t pos = p0 - wlo + lane;   // window position of this lane's neighbour
                            const int src = (int)(pos & 31);
                            const uint32_t ia = __shfl_sync(FULL, idA, src), ib = __shfl_sync(FULL, idB, src);
                            const bool ua = __shfl_sync(FULL, uvA, src), ub = __shfl_sync(FULL, uvB, src);
                            const bool second = (pos >> 5) != c;
                            id = second ? ib : ia;
                            const bool uv = (uint32_t)lane < endM - p0 && (second ? ub : ua);
                            // an id in both chunks: its first position only, as the reference's
                            // in-order loop marks it visited there (kgraph.cpp:497-498)
                            const unsigned same = __match_any_sync(FULL, uv ? id : 0xFFFFFFFFu);
                            cand = uv && (__ffs(same) - 1) == lane;
                            p1 = endM;
                        } else {
                            const uint32_t cbase = wlo + 32 * c;
                            p1 = min(endM, cbase + 32);
                            const uint32_t lo = p0 - cbase, hi = p1 - cbase;
                            bool uv = false;
#pragma unroll
                            for (int cc = 0; cc < 4; ++cc)
                                if ((uint32_t)cc == c) { id = wid[cc]; uv = wuv[cc]; }
                            cand = uv && (uint32_t)lane >= lo && (uint32_t)lane < hi;
                        }
                        const unsigned cm = __ballot_sync(FULL, cand);
                        // L2 prefetch of the rows the next PF batches of this entry will
                        // read (unvisited window ids), behind this batch's loads
                        if constexpr (PF > 0) {
#pragma unroll
                            for (int cc = 0; cc < 4; ++cc) {
                                const uint32_t pos = wlo + 32 * cc + lane;
                                if (wuv[cc] && pos >= p1 && pos < p1 + PF * S && pos < whi) {
                                    if (PREC && L == cap - 1) prefetch_crow<PREC>(a, wid[cc]);
                                    else prefetch_row(a.D, wid[cc]);
                                }
                            }
                        }
                        if (PREC && cm && L == cap - 1) {
                            // Full pool: the visited test-and-set and the compressed rows in flight
                            // together; the lower bound drops candidates that would land in the
                            // spare slot, the others take the FP32 path below, restricted to them.
                            bool isnew = false;
                            if (cand) {
                                const uint32_t bit = 1u << (id & 31);
                                isnew = !(atomicOr(vis + (id >> 5), bit) & bit);
                            }
                            const float lb = warp_cand_lb<PREC, G>(a, s.q, qn, cm, cand, id, lane);
                            const float worst = s.pd[L - 1];
                            const bool keep = isnew && !(lb >= worst);
                            const unsigned nm = __ballot_sync(FULL, isnew);
                            const unsigned km = __ballot_sync(FULL, keep);
                            n_comps += __popc(nm);
                            n_apx += __popc(nm);
                            n_skip += __popc(nm & ~km);
                            if (km) {
                                const uint32_t aM = (!CP && keep) ? actual_M(a, a.Mp, id) : 0u;
                                const float dd = warp_cand_dist<G>(a, s.q, qn, s.cid, km, keep, id, lane);
                                const unsigned im = __ballot_sync(FULL, keep && dd < worst);
                                if (im) {
                                    uint32_t mr;
                                    L = warp_batch_insert(s.pd, s.pid, CP ? nullptr : s.pm, L, cap, im, dd, id | FLAG_BIT, aM << 16,
                                                          &mr, lane);
                                    if (mr <= k) moved = true;
                                    if (mr < k) k = mr;
                                }
                            }
                        } else if (cm) {
                            // All three in flight together: the exact test-and-set of the
                            // visited bit, the candidate's {M, degree}, and its row (distance).
                            bool isnew = false;
                            uint32_t aM = 0;
                            if (cand) {
                                const uint32_t bit = 1u << (id & 31);
                                isnew = !(atomicOr(vis + (id >> 5), bit) & bit);
                                if constexpr (!CP) aM = actual_M(a, a.Mp, id);
                            }
                            const float dd = warp_cand_dist<G>(a, s.q, qn, s.cid, cm, cand, id, lane);
                            const unsigned nm = __ballot_sync(FULL, isnew);
                            n_comps += __popc(nm);
                            // A full pool takes a candidate only below its last entry: one at or
                            // above it lands in the spare slot (kgraph.cpp:503-506), and so does
                            // every later candidate of the batch that is not closer than it, so
                            // leaving those out of the merge changes no position.
                            const unsigned im =
                                L == cap - 1 ? __ballot_sync(FULL, isnew && dd < s.pd[L - 1]) : nm;
                            if (im) {
                                uint32_t mr;   // new entries: flag set, m = 0, M = actual_M
                                L = warp_batch_insert(s.pd, s.pid, CP ? nullptr : s.pm, L, cap, im, dd, id | FLAG_BIT, aM << 16,
                                                      &mr, lane);
                                if (mr <= k) moved = true;   // the expanded entry is no longer at k
                                if (mr < k) k = mr;
                            }
                        }
                        p0 = p1;
                    }
                    m = endM;
                    ++bq;
                    if (done || moved) break;   // the loop head picks the reference's next k
                }
                if (k >= L) break;
            }
            if (L > K) L = K;   // kgraph.cpp:515
            if (!have_results) {
                for (uint32_t j = lane; j < L; j += 32) { s.rd[j] = s.pd[j]; s.rid[j] = s.pid[j] & (IDM | FLAG_BIT); }
                rn = L;
                have_results = true;
                __syncwarp();
            } else {   // kgraph.cpp:521-528
                for (uint32_t l = 0; l < L; ++l) {
                    uint32_t r = warp_update_knn(s.rd, s.rid, (uint32_t *)nullptr, rn, s.pd[l], s.pid[l] & (IDM | FLAG_BIT),
                                                 0u, lane);
                    if (r < rn + 1 && rn + 1 < K + 1) ++rn;
                }
            }
        }
        // kgraph.cpp:531-540: drop the spare slot, epsilon filter
        count = rn;
        for (uint32_t base = 0; base < count; base += 32) {
            uint32_t j = base + lane;
            unsigned m = __ballot_sync(FULL, j < count && s.rd[j] > a.epsilon);
            if (m) { count = base + __ffs(m) - 1; break; }
        }
        for (uint32_t k = lane; k < count; k += 32) {
            out_i[k] = s.rid[k] & ID_MASK;
            if (out_d) out_d[k] = s.rd[k];
        }
        cost = __fdiv_rn((float)n_comps, (float)N);   // kgraph.cpp:561
        if (lane == 0) {
            a.out_count[qi] = count;
            if (a.out_cost) a.out_cost[qi] = cost;
            if (a.work) {
                atomicAdd(a.work, (unsigned long long)(n_comps + n_seed));
                atomicAdd(a.work + 1, (unsigned long long)n_adj);
                if (PREC && n_apx) {
                    atomicAdd(a.work + 2, (unsigned long long)n_apx);
                    atomicAdd(a.work + 3, (unsigned long long)n_skip);
                }
            }
        }
        __syncwarp();
    }
}

// The filter's lower bound and the canonical distance for `per` dataset rows
// per query (one warp per query, one 4-lane group per row): the check of the
// bound's arithmetic, lb <= dist for every pair.
template <int PREC>
__global__ void __launch_bounds__(256) filter_bounds_kernel(SearchArgs a, const uint32_t *ids, uint32_t per, float *lb,
                                                            float *dist) {
    __shared__ __align__(16) float qs[8][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t qi = blockIdx.x * 8 + w;
    if (qi >= a.nq) return;   // whole warps
    float *q = qs[w];
    for (uint32_t x = lane; x < a.D.ld; x += 32) q[x] = x < a.D.d ? a.Q[(size_t)qi * a.q_ld + x] : 0.f;
    __syncwarp();
    float qn = 0.f;
    if (a.D.metric != METRIC_L2SQR) qn = norm_term(group4_raw(q, q, a.D.d, METRIC_EUCLIDEAN, lane & 3, FULL), a.D.metric);
    const int g = lane >> 2, t = lane & 3;
    for (uint32_t base = 0; base < per; base += 8) {
        const uint32_t j = base + g;
        const uint32_t row = j < per ? ids[(size_t)qi * per + j] : 0u;
        const float4 md = a.cmeta[row];
        const float raw = approx_raw<PREC, 4>(a, q, row, t, md.y);
        const float b = filter_lb(a.D.metric, raw, md.x, qn, md.z, a.D.d, a.D.ld);
        const float dd = query_dist(a.D, q, qn, row, t, FULL);
        if (j < per && t == 0) {
            lb[(size_t)qi * per + j] = b;
            dist[(size_t)qi * per + j] = dd;
        }
    }
}

cudaError_t launch_filter_bounds(const SearchArgs &a, const uint32_t *ids, uint32_t per, float *lb, float *dist,
                                 cudaStream_t st) {
    if (a.D.ld > 256) return cudaErrorInvalidValue;
    const uint32_t grid = (a.nq + 7) / 8;
    if (a.prec == 1) filter_bounds_kernel<1><<<grid, 256, 0, st>>>(a, ids, per, lb, dist);
    else if (a.prec == 2) filter_bounds_kernel<2><<<grid, 256, 0, st>>>(a, ids, per, lb, dist);
    else return cudaErrorInvalidValue;
    return cudaGetLastError();
}

size_t search_warp_smem_bytes(uint32_t ld, uint32_t cap, uint32_t rcap, bool compact) {
    size_t b = sizeof(float) * ld + (compact ? 8ull : 12ull) * cap + 8ull * rcap + 12ull * 32;
    return (b + 15) & ~size_t(15);
}

namespace {

using SearchFn = void (*)(SearchArgs);
template <int PREC, int MB, int CP>
SearchFn search_fn_prec(uint32_t split, bool pf) {
    switch (split) {
        case 2: return pf ? search_kernel<2, 2, PREC, MB, CP> : search_kernel<2, 0, PREC, MB, CP>;
        case 8: return pf ? search_kernel<8, 2, PREC, MB, CP> : search_kernel<8, 0, PREC, MB, CP>;
        default: return pf ? search_kernel<4, 2, PREC, MB, CP> : search_kernel<4, 0, PREC, MB, CP>;
    }
}
// The compiled (D-split, prefetch, filter precision, register budget, pool
// entry) variants; the 80-register budget and the compact pool exist for the
// FP32 walk.
SearchFn search_fn(uint32_t split, uint32_t prefetch, uint32_t prec, uint32_t regs, bool compact) {
    const bool pf = prefetch > 0;
    if (prec == 1) return search_fn_prec<1, 4, 0>(split, pf);
    if (prec == 2) return search_fn_prec<2, 4, 0>(split, pf);
    if (compact) {
        if (regs == 56) return search_fn_prec<0, 9, 1>(split, pf);
        return regs == 80 ? search_fn_prec<0, 3, 1>(split, pf) : search_fn_prec<0, 4, 1>(split, pf);
    }
    return regs == 80 ? search_fn_prec<0, 3, 0>(split, pf) : search_fn_prec<0, 4, 0>(split, pf);
}
// The compact pool runs where the shape asks for it and the graph allows it.
bool use_compact(const SearchArgs &a, const SearchShape &sh) { return search_uses_compact(a, sh); }

// Warps per block: the requested query tile, or as many as fit 200 KB of
// shared memory (at most 8); halved until the block fits.
uint32_t pick_wpb(const SearchShape &sh, size_t warp_bytes) {
    const uint32_t most = sh.regs == 56 ? 4u : 8u;   // the 56-register variant takes blocks of at most 128 threads
    uint32_t wpb = sh.warps_per_block ? std::min<uint32_t>(sh.warps_per_block, most) : most;
    while (wpb > 1 && (size_t)wpb * warp_bytes > 200 * 1024) wpb >>= 1;
    return wpb;
}

}  // namespace

bool search_uses_compact(const SearchArgs &a, const SearchShape &sh) {
    return sh.compact && a.compact_ok && a.prec == 0;
}

bool search_shape_valid(const SearchShape &sh) {
    const bool split_ok = sh.split == 0 || sh.split == 2 || sh.split == 4 || sh.split == 8;
    const bool wpb_ok = sh.warps_per_block == 0 || sh.warps_per_block == 1 || sh.warps_per_block == 2 ||
                        sh.warps_per_block == 4 || sh.warps_per_block == 8;
    const bool pf_ok = sh.prefetch == 0 || sh.prefetch == 2;
    const bool regs_ok = sh.regs == 0 || sh.regs == 56 || sh.regs == 64 || sh.regs == 80;
    return split_ok && wpb_ok && pf_ok && regs_ok && sh.compact <= 1;
}

cudaError_t launch_search(SearchArgs &a, const SearchShape &sh, int num_sms, cudaStream_t st, uint32_t *grid_out) {
    const bool cp = use_compact(a, sh);
    a.warp_smem_bytes = (uint32_t)search_warp_smem_bytes(a.D.ld, a.cap, a.rcap, cp);
    const uint32_t wpb = pick_wpb(sh, a.warp_smem_bytes);
    if ((size_t)wpb * a.warp_smem_bytes > 227 * 1024) return cudaErrorInvalidValue;
    a.warps_per_block = wpb;
    size_t smem = (size_t)wpb * a.warp_smem_bytes;
    SearchFn fn = search_fn(sh.split, sh.prefetch, a.prec, sh.regs, cp);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, wpb * 32, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    uint32_t grid = (uint32_t)(num_sms * per_sm);
    uint32_t need = (a.nq + wpb - 1) / wpb;
    if (grid > need) grid = need;
    if (grid < 1) grid = 1;
    if (grid_out) *grid_out = grid;
    if (grid * wpb > a.visited_slots) return cudaErrorInvalidValue;
    fn<<<grid, wpb * 32, smem, st>>>(a);
    return cudaGetLastError();
}

uint32_t search_max_slots(const SearchArgs &a, const SearchShape &sh, int num_sms) {
    const bool cp = use_compact(a, sh);
    const size_t wb = search_warp_smem_bytes(a.D.ld, a.cap, a.rcap, cp);
    const uint32_t wpb = pick_wpb(sh, wb);
    const size_t smem = (size_t)wpb * wb;
    SearchFn fn = search_fn(sh.split, sh.prefetch, a.prec, sh.regs, cp);
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, wpb * 32, smem);
    if (per_sm < 1) per_sm = 1;
    return (uint32_t)(num_sms * per_sm) * wpb;
}

}  // namespace kgb
