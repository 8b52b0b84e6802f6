// NN-descent construction on the GPU: KGraphConstructor (kgraph.cpp:705-1001).
//
// Per node the state lives in HBM as structure-of-arrays rows (kg_build.h).
// One iteration is the reference's  join -> statistics -> stop test -> update:
//
//   join_kernel      one warp per node: every new x new pair (i < j by id) and
//                    new x old pair, canonical FP32 distance by 4-lane groups
//                    (8 pairs per pass), then Nhood::parallel_try_insert into
//                    both pools: unlocked radius test, per-node lock, the
//                    warp's sorted insert with the reference's duplicate and
//                    overflow-slot rules (kgraph.cpp:723-736, 797-815).
//   stats kernels    delta, mean M, control recall/accuracy (kgraph.cpp:927-963).
//   update kernels   radius = pool[L], M growth, radiusM, new/old split with
//                    flag clearing, reverse samples by the radiusM rule in an
//                    exact count-scan-fill CSR, then a uniform R-subset per
//                    node (kgraph.cpp:816-883).
//
// Randomness.  The reference's init draws from one mt19937 per OpenMP thread
// and its R cap from the C library rand(), so its graph depends on thread
// count and scheduling.  Here each node draws from its own SplitMix64 stream
// keyed by (seed, node, purpose): same GenRandom algorithm and distribution,
// independent of launch shape.
#include <cub/cub.cuh>
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <iostream>
#include <numeric>
#include <random>
#include "kg_build.h"
#include "kg_ctx.h"
#include "kg_sort.h"
#include "kg_insert.cuh"
#include "kg_warp.cuh"

namespace kgb {

unsigned g_verbosity = 1;

namespace {

// SplitMix64 (Steele, Lea, Flood 2014): one stream per (seed, node, purpose).
struct Rng {
    uint64_t s;
    __device__ uint32_t next() {
        s += 0x9E3779B97F4A7C15ull;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return (uint32_t)((z ^ (z >> 31)) >> 32);
    }
};
__device__ Rng make_rng(uint64_t seed, uint64_t node, uint64_t purpose) {
    Rng r{seed ^ (node * 0xD1B54A32D192ED03ull) ^ (purpose << 56)};
    r.next();
    r.next();
    return r;
}

// GenRandom (kgraph.cpp:44-65) by one thread, in place in global memory.
__device__ void gen_random_dev(Rng &rng, uint32_t *addr, uint32_t size, uint32_t N) {
    if (N == size) {
        for (uint32_t i = 0; i < size; ++i) addr[i] = i;
        return;
    }
    for (uint32_t i = 0; i < size; ++i) addr[i] = rng.next() % (N - size);
    for (uint32_t i = 1; i < size; ++i) {   // insertion sort (size is 2S or S+1)
        uint32_t v = addr[i];
        uint32_t j = i;
        while (j > 0 && addr[j - 1] > v) { addr[j] = addr[j - 1]; --j; }
        addr[j] = v;
    }
    for (uint32_t i = 1; i < size; ++i)
        if (addr[i] <= addr[i - 1]) addr[i] = addr[i - 1] + 1;
    uint32_t off = rng.next() % N;
    for (uint32_t i = 0; i < size; ++i) addr[i] = (addr[i] + off) % N;
}

struct GPoolAcc {   // gnu_sort over one pool row (dist, id) in global memory
    float *d; uint32_t *i;
    struct Rec { float d; uint32_t i; };
    __device__ float key(int x) const { return d[x]; }
    __device__ void swap(int x, int y) const {
        float td = d[x]; d[x] = d[y]; d[y] = td;
        uint32_t ti = i[x]; i[x] = i[y]; i[y] = ti;
    }
    __device__ Rec get(int x) const { return Rec{d[x], i[x]}; }
    __device__ void put(int x, Rec r) const { d[x] = r.d; i[x] = r.i; }
    __device__ float rkey(Rec r) const { return r.d; }
};

__device__ __forceinline__ uint32_t warp_id_global() { return (blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ uint32_t warps_total() { return (gridDim.x * blockDim.x) >> 5; }

// Pinned host memory released on scope exit.
struct HostPinned {
    char *p = nullptr;
    cudaError_t alloc(size_t b) { return cudaMallocHost(reinterpret_cast<void **>(&p), b); }
    ~HostPinned() { if (p) cudaFreeHost(p); }
};

// A stream capture, instantiated once and replayed; released on scope exit.
struct StreamGraph {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
    StreamGraph() = default;
    StreamGraph(const StreamGraph &) = delete;
    StreamGraph &operator=(const StreamGraph &) = delete;
    ~StreamGraph() {
        if (x) cudaGraphExecDestroy(x);
        if (g) cudaGraphDestroy(g);
    }
    bool ready() const { return x != nullptr; }
    template <class F> cudaError_t capture(cudaStream_t st, F &&record) {
        cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess) return e;
        const cudaError_t er = record();
        const cudaError_t ee = cudaStreamEndCapture(st, &g);
        if (er != cudaSuccess) return er;
        if (ee != cudaSuccess) return ee;
        return cudaGraphInstantiate(&x, g, 0);
    }
    cudaError_t launch(cudaStream_t st) const { return cudaGraphLaunch(x, st); }
};

// ------------------------------------------------------------------ init
// kgraph.cpp:760-796 for one node per warp.
__global__ void __launch_bounds__(256) init_kernel(BuildState s) {
    const int lane = threadIdx.x & 31;
    const uint32_t N = s.D.n;
    for (uint32_t n = warp_id_global(); n < N; n += warps_total()) {
        uint32_t *pi = s.pool_i + (size_t)n * s.PS;
        float *pd = s.pool_d + (size_t)n * s.PS;
        if (lane == 0) {
            Rng rng = make_rng(s.seed, n, 1);
            gen_random_dev(rng, s.nn_new + (size_t)n * s.NEWCAP, 2 * s.S, N);
            gen_random_dev(rng, pi, s.S + 1, N);        // `random`, consumed in place below
            uint32_t i = 0;
            for (uint32_t l = 0; l < s.S; ++l) {
                if (pi[i] == n) ++i;
                pi[l] = pi[i++];
            }
        }
        __syncwarp();
        const int g = lane >> 2, t = lane & 3;
        for (uint32_t base = 0; base < s.S; base += 8) {
            uint32_t l = base + g;
            uint32_t id = l < s.S ? pi[l] : n;
            float dd = pair_dist(s.D, id, n, t, FULL);
            __syncwarp();
            if (l < s.S && t == 0) { pd[l] = dd; pi[l] = id | FLAG_BIT; }
        }
        for (uint32_t l = s.S + lane; l < s.PS; l += 32) { pd[l] = FLT_MAX; pi[l] = UNSET_ID; }
        __syncwarp();
        if (lane == 0) {
            GPoolAcc acc{pd, pi};
            gnu_sort(acc, 0, (int)s.S);   // kgraph.cpp:793
            s.nodeL[n] = s.S;
            s.nodeM[n] = s.S;
            s.radius[n] = FLT_MAX;
            s.cnt_new[n] = 2 * s.S;
            s.cnt_old[n] = 0;
            s.found[n] = 0;
            s.lock[n] = 0;
        }
        __syncwarp();
    }
}

// Two pair distances sharing row j (4-lane group): dist(i0, j) and dist(i1, j)
// with the bits of pair_dist (the canonical distance is symmetric bit for bit:
// products, squares of differences and the norm sum all commute), row j read
// once for both.
__device__ __forceinline__ void pair_dist_shared(const DataView &D, uint32_t j, uint32_t i0, uint32_t i1, int t,
                                                 unsigned mask, float &d0, float &d1) {
    const float *rj = D.X + (size_t)j * D.ld, *r0 = D.X + (size_t)i0 * D.ld, *r1 = D.X + (size_t)i1 * D.ld;
    float4 a0 = make_float4(0.f, 0.f, 0.f, 0.f), a1 = make_float4(0.f, 0.f, 0.f, 0.f);
    const int chunks = (int)D.d >> 4;
    for (int c = 0; c < chunks; ++c) {
        const float4 y = ld4(rj + 16 * c + 4 * t);
        lane_acc(a0, ld4(r0 + 16 * c + 4 * t), y, D.metric);
        lane_acc(a1, ld4(r1 + 16 * c + 4 * t), y, D.metric);
    }
    float s0 = group4_reduce(a0, mask), s1 = group4_reduce(a1, mask);
    int i = chunks << 4;
    const int d = (int)D.d;
    if (d - i >= 8) {   // the tail exactly as group4_raw
        for (int e = i + 8; i < e; ++i) {
            float x0 = r0[i], x1 = r1[i], y0 = rj[i], y1 = rj[i];
            if (D.metric == METRIC_L2SQR) { x0 = __fsub_rn(x0, y0); y0 = x0; x1 = __fsub_rn(x1, y1); y1 = x1; }
            s0 = __fadd_rn(s0, __fmul_rn(x0, y0));
            s1 = __fadd_rn(s1, __fmul_rn(x1, y1));
        }
    }
    for (; i < d; ++i) {
        float x0 = r0[i], x1 = r1[i], y0 = rj[i], y1 = rj[i];
        if (D.metric == METRIC_L2SQR) { x0 = __fsub_rn(x0, y0); y0 = x0; x1 = __fsub_rn(x1, y1); y1 = x1; }
        s0 = __fmaf_rn(x0, y0, s0);
        s1 = __fmaf_rn(x1, y1, s1);
    }
    if (D.metric == METRIC_L2SQR) { d0 = s0; d1 = s1; return; }
    d0 = finish_metric(s0, D.norms[i0], D.norms[j], D.metric);
    d1 = finish_metric(s1, D.norms[i1], D.norms[j], D.metric);
}

// ------------------------------------------------------------------ join
// KGraphConstructor::join + Nhood::join (kgraph.cpp:740-751, 797-815).  The
// node's new entries are taken two at a time: the second one's partners are
// the first one's minus the second itself, so each partner row read serves
// both pairs.
__global__ void __launch_bounds__(256) join_kernel(BuildState s) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const uint32_t N = s.D.n;
    unsigned long long comps = 0;
    InsertTally tally;
    for (;;) {
        uint32_t n = 0;
        if (lane == 0) n = s.node_lo + atomicAdd(s.work, 1u);
        n = __shfl_sync(FULL, n, 0);
        if (n >= s.node_hi) break;
        const uint32_t a = s.cnt_new[n], b = s.cnt_old[n];
        const uint32_t *nw = s.nn_new + (size_t)n * s.NEWCAP;
        const uint32_t *od = s.nn_old + (size_t)n * s.OLDCAP;
        bool uu = false;
        auto settle = [&](bool valid, uint32_t x, uint32_t y, float dd) {
            settle_pass(s, lane, t, valid, x, y, dd, n, comps, uu, tally);
        };
        for (uint32_t ii = 0; ii < a; ii += 2) {
            const bool two = ii + 1 < a;
            uint32_t i0 = nw[ii], i1 = two ? nw[ii + 1] : 0u;
            const bool bad0 = i0 >= N, bad1 = two && i1 >= N;
            if (bad0 || bad1) {
                if (lane == 0) raise_error(s.err, ERR_BAD_ID);
                if (bad0) i0 = 0;
                if (bad1) i1 = 0;
            }
            const uint32_t nnn = a - ii - 1, inner = nnn + b;   // i0's partners: new[ii+1..a) then old
            for (uint32_t base = 0; base < inner; base += 8) {
                const uint32_t k = base + g;
                const bool in = k < inner;
                const bool is_nn = k < nnn;
                uint32_t jid = in ? (is_nn ? nw[ii + 1 + k] : od[k - nnn]) : 0u;
                const bool badj = in && jid >= N;
                if (badj) { raise_error(s.err, ERR_BAD_ID); jid = 0; }
                // i < j by id excludes equal ids; i1's partners start after itself (k >= 1)
                const bool v0 = in && !badj && !bad0 && !(is_nn && jid == i0);
                const bool v1 = two && in && k >= 1 && !badj && !bad1 && !(is_nn && jid == i1);
                float d0, d1;
                pair_dist_shared(s.D, jid, i0, i1, t, FULL, d0, d1);
                settle(v0, v0 ? (is_nn ? min(i0, jid) : i0) : 0u, v0 ? (is_nn ? max(i0, jid) : jid) : 0u, d0);
                if (two)
                    settle(v1, v1 ? (is_nn ? min(i1, jid) : i1) : 0u, v1 ? (is_nn ? max(i1, jid) : jid) : 0u, d1);
            }
        }
        if (lane == 0) s.found[n] = uu ? 1u : 0u;
    }
    if (lane == 0 && comps) atomicAdd(s.n_comps, comps);
    if (lane == 0 && tally.attempts) {
        atomicAdd(s.inserts, tally.attempts);
        atomicAdd(s.inserts + 1, tally.landed);
    }
}

// The same join with a node's lists staged in shared memory: one CTA per node
// copies the rows of new ++ old (jt_rows of them; rows beyond are read from
// global memory) and their norm terms once, then evaluates the node's pairs
// from there -- each 4-lane group one pair per pass with the canonical
// arithmetic (group4_raw, the same bits as pair_dist) -- so a node's partner
// rows cross from L2/DRAM once per node instead of once per pair.  Pairs: for
// new entry i (warp-strided), new[i+1 ..) then old, as join_kernel.
constexpr int JT_WARPS = 4;
// Shared memory per CTA; rows past it are read from L2.  24 KB lets 8 CTAs
// share an SM: at 1M x 128 the join runs 0.73 s a build against 0.89 s with
// 48 KB (4 CTAs), the occupancy hiding the L2 reads of the rows left out.
// Rows too wide for 8 of them in 24 KB take the 48 KB budget.
#ifndef JT_SMEM_BUDGET
#define JT_SMEM_BUDGET (24 * 1024)
#endif
constexpr size_t JT_SMEM_WIDE = 48 * 1024;
constexpr uint32_t JT_BUF = 64;   // offers a warp collects before it appends them to the record buffer
// Shared memory of join_tile_kernel besides the rows: per list entry its id,
// norm term and radius, per warp the offer buffer.
__host__ __device__ constexpr size_t jt_fixed_bytes(uint32_t list_cap) {
    return (size_t)list_cap * 12 + (size_t)JT_WARPS * JT_BUF * 16;
}

// Deferred mode: the offers a warp collected (all of the CTA's current node)
// go to the record buffer with one cursor atomic; those beyond its capacity
// are inserted under the lock here (their uu counts for the current node).
__device__ __forceinline__ void jt_flush(const BuildState &s, uint4 *buf, uint32_t &cnt, int lane, bool &uu,
                                         InsertTally &tally) {
    if (!cnt) return;
    unsigned long long b0 = 0;
    if (lane == 0) b0 = atomicAdd(s.off_cursor, (unsigned long long)cnt);
    b0 = __shfl_sync(FULL, b0, 0);
    const uint32_t fit = b0 >= s.off_cap ? 0u : (uint32_t)min((unsigned long long)cnt, s.off_cap - b0);
    for (uint32_t k = lane; k < fit; k += 32) {
        const uint4 o = buf[k];
        s.off_lin[b0 + k] = o;
        atomicAdd(s.off_cnt + o.x, 1u);
    }
    for (uint32_t k = fit; k < cnt; ++k) {
        const uint4 o = buf[k];
        const uint32_t r = locked_insert(s, o.x, o.y, __uint_as_float(o.z), lane, tally);
        if ((o.w & OFFER_UU) && r < s.K) uu = true;
    }
    cnt = 0;
    __syncwarp();
}

__global__ void __launch_bounds__(JT_WARPS * 32) join_tile_kernel(BuildState s) {
    extern __shared__ __align__(16) float jt_smem[];
    __shared__ uint32_t s_node, s_uu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const uint32_t N = s.D.n, stride = s.D.ld + 4;   // 16 bytes of padding: rows start on different banks
    const int metric = s.D.metric;
    const uint32_t cap = s.NEWCAP + s.OLDCAP;
    uint4 *bufs = reinterpret_cast<uint4 *>(jt_smem);   // 16-byte aligned at the start
    uint4 *buf = bufs + (size_t)warp * JT_BUF;
    float *rows = reinterpret_cast<float *>(bufs + (size_t)JT_WARPS * JT_BUF);
    float *nrm = rows + (size_t)s.jt_rows * stride;
    float *rad = nrm + cap;
    uint32_t *uid = reinterpret_cast<uint32_t *>(rad + cap);
    const bool deferred = s.off_lin != nullptr;
    unsigned long long comps = 0;
    InsertTally tally;
    uint32_t bcnt = 0;
    for (;;) {
        if (threadIdx.x == 0) { s_node = s.node_lo + atomicAdd(s.work, 1u); s_uu = 0; }
        __syncthreads();
        const uint32_t n = s_node;
        if (n >= s.node_hi) break;
        const uint32_t a = min(s.cnt_new[n], s.NEWCAP), b = min(s.cnt_old[n], s.OLDCAP);
        if (a == 0) {
            if (threadIdx.x == 0) s.found[n] = 0u;
            __syncthreads();
            continue;
        }
        const uint32_t U = a + b;
        const uint32_t *nw = s.nn_new + (size_t)n * s.NEWCAP, *od = s.nn_old + (size_t)n * s.OLDCAP;
        for (uint32_t u = threadIdx.x; u < U; u += blockDim.x) {
            uint32_t id = u < a ? nw[u] : od[u - a];
            if (id >= N) { raise_error(s.err, ERR_BAD_ID); id = NO_ID; }
            uid[u] = id;
            nrm[u] = (id != NO_ID && metric != METRIC_L2SQR) ? s.D.norms[id] : 0.f;
            // deferred: the radii as the join starts (they change only in the merge after it; a
            // larger radius lets more offers through to the merge's exact test)
            rad[u] = id != NO_ID ? *reinterpret_cast<volatile float *>(s.radius + id) : 0.f;
        }
        __syncthreads();
        const uint32_t staged = min(U, s.jt_rows);
        for (uint32_t r = warp; r < staged; r += JT_WARPS) {
            const uint32_t id = uid[r] == NO_ID ? 0u : uid[r];
            const float *src = s.D.X + (size_t)id * s.D.ld;
            float *dst = rows + (size_t)r * stride;
            for (uint32_t k = 4 * lane; k < s.D.ld; k += 128) *reinterpret_cast<float4 *>(dst + k) = ld4(src + k);
        }
        __syncthreads();
        bool uu = false;
        for (uint32_t i = warp; i < a; i += JT_WARPS) {
            const uint32_t idi = uid[i];
            const float *ri = i < s.jt_rows ? rows + (size_t)i * stride : s.D.X + (size_t)(idi == NO_ID ? 0u : idi) * s.D.ld;
            const float ni = nrm[i], radi = rad[i];
            const uint32_t nnn = a - 1 - i, inner = nnn + b;   // partners: new[i+1..a) then old
            for (uint32_t base = 0; base < inner; base += 8) {
                const uint32_t k = base + g;
                const bool in = k < inner;
                const uint32_t u = in ? (k < nnn ? i + 1 + k : a + (k - nnn)) : i;
                const bool is_nn = u < a;
                const uint32_t jid = uid[u];
                // i < j by id excludes equal ids among the new entries (kgraph.cpp:742-743)
                const bool v = in && idi != NO_ID && jid != NO_ID && !(is_nn && jid == idi);
                const float *rj = u < s.jt_rows ? rows + (size_t)u * stride : s.D.X + (size_t)(jid == NO_ID ? 0u : jid) * s.D.ld;
                const float raw = group4_raw(ri, rj, (int)s.D.d, metric, t, FULL);
                const float dd = metric == METRIC_L2SQR ? raw : finish_metric(raw, ni, nrm[u], metric);
                const bool i_is_x = !is_nn || idi < jid;
                const uint32_t x = v ? (i_is_x ? idi : jid) : 0u, y = v ? (i_is_x ? jid : idi) : 0u;
                if (!deferred) {
                    settle_pass(s, lane, t, v, x, y, dd, n, comps, uu, tally);
                    continue;
                }
                // the unlocked radius test of both directions (kgraph.cpp:725) on the staged radii
                const float rx = i_is_x ? radi : rad[u], ry = i_is_x ? rad[u] : radi;
                comps += __popc(__ballot_sync(FULL, v && t == 0));
                const bool off = v && ((t == 0 && !(dd > rx)) || (t == 1 && !(dd > ry)));
                const unsigned om = __ballot_sync(FULL, off);
                if (!om) continue;
                if (bcnt + __popc(om) > JT_BUF) jt_flush(s, buf, bcnt, lane, uu, tally);
                if (off) {
                    const uint32_t pos = bcnt + __popc(om & ((1u << lane) - 1u));
                    buf[pos] = make_uint4(t == 0 ? x : y, t == 0 ? y : x, __float_as_uint(dd), n | (t == 0 ? OFFER_UU : 0u));
                }
                bcnt += __popc(om);
                __syncwarp();
            }
        }
        if (deferred) jt_flush(s, buf, bcnt, lane, uu, tally);
        if (uu && lane == 0) atomicOr(&s_uu, 1u);
        __syncthreads();
        if (threadIdx.x == 0) s.found[n] = s_uu;
    }
    if (lane == 0 && comps) atomicAdd(s.n_comps, comps);
    if (lane == 0 && tally.attempts) {
        atomicAdd(s.inserts, tally.attempts);
        atomicAdd(s.inserts + 1, tally.landed);
    }
}

// ------------------------------------------------------------------ deferred inserts
// Offers of one join grouped by target: off_grp[off_pos[x] ..) holds x's.
__global__ void offer_scatter_kernel(BuildState s) {
    const unsigned long long total = min(*s.off_cursor, s.off_cap);
    for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        const uint4 o = s.off_lin[i];
        const uint32_t at = atomicAdd(s.off_fill + o.x, 1u);
        s.off_grp[s.off_pos[o.x] + at] = o;
    }
}

// Order-preserving map of a float's bits to an unsigned key, and back.
__device__ __forceinline__ uint32_t f2ord(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float ord2f(uint32_t u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u); }

// Ascending bitonic sort of the 32 E keys at keys[0, 32 E) by one warp, in
// registers: lane l holds elements l E .. l E + E - 1, so partners closer than
// E are in the lane and farther ones are an XOR shuffle away.
template <int E>
__device__ __forceinline__ void warp_sort_keys(unsigned long long *keys, int lane) {
    unsigned long long v[E];
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = keys[lane * E + e];
#pragma unroll
    for (int k = 2; k <= 32 * E; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= E) {
                const int lj = j / E;
                const bool lower = (lane & lj) == 0;
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    const unsigned long long o = __shfl_xor_sync(FULL, v[e], lj);
                    const bool asc = ((lane * E + e) & k) == 0;
                    v[e] = (lower == asc) ? (v[e] < o ? v[e] : o) : (v[e] > o ? v[e] : o);
                }
            } else {
#pragma unroll
                for (int e = 0; e < E; ++e) {
                    if (e & j) continue;
                    const bool asc = ((lane * E + e) & k) == 0;
                    const unsigned long long a = v[e], b = v[e | j];
                    if ((a > b) == asc) { v[e] = b; v[e | j] = a; }
                }
            }
        }
    }
#pragma unroll
    for (int e = 0; e < E; ++e) keys[lane * E + e] = v[e];
    __syncwarp();
}

constexpr uint32_t MG_CH = 512;     // offers merged per pass at most (sorted in shared memory)
constexpr uint32_t MG_PASS = 224;   // offers a value-mode pass aims at
constexpr int MG_WARPS = 8;
size_t merge_warp_bytes(uint32_t PS) { return (size_t)MG_CH * 20 + (size_t)PS * 16; }

// Nhood::parallel_try_insert (kgraph.cpp:723-736) of every deferred offer
// into its pool, one warp per pool, without locks (the join has finished).
// A pool takes its offers in ascending (distance, id) order -- inserts into
// different pools touch disjoint state, so a pool's outcome depends only on
// the order of its own offers, which the reference's threads leave arbitrary
// -- in passes of up to MG_CH, each pass
// in one merge that reproduces the successive UpdateKnnListHelper calls
// (kgraph.cpp:176-202):
//  * an offer equal to an earlier one or to a pool entry (same id, same
//    distance) is a duplicate;
//  * the q-th non-duplicate lands at p = (pool entries <= d) + q, and every
//    non-duplicate with p < L passes the radius test (the list's last entry
//    then lies after it): these are a prefix of the non-duplicates;
//  * the rest reach a full list: the first of them passes only against the
//    stored radius, which an insert sets only when the list was already full
//    (it may still be FLT_MAX), later ones only at a distance equal to the
//    list's last entry; each lands in the overflow slot L, its duplicate test
//    made against the list as it then is;
//  * `found` of the offer's source node is set when an x <- y offer lands
//    below K; L and the radius end as after the serial inserts.
__global__ void __launch_bounds__(MG_WARPS * 32) offer_merge_kernel(BuildState s) {
    extern __shared__ __align__(16) unsigned char mg_smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    unsigned char *wbase = mg_smem + (size_t)wib * s.mg_warp_bytes;
    unsigned long long *keys = reinterpret_cast<unsigned long long *>(wbase);
    uint32_t *paux = reinterpret_cast<uint32_t *>(keys + MG_CH);   // p of a non-duplicate, else ~0
    uint32_t *qaux = paux + MG_CH;                              // its index among the non-duplicates
    float *acc_d = reinterpret_cast<float *>(qaux + MG_CH);     // the accepted offers, in order
    float *pdA = acc_d + MG_CH;
    uint32_t *piA = reinterpret_cast<uint32_t *>(pdA + s.PS);
    float *pdB = reinterpret_cast<float *>(piA + s.PS);
    uint32_t *piB = reinterpret_cast<uint32_t *>(pdB + s.PS);
    const uint32_t N = s.D.n, L = s.L, Lp = s.Lp;
    unsigned long long att = 0, landed = 0;
    for (;;) {
        uint32_t x = 0;
        if (lane == 0) x = atomicAdd(s.mg_work, 1u);
        x = __shfl_sync(FULL, x, 0);
        if (x >= N) break;
        const uint32_t m = s.off_cnt[x];
        if (m == 0) continue;
        const uint64_t o0 = s.off_pos[x];
        float *pd = pdA, *pdn = pdB;
        uint32_t *pi = piA, *pin = piB;
        float *gpd = s.pool_d + (size_t)x * s.PS;
        uint32_t *gpi = s.pool_i + (size_t)x * s.PS;
        for (uint32_t j = lane; j < Lp; j += 32) { pd[j] = gpd[j]; pi[j] = gpi[j]; }
        uint32_t Lc = s.nodeL[x];
        float rad = s.radius[x];
        bool rad_set = false;
        __syncwarp();
        // `found` (kgraph.cpp:808-810): an x <- y insert that lands below K at its
        // time.  Whether an insert lands below K depends on the order the offers
        // arrive in, not only on the final list; the reference's threads deliver
        // them in an arbitrary interleaving, and so does the grouping here (record
        // order within a pool), so the offers are replayed in that order against a
        // copy of the list's first K positions -- the positions below K are all
        // that decide it, an entry pushed past them never comes back, and a
        // duplicate of an entry pushed past them lands at K or later anyway; a
        // duplicate's return value (the list's length + 1) is below K only while
        // the copy holds the whole list.
        {
            const uint32_t Kc = min(s.K, L);
            float *kd = pdn;
            uint32_t *ki = pin;
            uint32_t kc = min(Lc, Kc);
            for (uint32_t j = lane; j < kc; j += 32) { kd[j] = pd[j]; ki[j] = pi[j]; }
            __syncwarp();
            float kth = kc == Kc && Kc ? kd[Kc - 1] : FLT_MAX;
            // 32 offers at a time, in arrival order.  An offer lands below K iff (the
            // copy's entries <= d) + (earlier non-duplicate offers of its chunk with
            // distance <= d) < K: an earlier offer that does not land is no closer
            // than one that does, so counting it never changes the answer.
            for (uint32_t k0 = 0; k0 < m && Kc; k0 += 32) {
                const uint32_t k = k0 + lane;
                uint4 o = make_uint4(0u, 0u, 0u, 0u);
                if (k < m) o = s.off_grp[o0 + k];
                const float d = __uint_as_float(o.z);
                const bool possible = k < m && (kc < Kc || d < kth);
                if (!__any_sync(FULL, possible)) continue;
                uint32_t base = 0;
                bool dupK = false;
                if (possible) {
                    uint32_t lo = 0, hi = kc;   // the copy's entries <= d
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (kd[mid] <= d) lo = mid + 1; else hi = mid;
                    }
                    base = lo;
                    for (int j = (int)base - 1; !dupK && j >= 0 && kd[j] == d; --j) dupK = (ki[j] & ID_MASK) == o.y;
                }
                // the first of identical offers (same distance and id) in the chunk
                const unsigned long long key = possible ? (((unsigned long long)o.z << 32) | o.y) : ~0ull - lane;
                const unsigned same = __match_any_sync(FULL, key);
                const int first = __ffs(same) - 1;
                const bool nd = possible && !dupK && first == lane;
                const unsigned ndm = __ballot_sync(FULL, nd);
                uint32_t cnt = 0;
                for (unsigned rest = ndm; rest; rest &= rest - 1) {   // ndm is warp-uniform
                    const int j = __ffs(rest) - 1;
                    const float dj = __shfl_sync(FULL, d, j);
                    if (j < lane && dj <= d) ++cnt;
                }
                const bool landed = nd && base + cnt < Kc;
                const unsigned lm = __ballot_sync(FULL, landed);
                const bool first_landed = (lm >> first) & 1u;
                if (landed && (o.w & OFFER_UU)) s.found[o.w & ~OFFER_UU] = 1u;
                // a duplicate returns the list's length + 1 (kgraph.cpp:193): below K only while
                // the copy holds the whole list
                const bool dup = possible && (dupK || (first != lane && first_landed));
                if (dup && (o.w & OFFER_UU) && kc + __popc(lm & ((1u << lane) - 1u)) + 1 < s.K)
                    s.found[o.w & ~OFFER_UU] = 1u;
                if (lm) {
                    uint32_t mr;
                    kc = warp_batch_insert(kd, ki, nullptr, kc, Kc + 1, lm, d, o.y | FLAG_BIT, 0u, &mr, lane);
                    __syncwarp();
                    kth = kc == Kc ? kd[Kc - 1] : FLT_MAX;
                }
            }
            __syncwarp();
        }
        // The offers go in passes.  Value mode: each pass takes the offers whose
        // distance key lies in (lo, hi], hi cut from a 32-offer sample so that
        // about MG_PASS fall in; passes follow in ascending order, so the pass
        // that meets the first radius rejection ends the pool (every later
        // offer is farther).  A range that no sample cut keeps within MG_CH
        // (massive ties) switches the rest of the pool to scan mode: chunks of
        // up to MG_CH in record order, each merged as it comes.
        uint32_t lo_key = 0, rem = m, cursor = 0;
        bool have_lo = false, scan_mode = false, stop = false;
        while (rem && !stop) {
            uint32_t cm = 0;
            if (!scan_mode) {
                uint32_t hi_key = 0xFFFFFFFFu;
                int idx = -1;
                uint32_t sk = 0xFFFFFFFFu;
                if (rem > MG_PASS) {
                    const uint32_t si = (uint32_t)(((uint64_t)lane * m) >> 5);
                    const uint32_t so = f2ord(__uint_as_float(s.off_grp[o0 + si].z));
                    const bool valid = !have_lo || so > lo_key;
                    sk = valid ? so : 0xFFFFFFFFu;
                    for (int kk = 2; kk <= 32; kk <<= 1)   // sort the sample (bitonic across lanes)
                        for (int jj = kk >> 1; jj > 0; jj >>= 1) {
                            const uint32_t other = __shfl_xor_sync(FULL, sk, jj);
                            const bool keep_min = ((lane & jj) == 0) == ((lane & kk) == 0);
                            sk = keep_min ? min(sk, other) : max(sk, other);
                        }
                    const uint32_t nv = __popc(__ballot_sync(FULL, valid));
                    if (nv == 0) scan_mode = true;
                    else idx = (int)min(nv - 1, (uint32_t)(((uint64_t)MG_PASS * nv) / rem));
                }
                while (!scan_mode) {
                    if (idx >= 0) hi_key = __shfl_sync(FULL, sk, idx);
                    cm = 0;
                    for (uint32_t k0 = 0; k0 < m; k0 += 32) {
                        const uint32_t k = k0 + lane;
                        bool in = false;
                        uint4 o = make_uint4(0u, 0u, 0u, 0u);
                        uint32_t ko = 0;
                        if (k < m) {
                            o = s.off_grp[o0 + k];
                            ko = f2ord(__uint_as_float(o.z));
                            in = (!have_lo || ko > lo_key) && ko <= hi_key;
                        }
                        const unsigned bal = __ballot_sync(FULL, in);
                        const uint32_t pos = cm + __popc(bal & ((1u << lane) - 1u));
                        if (in && pos < MG_CH) keys[pos] = ((unsigned long long)ko << 32) | o.y;
                        cm += __popc(bal);
                    }
                    if (cm <= MG_CH) {
                        lo_key = hi_key;
                        have_lo = true;
                        break;
                    }
                    if (idx <= 0) scan_mode = true;   // ties: no cut fits one pass
                    else idx /= 2;
                }
                __syncwarp();
            }
            if (scan_mode) {   // the next chunk of the remaining offers in record order
                cm = 0;
                while (cursor < m && cm < MG_CH) {
                    const uint32_t k = cursor + lane;
                    bool in = false;
                    uint4 o = make_uint4(0u, 0u, 0u, 0u);
                    uint32_t ko = 0;
                    if (k < m) {
                        o = s.off_grp[o0 + k];
                        ko = f2ord(__uint_as_float(o.z));
                        in = !have_lo || ko > lo_key;
                    }
                    const unsigned bal = __ballot_sync(FULL, in);
                    const uint32_t take = min((uint32_t)__popc(bal), MG_CH - cm);
                    const uint32_t rank = __popc(bal & ((1u << lane) - 1u));
                    if (in && rank < take) keys[cm + rank] = ((unsigned long long)ko << 32) | o.y;
                    cursor += (take < (uint32_t)__popc(bal)) ? (uint32_t)(__fns(bal, 0, take + 1)) : 32u;
                    cm += take;
                }
                __syncwarp();
            }
            if (cm == 0) break;   // nothing left (the counts agree; this only guards the loop)
            rem -= cm;
            uint32_t P2 = 32;
            while (P2 < cm) P2 <<= 1;
            for (uint32_t k = cm + lane; k < P2; k += 32) keys[k] = ~0ull;
            __syncwarp();
            switch (P2) {   // ascending (distance, id)
                case 32: warp_sort_keys<1>(keys, lane); break;
                case 64: warp_sort_keys<2>(keys, lane); break;
                case 128: warp_sort_keys<4>(keys, lane); break;
                case 256: warp_sort_keys<8>(keys, lane); break;
                default: warp_sort_keys<16>(keys, lane); break;
            }
            // positions of the non-duplicates
            uint32_t nnd = 0;
            for (uint32_t k0 = 0; k0 < cm; k0 += 32) {
                const uint32_t k = k0 + lane;
                bool nd = false;
                uint32_t rk = 0;
                if (k < cm) {
                    const unsigned long long key = keys[k];
                    const float d = ord2f((uint32_t)(key >> 32));
                    const uint32_t c = (uint32_t)key;
                    bool dup = k > 0 && keys[k - 1] == key;
                    uint32_t lo = 0, hi = Lc;   // pool entries <= d
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi) >> 1;
                        if (pd[mid] <= d) lo = mid + 1; else hi = mid;
                    }
                    rk = lo;
                    for (int j = (int)rk - 1; !dup && j >= 0 && pd[j] == d; --j) dup = (pi[j] & ID_MASK) == c;
                    nd = !dup;
                }
                const unsigned ndm = __ballot_sync(FULL, nd);
                const uint32_t q = nnd + __popc(ndm & ((1u << lane) - 1u));
                if (k < cm) {
                    paux[k] = nd ? rk + q : 0xFFFFFFFFu;
                    qaux[k] = q;
                }
                nnd += __popc(ndm);
            }
            __syncwarp();
            // the main inserts (p < L), in order; `found` of their sources
            uint32_t qs = 0;
            for (uint32_t k = lane; k < cm; k += 32) {
                const uint32_t p = paux[k];
                if (p < L) {
                    ++qs;
                    acc_d[qaux[k]] = ord2f((uint32_t)(keys[k] >> 32));
                }
            }
            for (int o = 16; o; o >>= 1) qs += __shfl_xor_sync(FULL, qs, o);
            for (uint32_t j = lane; j < Lp; j += 32) { pdn[j] = pd[j]; pin[j] = pi[j]; }
            __syncwarp();
            for (uint32_t j = lane; j < Lc; j += 32) {   // pool entries move up past the accepted offers below them
                const float dj = pd[j];
                uint32_t lo = 0, hi = qs;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (acc_d[mid] < dj) lo = mid + 1; else hi = mid;
                }
                const uint32_t np = j + lo;
                if (np < Lp) { pdn[np] = dj; pin[np] = pi[j]; }
            }
            __syncwarp();
            for (uint32_t k = lane; k < cm; k += 32) {
                const uint32_t p = paux[k];
                if (p < L) { pdn[p] = ord2f((uint32_t)(keys[k] >> 32)); pin[p] = (uint32_t)keys[k] | FLAG_BIT; }
            }
            __syncwarp();
            const bool full_main = qs + Lc > L;   // an insert reached a full list
            uint32_t ntail = 0;
            bool rejected = false;
            if (Lc + qs >= L && lane == 0) {
                // the offers beyond the list, in order (lane 0; a short run: at most one offer
                // above the list's last distance can land)
                const float dL = pdn[L - 1];
                float rc = full_main ? dL : rad;
                // first offer at or above dL that is not a main insert
                uint32_t lo = 0, hi = cm;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (ord2f((uint32_t)(keys[mid] >> 32)) < dL) lo = mid + 1; else hi = mid;
                }
                for (uint32_t k = lo; k < cm; ++k) {
                    if (paux[k] < L) continue;
                    const float d = ord2f((uint32_t)(keys[k] >> 32));
                    if (d > rc) { rejected = true; break; }
                    const uint32_t c = (uint32_t)keys[k];
                    bool dup = false;
                    for (int j = (int)L - 1; !dup && j >= 0 && pdn[j] == d; --j) dup = (pin[j] & ID_MASK) == c;
                    if (dup) continue;
                    pdn[L] = d;
                    pin[L] = c | FLAG_BIT;
                    rc = dL;
                    ++ntail;
                }
            }
            ntail = __shfl_sync(FULL, ntail, 0);
            // a radius rejection in value mode: the offers still to come are all farther
            stop = !scan_mode && __shfl_sync(FULL, rejected, 0);
            __syncwarp();
            // counts: offers that passed the radius test (duplicates included), and those that landed
            att += (cm - nnd) + qs + ntail;
            landed += qs + ntail;
            if (full_main || ntail) { rad = pdn[L - 1]; rad_set = true; }
            Lc = min(L, Lc + qs);
            float *tf = pd; pd = pdn; pdn = tf;
            uint32_t *ti = pi; pi = pin; pin = ti;
            __syncwarp();
        }
        for (uint32_t j = lane; j < Lp; j += 32) { gpd[j] = pd[j]; gpi[j] = pi[j]; }
        if (lane == 0) {
            s.nodeL[x] = Lc;
            if (rad_set) s.radius[x] = rad;
        }
        __syncwarp();
    }
    if (lane == 0 && att) {   // warp-uniform counts
        atomicAdd(s.inserts, att);
        atomicAdd(s.inserts + 1, landed);
    }
}

// ------------------------------------------------------------------ statistics
// Flags in pool[0..K) (EvaluateDelta, kgraph.cpp:148-156), the sum of M,
// the number of full pools, and the join's list entries (|new| + |old|, the
// rows the join read; accumulated over the build for its byte count).
__global__ void stats_kernel(BuildState s) {
    unsigned long long fl = 0, msum = 0, full = 0, lists = 0;
    const uint32_t lim = min(s.K, s.Lp);
    for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < s.D.n; n += gridDim.x * blockDim.x) {
        const uint32_t *pi = s.pool_i + (size_t)n * s.PS;
        for (uint32_t l = 0; l < lim; ++l) fl += (pi[l] & FLAG_BIT) ? 1 : 0;
        msum += s.nodeM[n];
        full += s.nodeL[n] + 1 >= s.Lp ? 1 : 0;   // pool full: a finite radius
        lists += s.cnt_new[n] + s.cnt_old[n];
    }
    for (int o = 16; o; o >>= 1) {
        fl += __shfl_xor_sync(FULL, fl, o);
        msum += __shfl_xor_sync(FULL, msum, o);
        full += __shfl_xor_sync(FULL, full, o);
        lists += __shfl_xor_sync(FULL, lists, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(s.stat + 0, fl);
        atomicAdd(s.stat + 1, msum);
        atomicAdd(s.stat + 2, full);
        atomicAdd(s.list_entries, lists);
    }
}

// Control nodes: EvaluateRecall / EvaluateAccuracy / EvaluateOneRecall
// (kgraph.cpp:96-146) against their exact K-NN.  out[c*5 + ...] = recall,
// accuracy, one-recall, pool[0].dist, exact[0].dist; recall < 0 marks the
// reference's "distance is unstable" failure.
__global__ void controls_kernel(BuildState s, const uint32_t *ctrl, const float *exact_d, uint32_t C, float *out) {
    uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    const uint32_t node = ctrl[c];
    const float *pd = s.pool_d + (size_t)node * s.PS;
    const float *kd = exact_d + (size_t)c * s.K;
    const uint32_t P = s.Lp, K = s.K;
    float recall;
    if (K == 0) recall = 1.0f;
    else {
        uint32_t found = 0, np = 0, nk = 0;
        bool bad = false;
        while (np < P && nk < K) {
            if (kd[nk] < pd[np]) ++nk;
            else if (kd[nk] == pd[np]) { ++found; ++nk; ++np; }
            else { bad = true; break; }
        }
        recall = bad ? -1.0f : __fdiv_rn((float)found, (float)K);
    }
    uint32_t m = min(P, K), cnt = 0;
    float sum = 0.f;
    for (uint32_t i = 0; i < m; ++i)
        if (kd[i] > 0) { sum = __fadd_rn(sum, __fdiv_rn(fabsf(__fsub_rn(pd[i], kd[i])), kd[i])); ++cnt; }
    out[c * 5 + 0] = recall;
    out[c * 5 + 1] = cnt > 0 ? __fdiv_rn(sum, (float)cnt) : 0.f;
    out[c * 5 + 2] = (K > 0 && pd[0] == kd[0]) ? 1.f : 0.f;
    out[c * 5 + 3] = pd[0];
    out[c * 5 + 4] = K > 0 ? kd[0] : 0.f;
}

// ------------------------------------------------------------------ update
// kgraph.cpp:818-841: radius, M growth, radiusM; clears the per-node lists.
__global__ void update_m_kernel(BuildState s) {
    for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < s.D.n; n += gridDim.x * blockDim.x) {
        const float *pd = s.pool_d + (size_t)n * s.PS;
        const uint32_t *pi = s.pool_i + (size_t)n * s.PS;
        s.radius[n] = pd[s.L];   // pool.back()
        uint32_t M = s.nodeM[n];
        if (s.found[n]) {
            uint32_t maxl = min(M + s.S, s.nodeL[n]);
            uint32_t c = 0, l = 0;
            while (l < maxl && c < s.S) {
                if (pi[l] & FLAG_BIT) ++c;
                ++l;
            }
            M = l;
            s.nodeM[n] = M;
        }
        if (M == 0) { raise_error(s.err, ERR_CAPACITY); M = 1; }
        s.radiusM[n] = pd[M - 1];
        s.rcnt_new[n] = 0;
        s.rcnt_old[n] = 0;
    }
}

// Counts the reverse samples each node will receive (kgraph.cpp:852, 860).
__global__ void update_count_kernel(BuildState s) {
    const int lane = threadIdx.x & 31;
    for (uint32_t n = warp_id_global(); n < s.D.n; n += warps_total()) {
        const float *pd = s.pool_d + (size_t)n * s.PS;
        const uint32_t *pi = s.pool_i + (size_t)n * s.PS;
        const uint32_t M = s.nodeM[n];
        for (uint32_t l = lane; l < M; l += 32) {
            uint32_t e = pi[l], id = e & ID_MASK;
            if (id >= s.D.n) { raise_error(s.err, ERR_BAD_ID); continue; }
            if (pd[l] > s.radiusM[id]) atomicAdd((e & FLAG_BIT) ? s.rcnt_new + id : s.rcnt_old + id, 1u);
        }
    }
}

// kgraph.cpp:842-866: forward new/old lists in pool order, flags cleared on
// the new ones, reverse samples appended to their targets' CSR buckets.
__global__ void update_fill_kernel(BuildState s) {
    const int lane = threadIdx.x & 31;
    for (uint32_t n = warp_id_global(); n < s.D.n; n += warps_total()) {
        float *pd = s.pool_d + (size_t)n * s.PS;
        uint32_t *pi = s.pool_i + (size_t)n * s.PS;
        uint32_t *nw = s.nn_new + (size_t)n * s.NEWCAP;
        uint32_t *od = s.nn_old + (size_t)n * s.OLDCAP;
        const uint32_t M = s.nodeM[n];
        uint32_t cn = 0, co = 0;
        for (uint32_t base = 0; base < M; base += 32) {
            const uint32_t l = base + lane;
            const bool act = l < M;
            uint32_t e = act ? pi[l] : 0u, id = e & ID_MASK;
            const bool fl = act && (e & FLAG_BIT);
            const bool ok = act && id < s.D.n;
            unsigned mn = __ballot_sync(FULL, fl), mo = __ballot_sync(FULL, act && !fl);
            unsigned below = (1u << lane) - 1u;
            if (fl) { nw[cn + __popc(mn & below)] = id; pi[l] = id; }
            if (act && !fl) od[co + __popc(mo & below)] = id;
            if (ok && pd[l] > s.radiusM[id]) {
                if (fl) {
                    uint32_t p = atomicAdd(s.rcnt_new + id, 1u);
                    s.rbuf_new[s.roff_new[id] + p] = n;
                } else {
                    uint32_t p = atomicAdd(s.rcnt_old + id, 1u);
                    s.rbuf_old[s.roff_old[id] + p] = n;
                }
            }
            cn += __popc(mn);
            co += __popc(mo);
        }
        if (lane == 0) { s.cnt_new[n] = cn; s.cnt_old[n] = co; }
    }
}

// kgraph.cpp:867-882: at most R reverse samples, a uniform random subset, appended.
__global__ void update_cap_kernel(BuildState s) {
    const int lane = threadIdx.x & 31;
    for (uint32_t n = warp_id_global(); n < s.D.n; n += warps_total()) {
        for (int kind = 0; kind < 2; ++kind) {
            uint32_t *src = kind == 0 ? s.rbuf_new + s.roff_new[n] : s.rbuf_old + s.roff_old[n];
            const uint32_t c = (uint32_t)((kind == 0 ? s.roff_new[n + 1] : s.roff_old[n + 1]) -
                                          (kind == 0 ? s.roff_new[n] : s.roff_old[n]));
            uint32_t take = c;
            if (s.R && c > s.R) {
                take = s.R;
                if (lane == 0) {   // partial Fisher-Yates: the first R of a uniform shuffle
                    Rng rng = make_rng(s.seed, n, 16 + 2 * (uint64_t)*s.iter + kind);
                    for (uint32_t i = 0; i < take; ++i) {
                        uint32_t j = i + rng.next() % (c - i);
                        uint32_t tmp = src[i]; src[i] = src[j]; src[j] = tmp;
                    }
                }
                __syncwarp();
            }
            uint32_t *dst = kind == 0 ? s.nn_new + (size_t)n * s.NEWCAP : s.nn_old + (size_t)n * s.OLDCAP;
            uint32_t *cnt = kind == 0 ? s.cnt_new + n : s.cnt_old + n;
            const uint32_t cap = kind == 0 ? s.NEWCAP : s.OLDCAP;
            const uint32_t have = *cnt;
            if (have + take > cap) {
                if (lane == 0) raise_error(s.err, ERR_CAPACITY);
                take = cap > have ? cap - have : 0;
            }
            for (uint32_t i = lane; i < take; i += 32) dst[have + i] = src[i];
            __syncwarp();
            if (lane == 0) *cnt = have + take;
        }
    }
}

// Ends an update: the next iteration's number (the R-subset streams are keyed by it).
__global__ void iter_advance_kernel(BuildState s) {
    if (threadIdx.x == 0 && blockIdx.x == 0) ++*s.iter;
}

// ------------------------------------------------------------------ finalize
__global__ void finalize_count_kernel(BuildState s, uint64_t *cnt) {
    for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n < s.D.n; n += gridDim.x * blockDim.x)
        cnt[n] = min(s.L, s.nodeL[n]);
}
__global__ void finalize_fill_kernel(BuildState s, const uint64_t *off, uint32_t *ids, float *dists, uint32_t *M) {
    const int lane = threadIdx.x & 31;
    for (uint32_t n = warp_id_global(); n < s.D.n; n += warps_total()) {
        const uint64_t o = off[n];
        const uint32_t c = (uint32_t)(off[n + 1] - o);
        for (uint32_t l = lane; l < c; l += 32) {
            ids[o + l] = s.pool_i[(size_t)n * s.PS + l] & ID_MASK;
            dists[o + l] = s.pool_d[(size_t)n * s.PS + l];
        }
        if (lane == 0) M[n] = s.nodeM[n];
    }
}

// ------------------------------------------------------------------ controls' exact K-NN
// LinearSearch (kgraph.cpp:212-229): rows [lo, hi) of the scan for control c
// by one warp, keeping the K best by (distance, id) -- the order the
// reference's in-id-order insert-after-equals produces.
__global__ void __launch_bounds__(256) linear_part_kernel(DataView D, const uint32_t *ctrl, uint32_t C, uint32_t K,
                                                          uint32_t parts, float *part_d, uint32_t *part_i,
                                                          uint32_t *part_n) {
    extern __shared__ __align__(16) char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int g = lane >> 2, t = lane & 3;
    const uint32_t w = warp_id_global();
    if (w >= C * parts) return;   // whole warps exit together
    const uint32_t c = w / parts, part = w % parts;
    const uint32_t self = ctrl[c];
    const uint32_t chunk = (D.n + parts - 1) / parts;
    const uint32_t lo = part * chunk, hi = min(D.n, lo + chunk);
    float *ld = reinterpret_cast<float *>(smem) + (size_t)wib * (2 * (K + 1) + 16);
    uint32_t *li = reinterpret_cast<uint32_t *>(ld + (K + 1));
    float *cd = ld + 2 * (K + 1);
    uint32_t L = 0;
    for (uint32_t base = lo; base < hi; base += 8) {
        uint32_t row = base + g;
        bool v = row < hi && row != self;
        float dd = pair_dist(D, self, v ? row : self, t, FULL);
        if (t == 0) cd[g] = dd;
        __syncwarp();
        unsigned vm = __ballot_sync(FULL, v && t == 0);
        while (vm) {
            int src = __ffs(vm) - 1;
            vm &= vm - 1;
            float x = cd[src >> 2];
            if (L == K && (K == 0 || x >= ld[K - 1])) continue;
            warp_update_knn(ld, li, (uint32_t *)nullptr, L, x, base + (src >> 2), 0u, lane);
            if (L < K) ++L;
        }
        __syncwarp();
    }
    float *od = part_d + (size_t)w * K;
    uint32_t *oi = part_i + (size_t)w * K;
    for (uint32_t k = lane; k < L; k += 32) { od[k] = ld[k]; oi[k] = li[k]; }
    if (lane == 0) part_n[w] = L;
}

// Merges the parts of each control in part order (= id order), keeping K.
__global__ void __launch_bounds__(256) linear_merge_kernel(uint32_t C, uint32_t K, uint32_t parts, const float *part_d,
                                                           const uint32_t *part_i, const uint32_t *part_n, float *out_d,
                                                           uint32_t *out_i) {
    extern __shared__ __align__(16) char smem[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint32_t c = warp_id_global();
    if (c >= C) return;
    float *ld = reinterpret_cast<float *>(smem) + (size_t)wib * 2 * (K + 1);
    uint32_t *li = reinterpret_cast<uint32_t *>(ld + (K + 1));
    uint32_t L = 0;
    for (uint32_t p = 0; p < parts; ++p) {
        const uint32_t w = c * parts + p;
        for (uint32_t k = 0; k < part_n[w]; ++k) {
            float x = part_d[(size_t)w * K + k];
            if (L == K && (K == 0 || x >= ld[K - 1])) break;   // parts are sorted: the rest cannot enter
            warp_update_knn(ld, li, (uint32_t *)nullptr, L, x, part_i[(size_t)w * K + k], 0u, lane);
            if (L < K) ++L;
        }
    }
    for (uint32_t k = lane; k < K; k += 32) {
        out_d[(size_t)c * K + k] = k < L ? ld[k] : FLT_MAX;
        out_i[(size_t)c * K + k] = k < L ? li[k] : UNSET_ID;
    }
}

int grid_for(kg_ctx *ctx, int per_sm = 8) { return ctx->num_sms * per_sm; }

}  // namespace

// Exact K-NN of control rows (GenerateControl, kgraph.cpp:254-270).
cudaError_t launch_linear_search(kg_ctx *ctx, const uint32_t *rows, uint32_t C, uint32_t K, uint32_t *out_i,
                                 float *out_d) {
    DataView D{ctx->X.as<float>(), ctx->norms.as<float>(), ctx->n, ctx->d, ctx->ld, ctx->metric};
    uint32_t parts = std::max<uint32_t>(1, std::min<uint32_t>(ctx->n / 2048 + 1, (uint32_t)(ctx->num_sms * 64 / std::max(C, 1u))));
    size_t nw = (size_t)C * parts;
    DevBuf &pd = ctx->build_scratch[20], &pi = ctx->build_scratch[21], &pn = ctx->build_scratch[22];
    cudaError_t e;
    if ((e = pd.reserve(nw * K * 4 + 4)) != cudaSuccess || (e = pi.reserve(nw * K * 4 + 4)) != cudaSuccess ||
        (e = pn.reserve(nw * 4 + 4)) != cudaSuccess)
        return e;
    size_t smem1 = 8 * ((2 * (K + 1) + 16) * 4);
    size_t smem2 = 8 * (2 * (K + 1) * 4);
    if (smem1 > 48 * 1024) cudaFuncSetAttribute(linear_part_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1);
    if (smem2 > 48 * 1024) cudaFuncSetAttribute(linear_merge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2);
    linear_part_kernel<<<(unsigned)((nw + 7) / 8), 256, smem1, ctx->stream>>>(D, rows, C, K, parts, pd.as<float>(),
                                                                                 pi.as<uint32_t>(), pn.as<uint32_t>());
    linear_merge_kernel<<<(C + 7) / 8, 256, smem2, ctx->stream>>>(C, K, parts, pd.as<float>(), pi.as<uint32_t>(),
                                                                   pn.as<uint32_t>(), out_d, out_i);
    return cudaGetLastError();
}

// Exclusive scan of n u32/u64 counts into out[n+1] (CUB), with temporary
// storage in `tmp` (the shared scan buffer unless the caller gives its own).
cudaError_t scan_counts(kg_ctx *ctx, const uint32_t *in, uint64_t *out, uint32_t n, DevBuf *tmp = nullptr) {
    if (!tmp) tmp = &ctx->build_scratch[23];
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n + 1, ctx->stream);
    cudaError_t e = tmp->reserve(bytes);
    if (e != cudaSuccess) return e;
    return cub::DeviceScan::ExclusiveSum(tmp->p, bytes, in, out, n + 1, ctx->stream);
}
cudaError_t scan_counts64(kg_ctx *ctx, const uint64_t *in, uint64_t *out, uint32_t n) {
    DevBuf &tmp = ctx->build_scratch[23];
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, n + 1, ctx->stream);
    cudaError_t e = tmp.reserve(bytes);
    if (e != cudaSuccess) return e;
    return cub::DeviceScan::ExclusiveSum(tmp.p, bytes, in, out, n + 1, ctx->stream);
}

}  // namespace kgb

using namespace kgb;

extern "C" void kg_set_verbosity(unsigned v) { kgb::g_verbosity = v; }

// Implemented in kg_graph.cu.
namespace kgb {
int graph_reverse(kg_ctx *ctx, int rev_k);
int graph_prune(kg_ctx *ctx, unsigned level);
}

extern "C" int kg_build(kg_ctx *ctx, const kg_index_params *params, kg_index_info *info) {
    if (!ctx) return KG_E_INVALID;
    std::lock_guard<std::mutex> guard(ctx->mu);
    cudaSetDevice(ctx->device);
    if (!ctx->has_data) return set_error(ctx, KG_E_RUNTIME, "no dataset");
    if (!params) return set_error(ctx, KG_E_INVALID, "bad arguments");
    auto t_start = std::chrono::steady_clock::now();
    const uint32_t N = ctx->n;
    uint32_t L = params->L, K = params->K, S = params->S, C = params->controls;
    // kgraph.cpp:893-905
    if (N <= K) return set_error(ctx, KG_E_RUNTIME, "K larger than dataset size");
    if (N < C) {
        std::cerr << "Warning: small dataset, shrinking control size to " << N << "." << std::endl;
        C = N;
    }
    if (N <= L) {
        std::cerr << "Warning: small dataset, shrinking L to " << (N - 1) << "." << std::endl;
        L = N - 1;
    }
    if (N <= S) {
        std::cerr << "Warning: small dataset, shrinking S to " << (N - 1) << "." << std::endl;
        S = N - 1;
    }
    if (S == 0 || S > L) return set_error(ctx, KG_E_INVALID, "S must be in [1, L]");
    if (params->prune > 2) return set_error(ctx, KG_E_RUNTIME, "prune level not supported.");

    BuildState s{};
    s.D = DataView{ctx->X.as<float>(), ctx->norms.as<float>(), N, ctx->d, ctx->ld, ctx->metric};
    s.L = L; s.Lp = L + 1; s.K = K; s.S = S; s.R = params->R;
    s.node_lo = 0;
    s.node_hi = N;
    s.PS = (s.Lp + 7) / 8 * 8;
    s.NEWCAP = std::max(2 * S, L) + s.R;
    s.OLDCAP = L + s.R;
    s.seed = ((uint64_t)params->seed << 32) ^ 0x5851F42D4C957F2Dull;

    DevBuf *B = ctx->build_scratch;
    const size_t n = N;
    cudaError_t e;
    size_t need[] = {n * s.PS * 4, n * s.PS * 4, n * 4, n * 4, n * 4, n * 4, n * 4, n * 4,
                     n * s.NEWCAP * 4, n * 4, n * s.OLDCAP * 4, n * 4, (n + 1) * 4, (n + 1) * 4,
                     (n + 1) * 8, (n + 1) * 8, n * L * 4 + 4, n * L * 4 + 4, 128};
    for (int i = 0; i < 19; ++i)
        if ((e = B[i].reserve(need[i])) != cudaSuccess) return cuda_fail(ctx, e, "alloc build state");
    s.pool_d = B[0].as<float>(); s.pool_i = B[1].as<uint32_t>();
    s.nodeL = B[2].as<uint32_t>(); s.nodeM = B[3].as<uint32_t>();
    s.radius = B[4].as<float>(); s.radiusM = B[5].as<float>();
    s.found = B[6].as<uint32_t>(); s.lock = B[7].as<uint32_t>();
    s.nn_new = B[8].as<uint32_t>(); s.cnt_new = B[9].as<uint32_t>();
    s.nn_old = B[10].as<uint32_t>(); s.cnt_old = B[11].as<uint32_t>();
    s.rcnt_new = B[12].as<uint32_t>(); s.rcnt_old = B[13].as<uint32_t>();
    s.roff_new = B[14].as<uint64_t>(); s.roff_old = B[15].as<uint64_t>();
    s.rbuf_new = B[16].as<uint32_t>(); s.rbuf_old = B[17].as<uint32_t>();
    s.n_comps = B[18].as<unsigned long long>();
    s.stat = s.n_comps + 1;
    s.work = reinterpret_cast<uint32_t *>(s.n_comps + 4);
    s.iter = s.work + 2;
    // 128-byte counter block: n_comps, stat[3], work + iter, list_entries, inserts[2]
    s.list_entries = s.n_comps + 6;
    s.inserts = s.n_comps + 7;
    s.err = ctx->errw.as<uint32_t>();
    cudaStream_t st = ctx->stream;
    cudaMemsetAsync(B[18].p, 0, 128, st);
    if ((e = ctx->tcstat.reserve(sizeof(JoinTcStats))) != cudaSuccess) return cuda_fail(ctx, e, "alloc build state");
    s.tc = ctx->tcstat.as<JoinTcStats>();
    cudaMemsetAsync(s.tc, 0, sizeof(JoinTcStats), st);
    const bool fp8 = ctx->join_mode == KG_JOIN_FP8 || ctx->join_mode == KG_JOIN_FP8_ALWAYS;
    const bool use_tc = fp8 || ctx->join_mode == KG_JOIN_BF16 || ctx->join_mode == KG_JOIN_BF16_ALWAYS;
    const bool tc_always = ctx->join_mode == KG_JOIN_BF16_ALWAYS || ctx->join_mode == KG_JOIN_FP8_ALWAYS;
    if (use_tc && !join_tc_supported(s, fp8 ? 1 : 0))
        return set_error(ctx, KG_E_INVALID, fp8 ? "tensor-core join (FP8): needs d padded to a multiple of 32 and "
                                                  "lists that fit in shared memory"
                                                : "tensor-core join: lists do not fit in shared memory");
    JoinQueue jq{};
    uint64_t *jworst = nullptr, *jpre = nullptr, qcap = 0;
    if (use_tc) {
        // (x, y, node) entries for one round's pairs; rounds are cut to fit
        qcap = std::max<uint64_t>(64ull << 20, 4 * join_tc_node_max(s));
        if ((e = ctx->joinq.reserve(qcap * 12 + 64)) != cudaSuccess) return cuda_fail(ctx, e, "alloc join queue");
        if ((e = ctx->joinaux.reserve((n + 1) * 16)) != cudaSuccess) return cuda_fail(ctx, e, "alloc join queue");
        jq.x = ctx->joinq.as<uint32_t>();
        jq.y = jq.x + qcap;
        jq.n = jq.y + qcap;
        jq.tail = reinterpret_cast<unsigned long long *>(jq.n + qcap + (qcap & 1));
        jq.work = reinterpret_cast<uint32_t *>(jq.tail + 1);
        jworst = ctx->joinaux.as<uint64_t>();
        jpre = jworst + n + 1;
    }
    cudaMemsetAsync(s.rcnt_new + N, 0, 4, st);   // scan inputs carry one extra zero
    cudaMemsetAsync(s.rcnt_old + N, 0, 4, st);

    // The shared-memory join: rows of new ++ old per node within the CTA's
    // budget, the ids and norm terms beside them.
    size_t jt_smem = 0;
    int jt_blocks = 0;
    s.jt_rows = 0;
    // (with locked inserts the warp-per-node join: four warps of one node contend for the
    // same pools' locks)
    if (ctx->join_tile && ctx->join_inserts != KG_INSERTS_LOCKED) {
        const size_t fixed = jt_fixed_bytes(s.NEWCAP + s.OLDCAP);
        const size_t row_bytes = (size_t)(s.D.ld + 4) * 4;
        size_t budget = (size_t)JT_SMEM_BUDGET - 64;
        if (budget <= fixed + 8 * row_bytes) budget = JT_SMEM_WIDE - 64;
        if (budget > fixed + 8 * row_bytes) {
            s.jt_rows = (uint32_t)std::min<size_t>((budget - fixed) / row_bytes, s.NEWCAP + s.OLDCAP);
            jt_smem = fixed + (size_t)s.jt_rows * row_bytes;
            jt_blocks = (int)std::min<size_t>(8, (228u << 10) / (jt_smem + 1024));   // CTAs per SM it allows
        }
    }
    // Deferred inserts of the FP32 join: the offer records (linear and grouped,
    // 16 bytes each) hold up to 1024 offers per node within 30 % of the free
    // device memory and 20 GB; the per-target counts, cursors and offsets.
    size_t offer_scan_bytes = 0;
    s.mg_warp_bytes = (uint32_t)merge_warp_bytes(s.PS);
    const int mg_warps = (int)std::min<size_t>(MG_WARPS, (227u << 10) / s.mg_warp_bytes);
    if (ctx->join_inserts != KG_INSERTS_LOCKED && mg_warps >= 1) {
        size_t freeb = 0, totalb = 0;
        cudaMemGetInfo(&freeb, &totalb);
        const size_t own = ctx->offer_lin.bytes + ctx->offer_grp.bytes;
        size_t cap = std::min<size_t>((size_t)20 << 30, (freeb + own) / 10 * 3) / 32;
        cap = std::min<size_t>(cap, n * 1024);
        if (ctx->offer_cap) cap = std::min(cap, std::max<size_t>(ctx->offer_cap, 64));
        if (cap >= 1024 || (ctx->offer_cap && cap >= 64)) {
            if ((e = ctx->offer_lin.reserve(cap * 16)) != cudaSuccess || (e = ctx->offer_grp.reserve(cap * 16)) != cudaSuccess ||
                (e = ctx->offer_aux.reserve((n + 1) * 8 + (n + 1) * 4 + n * 4 + 16)) != cudaSuccess)
                return cuda_fail(ctx, e, "alloc join offers");
            s.off_lin = ctx->offer_lin.as<uint4>();
            s.off_grp = ctx->offer_grp.as<uint4>();
            s.off_cap = cap;
            s.off_pos = ctx->offer_aux.as<uint64_t>();
            s.off_cnt = reinterpret_cast<uint32_t *>(s.off_pos + n + 1);
            s.off_fill = s.off_cnt + n + 1;
            s.off_cursor = s.n_comps + 9;                                  // in the counter block
            s.mg_work = reinterpret_cast<uint32_t *>(s.n_comps + 10);
            cub::DeviceScan::ExclusiveSum(nullptr, offer_scan_bytes, s.off_cnt, s.off_pos, N + 1, st);
            if ((e = ctx->offer_scan.reserve(offer_scan_bytes)) != cudaSuccess) return cuda_fail(ctx, e, "alloc join offers");
            const size_t mg_smem = (size_t)mg_warps * s.mg_warp_bytes;
            if (mg_smem > 48 * 1024 &&
                (e = cudaFuncSetAttribute(offer_merge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mg_smem)) !=
                    cudaSuccess)
                return cuda_fail(ctx, e, "join merge");
        }
    }
    if (!s.off_lin) s.jt_rows = 0;   // locked inserts: the warp-per-node join

    // GenerateControl (kgraph.cpp:254-270): C distinct random nodes, exact K-NN.
    if (g_verbosity > 0) std::cerr << "Generating control..." << std::endl;
    std::vector<uint32_t> hctrl(C);
    {
        std::mt19937 rng(params->seed);
        std::vector<uint32_t> idx(N);
        std::iota(idx.begin(), idx.end(), 0u);
        for (uint32_t i = 0; i < C; ++i) {
            uint32_t j = i + rng() % (N - i);
            std::swap(idx[i], idx[j]);
            hctrl[i] = idx[i];
        }
    }
    DevBuf &dctrl = B[19];
    if ((e = dctrl.reserve((size_t)C * 4 + (size_t)C * K * 8 + (size_t)C * 5 * 4 + 16)) != cudaSuccess)
        return cuda_fail(ctx, e, "alloc controls");
    uint32_t *ctrl = dctrl.as<uint32_t>();
    uint32_t *ctrl_i = ctrl + C;
    float *ctrl_d = reinterpret_cast<float *>(ctrl_i + (size_t)C * K);
    float *ctrl_out = ctrl_d + (size_t)C * K;
    cudaMemcpyAsync(ctrl, hctrl.data(), (size_t)C * 4, cudaMemcpyHostToDevice, st);
    cudaEventRecord(ctx->ev0, st);
    if (C && (e = launch_linear_search(ctx, ctrl, C, K, ctrl_i, ctrl_d)) != cudaSuccess)
        return cuda_fail(ctx, e, "controls");

    if (g_verbosity > 0) std::cerr << "Initializing..." << std::endl;
    init_kernel<<<grid_for(ctx), 256, 0, st>>>(s);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "init");

    kg_index_info inf{};
    inf.stop_condition = 0;
    inf.recall = 0;
    inf.accuracy = std::numeric_limits<float>::max();
    inf.cost = 0;
    inf.iterations = 0;
    inf.delta = 1.0f;
    const float total = N * float(N - 1) / 2;
    // Pinned host copies of each iteration's statistics; the graphs copy into them.
    HostPinned hp;
    if ((e = hp.alloc(64 + (size_t)C * 5 * 4)) != cudaSuccess) return cuda_fail(ctx, e, "alloc host stats");
    const unsigned long long *hstat = reinterpret_cast<unsigned long long *>(hp.p);
    const float *hout = reinterpret_cast<float *>(hp.p + 64);
    unsigned long long fp32_pairs = 0, hstat_prev = 0;
    const unsigned long long *hwork = reinterpret_cast<const unsigned long long *>(hp.p + 40);
    unsigned long long work_prev[3] = {0, 0, 0};
    ctx->last_build_iters.clear();
    struct EventPair {   // device time of one iteration's launches
        cudaEvent_t a = nullptr, b = nullptr;
        ~EventPair() { if (a) cudaEventDestroy(a); if (b) cudaEventDestroy(b); }
    } itev;
    if ((e = cudaEventCreate(&itev.a)) != cudaSuccess || (e = cudaEventCreate(&itev.b)) != cudaSuccess)
        return cuda_fail(ctx, e, "events");
    double full_frac = 0.0;   // fraction of full pools after the last join
    unsigned tc_iters = 0;

    // One iteration's device work, recorded into the stream: the FP32 join,
    // the statistics with their copies to the host, and the update.
    // A deferred join goes in rounds of consecutive nodes (join, grouping and
    // merge each), as many as keep a round's offers -- at most 2 x C(2S, 2)
    // per node in the first iteration -- within the record buffer; each pool
    // then takes its offers round by round, one more order of its own offers.
    const uint32_t join_rounds =
        s.off_lin ? (uint32_t)std::min<uint64_t>(64, std::max<uint64_t>(1, ((uint64_t)N * 2 * S * (2 * S - 1) + s.off_cap - 1) / s.off_cap))
                  : 1u;
    // The deferred inserts around one join round: the record cursor and counts
    // cleared before it; the grouping and the pools' merge after it.
    auto rec_offers_begin = [&]() {
        cudaMemsetAsync(s.off_cursor, 0, 16, st);   // the offer cursor and the merge's claim counter
        cudaMemsetAsync(s.off_cnt, 0, (n + 1) * 4, st);
        cudaMemsetAsync(s.off_fill, 0, n * 4, st);
    };
    auto rec_offers_end = [&](const BuildState &sr) -> cudaError_t {
        size_t sb = offer_scan_bytes;
        cudaError_t e2 = cub::DeviceScan::ExclusiveSum(ctx->offer_scan.p, sb, s.off_cnt, s.off_pos, N + 1, st);
        if (e2 != cudaSuccess) return e2;
        offer_scatter_kernel<<<grid_for(ctx), 256, 0, st>>>(sr);
        const int bps = std::max(1, (int)((228u << 10) / ((size_t)mg_warps * s.mg_warp_bytes + 1024)));
        offer_merge_kernel<<<ctx->num_sms * bps, mg_warps * 32, (size_t)mg_warps * s.mg_warp_bytes, st>>>(sr);
        return cudaGetLastError();
    };
    auto rec_join = [&]() -> cudaError_t {
        for (uint32_t r = 0; r < join_rounds; ++r) {
            BuildState sr = s;
            sr.node_lo = (uint32_t)((uint64_t)N * r / join_rounds);
            sr.node_hi = (uint32_t)((uint64_t)N * (r + 1) / join_rounds);
            cudaMemsetAsync(s.work, 0, 4, st);
            if (s.off_lin) rec_offers_begin();
            if (s.jt_rows)
                join_tile_kernel<<<ctx->num_sms * jt_blocks, JT_WARPS * 32, jt_smem, st>>>(sr);
            else
                join_kernel<<<grid_for(ctx), 256, 0, st>>>(sr);
            if (s.off_lin) {
                cudaError_t e2 = rec_offers_end(sr);
                if (e2 != cudaSuccess) return e2;
            }
        }
        return cudaGetLastError();
    };
    auto rec_stats = [&]() -> cudaError_t {
        cudaMemsetAsync(s.stat, 0, 24, st);
        stats_kernel<<<grid_for(ctx, 4), 256, 0, st>>>(s);
        if (C) controls_kernel<<<(C + 127) / 128, 128, 0, st>>>(s, ctrl, ctrl_d, C, ctrl_out);
        cudaMemcpyAsync(hp.p, s.n_comps, 4 * 8, cudaMemcpyDeviceToHost, st);
        cudaMemcpyAsync(hp.p + 40, s.list_entries, 3 * 8, cudaMemcpyDeviceToHost, st);   // lists, inserts[2]
        if (C) cudaMemcpyAsync(hp.p + 64, ctrl_out, (size_t)C * 5 * 4, cudaMemcpyDeviceToHost, st);
        return cudaGetLastError();
    };
    DevBuf &gscan = B[24];   // scan storage owned by the captured update (never reallocated under it)
    auto rec_update = [&]() -> cudaError_t {
        update_m_kernel<<<grid_for(ctx, 4), 256, 0, st>>>(s);
        update_count_kernel<<<grid_for(ctx), 256, 0, st>>>(s);
        cudaError_t e2;
        if ((e2 = scan_counts(ctx, s.rcnt_new, s.roff_new, N, &gscan)) != cudaSuccess) return e2;
        if ((e2 = scan_counts(ctx, s.rcnt_old, s.roff_old, N, &gscan)) != cudaSuccess) return e2;
        cudaMemsetAsync(s.rcnt_new, 0, n * 4, st);
        cudaMemsetAsync(s.rcnt_old, 0, n * 4, st);
        update_fill_kernel<<<grid_for(ctx), 256, 0, st>>>(s);
        update_cap_kernel<<<grid_for(ctx), 256, 0, st>>>(s);
        iter_advance_kernel<<<1, 32, 0, st>>>(s);
        return cudaGetLastError();
    };
    // Everything a capture needs is set up before it: the join's cache carveout
    // and the update's scan storage.
    cudaFuncSetAttribute(join_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxL1);
    {
        size_t sb = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, sb, s.rcnt_new, s.roff_new, N + 1, st);
        if ((e = gscan.reserve(sb)) != cudaSuccess) return cuda_fail(ctx, e, "alloc scan");
    }
    // The iterations replay captured CUDA graphs.  An FP32 iteration is one
    // launch: the previous iteration's update (deferred until the host has read
    // that iteration's statistics and decided to go on), the join and the
    // statistics.  An iteration whose join runs on the tensor cores (its round
    // count is decided on the host) launches the update graph, its join rounds,
    // then the statistics graph.
    StreamGraph g_first, g_steady, g_update, g_stats;
    unsigned graph_launches = 0;
    bool pending_update = false;   // the last iteration's update is still to run
    bool stopped = false;
    auto run_graph = [&](StreamGraph &g, auto &&record) -> cudaError_t {
        if (!g.ready()) {
            cudaError_t e2 = g.capture(st, record);
            if (e2 != cudaSuccess) return e2;
        }
        ++graph_launches;
        return g.launch(st);
    };
    for (uint32_t it = 0; (params->iterations <= 0) || (it < params->iterations); ++it) {
        ++inf.iterations;
        cudaEventRecord(itev.a, st);
        // The tensor-core filter can only skip pairs against finite radii: while
        // most pools are still filling, every pair passes it and the fused
        // CUDA-core join is the cheaper path.
        const bool tc_now = use_tc && (tc_always || full_frac >= JOIN_TC_MIN_FULL);
        if (tc_now) {
            ++tc_iters;
            if (pending_update && (e = run_graph(g_update, rec_update)) != cudaSuccess)
                return cuda_fail(ctx, e, "update graph");
            cudaMemsetAsync(s.work, 0, 4, st);
            // rounds of nodes whose worst-case pair counts fit the queue
            if ((e = join_tc_worst(st, s, jworst)) != cudaSuccess) return cuda_fail(ctx, e, "join");
            if ((e = scan_counts64(ctx, jworst, jpre, N)) != cudaSuccess) return cuda_fail(ctx, e, "scan");
            cudaMemcpyAsync(hp.p + 32, jpre + N, 8, cudaMemcpyDeviceToHost, st);
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "join");
            const uint64_t total = reinterpret_cast<const uint64_t *>(hp.p)[4];
            const uint64_t slab = qcap - join_tc_node_max(s);
            const uint32_t R = (uint32_t)std::max<uint64_t>(1, (total + slab - 1) / slab);
            if ((e = ctx->joinb.reserve((size_t)(R + 1) * 4)) != cudaSuccess) return cuda_fail(ctx, e, "alloc");
            jq.bounds = ctx->joinb.as<uint32_t>();
            if ((e = join_tc_bounds(st, jpre, N, slab, R, jq.bounds)) != cudaSuccess) return cuda_fail(ctx, e, "join");
            // the rounds' offers (the queue bounds a round's pairs, not its offers) wait for one
            // merge after the last round: each pool takes all of its offers of the iteration
            // together, in the merge's order
            if (s.off_lin) rec_offers_begin();
            for (uint32_t r = 0; r < R; ++r)
                if ((e = launch_join_tc(ctx->num_sms, grid_for(ctx), st, s, jq, r, fp8 ? 1 : 0)) != cudaSuccess)
                    return cuda_fail(ctx, e, "join");
            if (s.off_lin && (e = rec_offers_end(s)) != cudaSuccess) return cuda_fail(ctx, e, "join merge");
            if ((e = run_graph(g_stats, rec_stats)) != cudaSuccess) return cuda_fail(ctx, e, "statistics graph");
        } else if (pending_update) {
            e = run_graph(g_steady, [&]() -> cudaError_t {
                cudaError_t e2 = rec_update();
                if (e2 == cudaSuccess) e2 = rec_join();
                return e2 == cudaSuccess ? rec_stats() : e2;
            });
            if (e != cudaSuccess) return cuda_fail(ctx, e, "iteration graph");
        } else {
            e = run_graph(g_first, [&]() -> cudaError_t {
                cudaError_t e2 = rec_join();
                return e2 == cudaSuccess ? rec_stats() : e2;
            });
            if (e != cudaSuccess) return cuda_fail(ctx, e, "iteration graph");
        }
        pending_update = false;
        cudaEventRecord(itev.b, st);
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "join");
        int de = check_device_error(ctx, "build");
        if (de != KG_OK) return de;
        {
            kg_build_iteration rec{};
            rec.pairs = hstat[0] - hstat_prev;
            rec.list_entries = hwork[0] - work_prev[0];
            rec.insert_attempts = hwork[1] - work_prev[1];
            rec.inserts_landed = hwork[2] - work_prev[2];
            cudaEventElapsedTime(&rec.ms, itev.a, itev.b);
            rec.tensor_core = tc_now ? 1u : 0u;
            for (int k = 0; k < 3; ++k) work_prev[k] = hwork[k];
            ctx->last_build_iters.push_back(rec);
        }
        // kgraph.cpp:927-963: the per-iteration statistics
        if (!tc_now) fp32_pairs += hstat[0] - hstat_prev;
        hstat_prev = hstat[0];
        full_frac = (double)hstat[3] / N;
        inf.cost = hstat[0] / total;
        inf.delta = (float)((double)hstat[1] / K / N);
        inf.M = (float)((double)hstat[2] / N);
        float rs = 0, as = 0, ors = 0, oa = 0, oe = 0;
        for (uint32_t c = 0; c < C; ++c) {
            if (hout[c * 5] < 0) return set_error(ctx, KG_E_RUNTIME, "distance is unstable");
            rs += hout[c * 5]; as += hout[c * 5 + 1]; ors += hout[c * 5 + 2]; oa += hout[c * 5 + 3]; oe += hout[c * 5 + 4];
        }
        inf.recall = C ? rs / C : 0.f;
        inf.accuracy = C ? as / C : 0.f;
        auto print_iteration = [&]() {
            auto now = std::chrono::steady_clock::now();
            std::cerr << "iteration: " << inf.iterations << " recall: " << inf.recall << " accuracy: " << inf.accuracy
                      << " cost: " << inf.cost << " M: " << inf.M << " delta: " << inf.delta
                      << " time: " << std::chrono::duration<double>(now - t_start).count()
                      << " one-recall: " << (C ? ors / C : 0.f) << " one-ratio: " << (C ? (oa / C) / (oe / C) : 0.f)
                      << std::endl;
        };
        if (g_verbosity > 0) print_iteration();
        if (inf.delta <= params->delta) { inf.stop_condition = 1; stopped = true; break; }
        if (inf.recall >= params->recall) { inf.stop_condition = 2; stopped = true; break; }
        if (ctx->last_build_iters.back().pairs == 0) {
            // A join of no pairs lands no insert: the pools stay as they are and
            // found is clear for every node, so the next update keeps every M
            // (kgraph.cpp:825-833) and finds no flagged entry below it (the last
            // update cleared them all), and the next join has no pairs again.
            // Every remaining iteration of the reference repeats this one, with
            // the same statistics, and its updates change nothing that reaches
            // the graph: they are counted, not run.  (Without an iteration cap
            // the reference would repeat it for ever; the build ends here.)
            while (params->iterations > 0 && inf.iterations < (uint32_t)params->iterations) {
                ++inf.iterations;
                kg_build_iteration idle{};
                idle.tensor_core = ctx->last_build_iters.back().tensor_core;
                ctx->last_build_iters.push_back(idle);
                if (g_verbosity > 0) print_iteration();
            }
            break;
        }
        pending_update = true;   // update (kgraph.cpp:816-883), launched with the next iteration
    }
    // The iteration cap ended the loop: the reference has run the last update
    // (its M growth and flag clearing reach the finalized graph).
    if (!stopped && pending_update && (e = run_graph(g_update, rec_update)) != cudaSuccess)
        return cuda_fail(ctx, e, "update graph");
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "update");
    ctx->last_build_graph_launches = graph_launches;

    ctx->joinq.release();   // the candidate queue is only needed while joining
    ctx->joinaux.release();
    ctx->joinb.release();

    // finalize (kgraph.cpp:975-988) into the context's CSR graph
    DevBuf &cnt = ctx->build_scratch[22];
    if ((e = cnt.reserve((n + 1) * 8)) != cudaSuccess) return cuda_fail(ctx, e, "alloc");
    cudaMemsetAsync(cnt.p, 0, (n + 1) * 8, st);
    finalize_count_kernel<<<grid_for(ctx, 4), 256, 0, st>>>(s, cnt.as<uint64_t>());
    if ((e = ctx->offsets.reserve((n + 1) * 8)) != cudaSuccess) return cuda_fail(ctx, e, "alloc graph");
    if ((e = scan_counts64(ctx, cnt.as<uint64_t>(), ctx->offsets.as<uint64_t>(), N)) != cudaSuccess)
        return cuda_fail(ctx, e, "scan");
    uint64_t E = 0;
    cudaMemcpyAsync(&E, ctx->offsets.as<uint64_t>() + N, 8, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    if ((e = ctx->nbr.reserve(E * 4 + 4)) != cudaSuccess || (e = ctx->nbr_d.reserve(E * 4 + 4)) != cudaSuccess ||
        (e = ctx->Mnode.reserve(n * 4)) != cudaSuccess)
        return cuda_fail(ctx, e, "alloc graph");
    finalize_fill_kernel<<<grid_for(ctx), 256, 0, st>>>(s, ctx->offsets.as<uint64_t>(), ctx->nbr.as<uint32_t>(),
                                                         ctx->nbr_d.as<float>(), ctx->Mnode.as<uint32_t>());
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "finalize");
    ctx->gn = N;
    ctx->E = E;
    ctx->no_dist = false;
    ctx->has_graph = true;
    ++ctx->graph_version;
    int de = check_device_error(ctx, "build");
    if (de != KG_OK) return de;
    if (params->reverse) {
        int r = graph_reverse(ctx, params->reverse);
        if (r != KG_OK) return r;
    }
    if (params->prune) {
        int r = graph_prune(ctx, params->prune);
        if (r != KG_OK) return r;
    }
    cudaEventRecord(ctx->ev1, st);
    JoinTcStats ts{};
    cudaMemcpyAsync(&ts, s.tc, sizeof(ts), cudaMemcpyDeviceToHost, st);
    unsigned long long lists = 0;
    cudaMemcpyAsync(&lists, s.list_entries, 8, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "build");
    cudaEventElapsedTime(&ctx->last_build_ms, ctx->ev0, ctx->ev1);
    kg_join_stats &js = ctx->last_join;
    js = kg_join_stats{};
    js.mode = tc_iters ? (fp8 ? KG_JOIN_FP8 : KG_JOIN_BF16) : KG_JOIN_FP32;
    js.tc_iterations = tc_iters;
    js.pairs = hstat_prev;
    js.rechecked = ts.rechecked + fp32_pairs;
    js.sampled = ts.sampled;
    js.violations = ts.violations;
    auto bits = [](unsigned u) { float f; std::memcpy(&f, &u, 4); return (double)f; };
    js.max_abs_err = bits(ts.max_abs_bits);
    js.max_rel_err = bits(ts.max_rel_bits);
    js.max_err_over_margin = bits(ts.max_ratio_bits);
    js.mean_abs_err = ts.sampled ? ts.sum_abs / ts.sampled : 0.0;
    js.mean_err_over_margin = ts.sampled ? ts.sum_ratio / ts.sampled : 0.0;
    js.mean_rel_err = ts.rel_count ? ts.sum_rel / ts.rel_count : 0.0;
    ctx->last_build_work[0] = hstat_prev;
    ctx->last_build_work[1] = lists;
    ctx->last_build_work[2] = inf.iterations;
    if (info) *info = inf;
    return KG_OK;
}

extern "C" int kg_last_build_iterations(kg_ctx *ctx, kg_build_iteration *out, unsigned cap, unsigned *n) {
    if (!ctx || !n) return KG_E_INVALID;
    std::lock_guard<std::mutex> guard(ctx->mu);
    *n = (unsigned)ctx->last_build_iters.size();
    for (unsigned i = 0; out && i < cap && i < *n; ++i) out[i] = ctx->last_build_iters[i];
    return KG_OK;
}

extern "C" int kg_last_build_work(kg_ctx *ctx, uint64_t *pairs, uint64_t *list_entries, unsigned *iterations) {
    if (!ctx) return KG_E_INVALID;
    std::lock_guard<std::mutex> guard(ctx->mu);
    if (pairs) *pairs = ctx->last_build_work[0];
    if (list_entries) *list_entries = ctx->last_build_work[1];
    if (iterations) *iterations = (unsigned)ctx->last_build_work[2];
    return KG_OK;
}

extern "C" int kg_set_join_precision(kg_ctx *ctx, int mode) {
    if (!ctx || mode < KG_JOIN_AUTO || mode > KG_JOIN_FP8_ALWAYS) return KG_E_INVALID;
    std::lock_guard<std::mutex> guard(ctx->mu);
    ctx->join_mode = mode;
    return KG_OK;
}

// The deferred-insert merge (offer_scatter_kernel + offer_merge_kernel) on
// caller data: n pools of Lp = L+1 entries (host rows of Lp, ids with the new
// flag in bit 31), their list lengths and radii (in/out), and n_off offers
// (target, candidate, distance, source | OFFER_UU); found[src] (out) is set as
// in the join.  For tests of the merge against serial inserts.
extern "C" int kg_join_merge_check(kg_ctx *ctx, unsigned n, unsigned L, unsigned K, float *pool_d, uint32_t *pool_i,
                                   uint32_t *nodeL, float *radius, size_t n_off, const uint32_t *target,
                                   const uint32_t *cand, const float *dist, const uint32_t *src, uint32_t *found) {
    if (!ctx) return KG_E_INVALID;
    std::lock_guard<std::mutex> guard(ctx->mu);
    cudaSetDevice(ctx->device);
    if (n == 0 || L == 0 || K > L || !pool_d || !pool_i || !nodeL || !radius || !found || (n_off && (!target || !cand || !dist || !src)))
        return set_error(ctx, KG_E_INVALID, "bad merge check arguments");
    for (size_t k = 0; k < n_off; ++k)
        if (target[k] >= n || (src[k] & ~OFFER_UU) >= n) return set_error(ctx, KG_E_INVALID, "offer node out of range");
    BuildState s{};
    s.L = L; s.Lp = L + 1; s.K = K;
    s.PS = (s.Lp + 7) / 8 * 8;
    s.D.n = n;
    s.mg_warp_bytes = (uint32_t)merge_warp_bytes(s.PS);
    const int mg_warps = (int)std::min<size_t>(MG_WARPS, (227u << 10) / s.mg_warp_bytes);
    if (mg_warps < 1) return set_error(ctx, KG_E_INVALID, "L too large for the merge");
    std::vector<float> hd((size_t)n * s.PS, FLT_MAX);
    std::vector<uint32_t> hi((size_t)n * s.PS, UNSET_ID), cnt(n + 1, 0);
    for (size_t x = 0; x < n; ++x)
        for (uint32_t j = 0; j < s.Lp; ++j) { hd[x * s.PS + j] = pool_d[x * s.Lp + j]; hi[x * s.PS + j] = pool_i[x * s.Lp + j]; }
    // grouped by target on the host, each pool's offers in the caller's order (the order they
    // arrive in for the merge's `found` replay)
    std::vector<uint4> lin(std::max<size_t>(n_off, 1));
    std::vector<uint64_t> pos(n + 1, 0);
    for (size_t k = 0; k < n_off; ++k) ++cnt[target[k]];
    for (size_t x = 0; x < n; ++x) pos[x + 1] = pos[x] + cnt[x];
    {
        std::vector<uint64_t> fill(pos.begin(), pos.end() - 1);
        for (size_t k = 0; k < n_off; ++k) {
            uint32_t db;
            std::memcpy(&db, &dist[k], 4);
            lin[fill[target[k]]++] = make_uint4(target[k], cand[k], db, src[k]);
        }
    }
    DevBuf b[10];
    cudaError_t e;
    const size_t rows = (size_t)n * s.PS;
    size_t scan_bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_bytes, (uint32_t *)nullptr, (uint64_t *)nullptr, n + 1, ctx->stream);
    if ((e = b[0].reserve(rows * 4)) != cudaSuccess || (e = b[1].reserve(rows * 4)) != cudaSuccess ||
        (e = b[2].reserve((size_t)n * 4)) != cudaSuccess || (e = b[3].reserve((size_t)n * 4)) != cudaSuccess ||
        (e = b[4].reserve((size_t)n * 4)) != cudaSuccess || (e = b[5].reserve(lin.size() * 16)) != cudaSuccess ||
        (e = b[6].reserve(lin.size() * 16)) != cudaSuccess || (e = b[7].reserve((size_t)(n + 1) * 12 + (size_t)n * 4)) != cudaSuccess ||
        (e = b[8].reserve(64)) != cudaSuccess || (e = b[9].reserve(scan_bytes)) != cudaSuccess)
        return cuda_fail(ctx, e, "alloc merge check");
    s.pool_d = b[0].as<float>(); s.pool_i = b[1].as<uint32_t>();
    s.nodeL = b[2].as<uint32_t>(); s.radius = b[3].as<float>(); s.found = b[4].as<uint32_t>();
    s.off_lin = b[5].as<uint4>(); s.off_grp = b[6].as<uint4>();
    s.off_pos = b[7].as<uint64_t>();
    s.off_cnt = reinterpret_cast<uint32_t *>(s.off_pos + n + 1);
    s.off_fill = s.off_cnt + n + 1;
    s.off_cursor = b[8].as<unsigned long long>();
    s.mg_work = reinterpret_cast<uint32_t *>(s.off_cursor + 1);
    s.inserts = s.off_cursor + 2;
    s.off_cap = n_off;
    cudaStream_t st = ctx->stream;
    const unsigned long long head[4] = {n_off, 0, 0, 0};
    cudaMemcpyAsync(s.pool_d, hd.data(), rows * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s.pool_i, hi.data(), rows * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s.nodeL, nodeL, (size_t)n * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s.radius, radius, (size_t)n * 4, cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(s.found, 0, (size_t)n * 4, st);
    cudaMemcpyAsync(s.off_grp, lin.data(), lin.size() * 16, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s.off_cnt, cnt.data(), (size_t)(n + 1) * 4, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s.off_pos, pos.data(), (size_t)(n + 1) * 8, cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(s.off_cursor, head, sizeof(head), cudaMemcpyHostToDevice, st);
    const size_t mg_smem = (size_t)mg_warps * s.mg_warp_bytes;
    if (mg_smem > 48 * 1024 &&
        (e = cudaFuncSetAttribute(offer_merge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)mg_smem)) != cudaSuccess)
        return cuda_fail(ctx, e, "merge check");
    offer_merge_kernel<<<ctx->num_sms, mg_warps * 32, mg_smem, st>>>(s);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(ctx, e, "merge check launch");
    cudaMemcpyAsync(hd.data(), s.pool_d, rows * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hi.data(), s.pool_i, rows * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(nodeL, s.nodeL, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(radius, s.radius, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(found, s.found, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "merge check");
    for (size_t x = 0; x < n; ++x)
        for (uint32_t j = 0; j < s.Lp; ++j) { pool_d[x * s.Lp + j] = hd[x * s.PS + j]; pool_i[x * s.Lp + j] = hi[x * s.PS + j]; }
    return KG_OK;
}

extern "C" int kg_set_join_offer_capacity(kg_ctx *ctx, size_t offers) {
    if (!ctx) return KG_E_INVALID;
    std::lock_guard<std::mutex> guard(ctx->mu);
    ctx->offer_cap = offers;
    return KG_OK;
}

extern "C" int kg_set_join_inserts(kg_ctx *ctx, int mode) {
    if (!ctx || mode < KG_INSERTS_AUTO || mode > KG_INSERTS_DEFERRED) return KG_E_INVALID;
    std::lock_guard<std::mutex> guard(ctx->mu);
    ctx->join_inserts = mode;
    return KG_OK;
}

extern "C" int kg_last_build_graphs(kg_ctx *ctx, unsigned *graph_launches) {
    if (!ctx || !graph_launches) return KG_E_INVALID;
    std::lock_guard<std::mutex> guard(ctx->mu);
    *graph_launches = ctx->last_build_graph_launches;
    return KG_OK;
}

extern "C" int kg_last_join_stats(kg_ctx *ctx, kg_join_stats *out) {
    if (!ctx || !out) return KG_E_INVALID;
    std::lock_guard<std::mutex> guard(ctx->mu);
    *out = ctx->last_join;
    return KG_OK;
}
