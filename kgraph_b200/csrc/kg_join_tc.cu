// Local join on the fifth-generation tensor cores (tcgen05), for D >= 64.
//
// KGraphConstructor::join + Nhood::join (kgraph.cpp:740-751, 797-815) visit,
// for every node n, the pairs new x new (i < j) and new x old of n's sample
// lists and try each pair's distance against both endpoints' pools.  Here one
// CTA takes one node at a time:
//
//   1. U = new ++ old (positions 0..a-1 are new).  U's rows are staged into
//      shared memory as BF16, CENTERED on x_n (row - x_n, in FP32, then
//      rounded): the distances are translation invariant, and centering makes
//      the BF16 error scale with |x_u - x_n| |x_j - x_n| -- neighbour
//      distances -- instead of the raw norms.  The same pass keeps, per row,
//      h = |x_u - x_n|^2 / 2 and c = (x_u - x_n) . x_n in FP32.
//   2. tcgen05.mma (kind::f16, BF16 x BF16 -> FP32 in TMEM) forms the Gram
//      block of U (128-row tiles, M) against the new rows (128-column tiles,
//      N); the new rows are the first rows of U, so B is read from the same
//      staged buffer.
//   3. Each epilogue thread owns one U row (one TMEM lane) and derives the
//      approximate distance of each of its pairs: euclidean h_u + h_j - g,
//      l2sqr twice that, angular -(g + c_u + c_j + |x_n|^2) / (n_u n_j + eps).
//      A pair whose approximate distance minus a rigorous error margin E is
//      above BOTH endpoints' radius cannot pass the reference's unlocked
//      radius test (kgraph.cpp:725, radii only shrink during a join), so it is
//      skipped.  Every other pair is recomputed with the canonical FP32
//      distance and goes through the same locked insert as the CUDA-core join:
//      every heap insert, ordering and stored distance is decided in FP32.
//
// The margin E bounds |approx - exact| + |canonical FP32 - exact| with a
// factor 2 of slack: BF16 rounding of both operands (2^-8 + 2^-17 relative to
// |x_u - x_n| |x_j - x_n|), FP32 accumulation of D products (up to 2^-23 each),
// the FP32 centering and norm sums, and the canonical distance's own error
// (D + 4 ulps of the uncentered norms).  A sample of nodes (about 1 in 2048)
// also evaluates every pair in FP64 and records the tile error and its ratio
// to E (JoinTcStats), so the bound is checked on every run.
//
// All waits are bounded: the MMA completion barrier gives up after ~1 s,
// raises ERR_TC_TIMEOUT and the CTA drains, frees its TMEM and returns.
#include <algorithm>
#include <cfloat>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include "kg_build.h"
#include "kg_insert.cuh"
#include "kg_tc.cuh"

namespace kgb {
namespace {

constexpr int TC_THREADS = 256;          // 8 warps: warp w reads TMEM lanes 32*(w%4).., columns 64*(w/4)..
constexpr uint32_t TC_M = 128;           // U rows per tile = TMEM lanes
constexpr uint32_t TC_N = 128;           // new columns per tile = TMEM columns
constexpr uint32_t TC_TMEM_COLS = 128;
constexpr long long TC_WAIT_CYCLES = 2000000000ll;
constexpr uint32_t TC_CLAIM = 16;               // nodes claimed per CTA at a time
constexpr uint32_t TC_MIN_SMEM = 58 * 1024;   // at most 3 CTAs (384 TMEM columns) per SM

__device__ __forceinline__ bool sampled_node(uint32_t n) { return ((n * 0x9E3779B1u) >> 21) == 0; }

// Approximate distance of a pair from its Gram entry g, and the margin E.
struct Approx { float d, e; };
__device__ __forceinline__ Approx approx_dist(int metric, float g, float hu, float hj, float cu, float cj, float nu,
                                              float nj, float qn, float et, float gam) {
    const float pt = 2.0f * sqrtf(hu * hj);   // |x_u - x_n| |x_j - x_n|
    Approx r;
    if (metric == METRIC_ANGULAR) {
        const float full = g + cu + cj + qn;
        const float den = nu * nj + FLT_EPSILON;
        r.d = -full / den;
        const float edot = et * pt + gam * (sqrtf(2.0f * hu) + sqrtf(2.0f * hj)) * sqrtf(qn) + gam * qn +
                           4.0f * 5.96e-8f * (fabsf(cu) + fabsf(cj) + qn + fabsf(g));
        r.e = 2.0f * (edot / den + gam * (nu * nj) / den + 2.0f * gam * fabsf(r.d)) + 1e-30f;
    } else if (metric == METRIC_L2SQR) {
        r.d = 2.0f * ((hu + hj) - g);
        r.e = 2.0f * (2.0f * et * pt + 6.0f * gam * (hu + hj)) + 1e-30f;
    } else {
        r.d = (hu + hj) - g;
        r.e = 2.0f * (et * pt + gam * (hu + hj) + 2.0f * gam * (nu + nj)) + 1e-30f;
    }
    return r;
}

// The pair's distance in FP64 from the FP32 rows, by one warp (every lane
// returns it).
__device__ double warp_dist64(const DataView &D, uint32_t i, uint32_t j, int lane) {
    const float *a = D.X + (size_t)i * D.ld, *b = D.X + (size_t)j * D.ld;
    double s = 0, na = 0, nb = 0;
    for (uint32_t k = lane; k < D.d; k += 32) {
        const double x = a[k], y = b[k];
        if (D.metric == METRIC_ANGULAR) { s += x * y; na += x * x; nb += y * y; }
        else s += (x - y) * (x - y);
    }
    for (int o = 16; o; o >>= 1) {
        s += __shfl_xor_sync(FULL, s, o);
        na += __shfl_xor_sync(FULL, na, o);
        nb += __shfl_xor_sync(FULL, nb, o);
    }
    if (D.metric == METRIC_ANGULAR) return -s / (sqrt(na) * sqrt(nb) + (double)FLT_EPSILON);
    return D.metric == METRIC_L2SQR ? s : 0.5 * s;
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

struct TcShared {
    uint8_t *bbuf, *abuf;   // two 128-row tiles (BF16 or E4M3), K-major core-matrix layout
    float *xn;              // x_n, FP32
    uint32_t *uid;          // U ids (NO_ID for a bad id)
    float *ht, *cc, *nu, *rad;   // per U row: h, c, canonical norm term, radius snapshot
    float *scl, *rel;       // E4M3 tiles: per U row the scale and ||v - scale q|| / ||v||
};

// Rows [u0, u0 + rows) of U into `buf` (all 128 tile rows written; rows past
// `rows` are zero).  Warp w stages row groups w, w+8: lane l owns row
// (l & 7) of the group and 16-byte chunks (l >> 3) + 4i, so each quarter-warp
// store covers one contiguous 128-byte core matrix.
template <int PREC>
__device__ void stage_rows(const BuildState &s, const TcShared &sh, uint8_t *buf, uint32_t u0, uint32_t rows,
                           int warp, int lane);

// E4M3 rows with a per-row scale: v = x_u - x_n in FP32 (as the BF16 rows),
// scale = max|v| / 448, q = e4m3_satfinite(v / scale); per row the exact
// ||v - scale q|| (FP64, every term exact there) relative to ||v||, rounded up.
// Lane l owns row (l & 7) of a group of 8 and 16-byte chunks (16 elements)
// (l >> 3) + 4i; the row's maximum needs a first pass over its elements.
template <>
__device__ void stage_rows<1>(const BuildState &s, const TcShared &sh, uint8_t *buf, uint32_t u0, uint32_t rows,
                              int warp, int lane) {
    const uint32_t Dp = s.D.ld, nk16 = Dp >> 4;
    for (uint32_t g = warp; g * 8 < rows; g += TC_THREADS / 32) {
        const uint32_t rl = g * 8 + (lane & 7);
        const bool valid = rl < rows;
        const uint32_t id = valid ? sh.uid[u0 + rl] : NO_ID;
        const bool ok = id != NO_ID;
        float nrm = 0.f, rd = -FLT_MAX;
        if (ok && lane < 8) {
            nrm = s.D.norms[id];
            rd = *reinterpret_cast<volatile const float *>(s.radius + id);
        }
        const float *row = s.D.X + (size_t)(ok ? id : 0u) * Dp;
        float hs = 0.f, cs = 0.f, mx = 0.f;
        for (uint32_t k16 = lane >> 3; k16 < nk16; k16 += 4) {
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const float4 n0 = *reinterpret_cast<const float4 *>(sh.xn + 16 * k16 + 4 * h);
                const float4 a0 = ok ? ld4(row + 16 * k16 + 4 * h) : n0;
                const float e0 = a0.x - n0.x, e1 = a0.y - n0.y, e2 = a0.z - n0.z, e3 = a0.w - n0.w;
                hs += e0 * e0 + e1 * e1 + e2 * e2 + e3 * e3;
                cs += e0 * n0.x + e1 * n0.y + e2 * n0.z + e3 * n0.w;
                mx = fmaxf(mx, fmaxf(fmaxf(fabsf(e0), fabsf(e1)), fmaxf(fabsf(e2), fabsf(e3))));
            }
        }
        hs += __shfl_xor_sync(FULL, hs, 8);
        hs += __shfl_xor_sync(FULL, hs, 16);
        cs += __shfl_xor_sync(FULL, cs, 8);
        cs += __shfl_xor_sync(FULL, cs, 16);
        mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, 8));
        mx = fmaxf(mx, __shfl_xor_sync(FULL, mx, 16));
        const float scale = mx > 0.f ? mx / 448.f : 1.f;
        double err2 = 0.0;
        for (uint32_t k16 = lane >> 3; k16 < nk16; k16 += 4) {
            uint32_t wv[4];
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const float4 n0 = *reinterpret_cast<const float4 *>(sh.xn + 16 * k16 + 4 * h);
                const float4 a0 = ok ? ld4(row + 16 * k16 + 4 * h) : n0;
                const float e[4] = {a0.x - n0.x, a0.y - n0.y, a0.z - n0.z, a0.w - n0.w};
                uint32_t word = 0;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const __nv_fp8_storage_t qv = __nv_cvt_float_to_fp8(e[i] / scale, __NV_SATFINITE, __NV_E4M3);
                    const double y = (double)__half2float(__half(__nv_cvt_fp8_to_halfraw(qv, __NV_E4M3))) * (double)scale;
                    const double df = (double)e[i] - y;
                    err2 += df * df;
                    word |= (uint32_t)qv << (8 * i);
                }
                wv[h] = word;
            }
            *reinterpret_cast<uint4 *>(buf + tc::kmajor_off8(rl, 16 * k16, Dp)) = make_uint4(wv[0], wv[1], wv[2], wv[3]);
        }
        err2 += __shfl_xor_sync(FULL, err2, 8);
        err2 += __shfl_xor_sync(FULL, err2, 16);
        if (lane < 8 && valid) {
            const uint32_t u = u0 + rl;
            sh.ht[u] = 0.5f * hs;
            sh.cc[u] = cs;
            sh.nu[u] = nrm;
            sh.rad[u] = rd;
            sh.scl[u] = scale;
            // relative to ||v|| (hs carries an FP32 rounding: one more relative step of slack)
            sh.rel[u] = hs > 0.f ? __double2float_ru(sqrt(err2) / sqrt((double)hs) * (1.0 + 1e-5)) : 0.f;
        }
    }
    tc::fence_async_shared();   // make the generic-proxy stores visible to the MMA
}

template <>
__device__ void stage_rows<0>(const BuildState &s, const TcShared &sh, uint8_t *buf, uint32_t u0, uint32_t rows,
                              int warp, int lane) {
    const uint32_t Dp = s.D.ld, nk8 = Dp >> 3;
    // Rows past `rows` are left as they are: the MMA reads them, but their
    // products land only in masked rows / columns of the accumulator.
    for (uint32_t g = warp; g * 8 < rows; g += TC_THREADS / 32) {
        const uint32_t rl = g * 8 + (lane & 7);
        const bool valid = rl < rows;
        const uint32_t id = valid ? sh.uid[u0 + rl] : NO_ID;
        const bool ok = id != NO_ID;
        float nrm = 0.f, rd = -FLT_MAX;
        if (ok && lane < 8) {   // issued ahead of the row loads
            nrm = s.D.norms[id];
            rd = *reinterpret_cast<volatile const float *>(s.radius + id);
        }
        const float *row = s.D.X + (size_t)(ok ? id : 0u) * Dp;
        float hs = 0.f, cs = 0.f;
#pragma unroll 4
        for (uint32_t k8 = lane >> 3; k8 < nk8; k8 += 4) {
            float e[8], xv[8];
            const float4 n0 = *reinterpret_cast<const float4 *>(sh.xn + 8 * k8);
            const float4 n1 = *reinterpret_cast<const float4 *>(sh.xn + 8 * k8 + 4);
            xv[0] = n0.x; xv[1] = n0.y; xv[2] = n0.z; xv[3] = n0.w;
            xv[4] = n1.x; xv[5] = n1.y; xv[6] = n1.z; xv[7] = n1.w;
            if (ok) {
                const float4 a0 = ld4(row + 8 * k8), a1 = ld4(row + 8 * k8 + 4);
                e[0] = a0.x - xv[0]; e[1] = a0.y - xv[1]; e[2] = a0.z - xv[2]; e[3] = a0.w - xv[3];
                e[4] = a1.x - xv[4]; e[5] = a1.y - xv[5]; e[6] = a1.z - xv[6]; e[7] = a1.w - xv[7];
            } else {
#pragma unroll
                for (int i = 0; i < 8; ++i) e[i] = 0.f;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) { hs += e[i] * e[i]; cs += e[i] * xv[i]; }
            uint4 pk;
            pk.x = pack_bf16(e[0], e[1]); pk.y = pack_bf16(e[2], e[3]);
            pk.z = pack_bf16(e[4], e[5]); pk.w = pack_bf16(e[6], e[7]);
            *reinterpret_cast<uint4 *>(buf + tc::kmajor_off(rl, 8 * k8, Dp)) = pk;
        }
        hs += __shfl_xor_sync(FULL, hs, 8);
        hs += __shfl_xor_sync(FULL, hs, 16);
        cs += __shfl_xor_sync(FULL, cs, 8);
        cs += __shfl_xor_sync(FULL, cs, 16);
        if (lane < 8 && valid) {
            const uint32_t u = u0 + rl;
            sh.ht[u] = 0.5f * hs;
            sh.cc[u] = cs;
            sh.nu[u] = nrm;
            sh.rad[u] = rd;
        }
    }
    tc::fence_async_shared();   // make the generic-proxy stores visible to the MMA
}

template <int PREC>
__global__ void __launch_bounds__(TC_THREADS, 3) join_tc_kernel(BuildState s, uint32_t Umax, JoinQueue jq,
                                                                  uint32_t round) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t tmem_base, s_base, s_cnt;
    __shared__ uint32_t s_list[TC_CLAIM], s_la[TC_CLAIM], s_lb[TC_CLAIM];
    __shared__ uint32_t s_wcnt[TC_THREADS / 32];
    __shared__ unsigned long long s_wbase[TC_THREADS / 32];
    __shared__ float s_qn;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t Dp = s.D.ld, N = s.D.n;
    const uint32_t n_begin = jq.bounds[round], n_end = jq.bounds[round + 1];
    const uint32_t tile_bytes = TC_M * Dp * (PREC ? 1 : 2);
    TcShared sh;
    sh.bbuf = smem;
    sh.abuf = smem + tile_bytes;
    sh.xn = reinterpret_cast<float *>(smem + 2 * tile_bytes);
    sh.uid = reinterpret_cast<uint32_t *>(sh.xn + Dp);
    sh.ht = reinterpret_cast<float *>(sh.uid + Umax);
    sh.cc = sh.ht + Umax;
    sh.nu = sh.cc + Umax;
    sh.rad = sh.nu + Umax;
    sh.scl = sh.rad + Umax;
    sh.rel = sh.scl + Umax;

    if (warp == 0) tc::tmem_alloc(&tmem_base, TC_TMEM_COLS);
    if (tid == 0) tc::mbar_init(&mbar, 1);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    const int q = warp & 3, half = warp >> 2;
    const float et = 0.00390625f + 7.63e-6f + (float)(s.D.d + 4) * 1.1921e-7f;   // 2^-8 + 2^-17 + (D+4) 2^-23
    // E4M3 tiles: the products' FP32 accumulation, allowed 2^-20 per add, and the two scale multiplies
    const float g8 = (float)(s.D.d + 4) * 9.5367e-7f + 8.f * 5.9605e-8f;
    const float gam = (float)(s.D.d + 4) * 5.9605e-8f;                             // (D+4) 2^-24
    const int metric = s.D.metric;
    uint32_t phase = 0;
    bool aborted = false;
    unsigned long long comps = 0, passed = 0, sampled = 0, viol = 0, relc = 0;
    double sum_abs = 0, sum_ratio = 0, sum_rel = 0;
    float max_abs = 0.f, max_ratio = 0.f, max_rel = 0.f;

    for (;;) {
        // claim TC_CLAIM nodes of this round's range; keep those with new entries
        if (tid == 0) s_base = n_begin + atomicAdd(jq.work, TC_CLAIM);
        __syncthreads();
        const uint32_t base = s_base;
        if (base >= n_end) break;
        if (warp == 0) {
            const uint32_t nn = base + lane;
            bool act = false;
            uint32_t ca = 0, cb = 0;
            if (lane < (int)TC_CLAIM && nn < n_end) {
                s.found[nn] = 0;   // set again by the insert phase (kgraph.cpp:808-810)
                ca = s.cnt_new[nn];
                cb = s.cnt_old[nn];
                act = ca > 0;
            }
            const unsigned am = __ballot_sync(FULL, act);
            if (act) {
                const int slot = __popc(am & ((1u << lane) - 1u));
                s_list[slot] = nn;
                s_la[slot] = ca;
                s_lb[slot] = cb;
            }
            if (lane == 0) s_cnt = __popc(am);
        }
        __syncthreads();
        const uint32_t cnt = s_cnt;
        for (uint32_t li = 0; li < cnt && !aborted; ++li) {
        const uint32_t n = s_list[li];
        uint32_t a = s_la[li], b = s_lb[li];
        if (a > s.NEWCAP || b > s.OLDCAP) {
            if (tid == 0) raise_error(s.err, ERR_CAPACITY);
            a = min(a, s.NEWCAP);
            b = min(b, s.OLDCAP);
        }
        const uint32_t U = a + b;
        const uint32_t *nw = s.nn_new + (size_t)n * s.NEWCAP, *od = s.nn_old + (size_t)n * s.OLDCAP;
        for (uint32_t u = tid; u < U; u += TC_THREADS) {
            uint32_t id = u < a ? nw[u] : od[u - a];
            if (id >= N) { raise_error(s.err, ERR_BAD_ID); id = NO_ID; }
            sh.uid[u] = id;
        }
        const float *xrow = s.D.X + (size_t)n * Dp;
        for (uint32_t k = tid; k < Dp; k += TC_THREADS) sh.xn[k] = xrow[k];
        __syncthreads();
        if (warp == 0) {
            float qs = 0.f;
            for (uint32_t k = lane; k < Dp; k += 32) qs += sh.xn[k] * sh.xn[k];
            for (int o = 16; o; o >>= 1) qs += __shfl_xor_sync(FULL, qs, o);
            if (lane == 0) s_qn = qs;
        }
        const bool samp = sampled_node(n);
        for (uint32_t j0 = 0; j0 < a && !aborted; j0 += TC_N) {
            const uint32_t j1 = min(a, j0 + TC_N);
            stage_rows<PREC>(s, sh, sh.bbuf, j0, min(U, j0 + TC_M) - j0, warp, lane);
            for (uint32_t u0 = 0; u0 < U; u0 += TC_M) {
                const uint32_t u1 = min(U, u0 + TC_M);
                if (!(u1 > max(u0, a) || (u0 < a && u0 + 1 < j1))) continue;   // no pair needed in this tile
                const bool same = u0 == j0;
                if (!same) stage_rows<PREC>(s, sh, sh.abuf, u0, u1 - u0, warp, lane);
                tc::fence_before_sync();
                __syncthreads();
                if (tid == 0) {
                    tc::fence_after_sync();
                    const uint32_t aa = tc::smem_addr(same ? sh.bbuf : sh.abuf), ba = tc::smem_addr(sh.bbuf);
                    if constexpr (PREC == 1) {   // K = 32 bytes per step, rows of Dp bytes
                        const uint32_t idesc = tc::idesc_e4m3_f32(TC_M, TC_N);
                        for (uint32_t kk = 0; kk < Dp / 32; ++kk)
                            tc::mma_e4m3(tmem, tc::smem_desc(aa + kk * 256, 128, Dp * 8),
                                         tc::smem_desc(ba + kk * 256, 128, Dp * 8), idesc, kk > 0);
                    } else {
                        const uint32_t idesc = tc::idesc_bf16_f32(TC_M, TC_N);
                        for (uint32_t kk = 0; kk < Dp / 16; ++kk)
                            tc::mma_bf16(tmem, tc::smem_desc(aa + kk * 256, 128, Dp * 16),
                                         tc::smem_desc(ba + kk * 256, 128, Dp * 16), idesc, kk > 0);
                    }
                    tc::mma_commit(&mbar);
                }
                const bool ok = tc::mbar_wait(&mbar, phase, TC_WAIT_CYCLES);
                if (__syncthreads_or(!ok)) {
                    if (tid == 0) raise_error(s.err, ERR_TC_TIMEOUT);
                    aborted = true;
                    break;
                }
                phase ^= 1;
                tc::fence_after_sync();

                // ---- epilogue: this thread's U row against 64 columns
                const uint32_t u = u0 + 32 * q + lane;
                const bool uval = u < u1 && sh.uid[u] != NO_ID;
                const uint32_t idu = uval ? sh.uid[u] : 0u;
                const bool unew = u < a;
                const float hu = uval ? sh.ht[u] : 0.f, cu = uval ? sh.cc[u] : 0.f, nuu = uval ? sh.nu[u] : 0.f;
                const float radu = uval ? sh.rad[u] : -FLT_MAX;
                const float su = (PREC == 1 && uval) ? sh.scl[u] : 1.f, ru = (PREC == 1 && uval) ? sh.rel[u] : 0.f;
                const float qn = s_qn;
                unsigned pmask[2] = {0u, 0u};
                for (int part = 0; part < 2; ++part) {
                    const uint32_t cb = 64 * half + 32 * part;
                    if (j0 + cb >= j1) break;   // warp-uniform
                    float v[32];
                    tc::tmem_ld32(tmem + ((uint32_t)(32 * q) << 16) + cb, v);
                    unsigned pm = 0;
#pragma unroll
                    for (int c = 0; c < 32; ++c) {
                        const uint32_t j = j0 + cb + c;
                        const uint32_t idj = j < j1 ? sh.uid[j] : NO_ID;
                        const bool need = uval && idj != NO_ID && (!unew || (j > u && idj != idu));
                        if (need) {
                            ++comps;
                            float gv = v[c], etp = et;
                            if constexpr (PREC == 1) {   // the scales, and this pair's relative error
                                gv = gv * su * sh.scl[j];
                                const float rj = sh.rel[j];
                                etp = ru + rj + ru * rj + g8 * (1.f + ru) * (1.f + rj);
                            }
                            const Approx ap = approx_dist(metric, gv, hu, sh.ht[j], cu, sh.cc[j], nuu, sh.nu[j],
                                                          qn, etp, gam);
                            if (!(ap.d - ap.e > fmaxf(radu, sh.rad[j]))) pm |= 1u << c;
                        }
                    }
                    if (samp) {   // FP64 tile error on this node's pairs, one pair at a time per warp
                        unsigned nm = 0;
                        for (int c = 0; c < 32; ++c) {
                            const uint32_t j = j0 + cb + c;
                            const uint32_t idj = j < j1 ? sh.uid[j] : NO_ID;
                            if (uval && idj != NO_ID && (!unew || (j > u && idj != idu))) nm |= 1u << c;
                        }
                        for (;;) {
                            const unsigned any = __ballot_sync(FULL, nm != 0);
                            if (!any) break;
                            const int src = __ffs(any) - 1;
                            uint32_t ia = 0, ib = 0;
                            float apd = 0.f, ape = 0.f;
                            if (lane == src) {
                                const int c = __ffs(nm) - 1;
                                nm &= nm - 1;
                                const uint32_t j = j0 + cb + c;
                                float g = 0.f;
#pragma unroll
                                for (int k = 0; k < 32; ++k) if (k == c) g = v[k];
                                float etp = et;
                                if constexpr (PREC == 1) {
                                    g = g * su * sh.scl[j];
                                    const float rj = sh.rel[j];
                                    etp = ru + rj + ru * rj + g8 * (1.f + ru) * (1.f + rj);
                                }
                                const Approx ap = approx_dist(metric, g, hu, sh.ht[j], cu, sh.cc[j], nuu, sh.nu[j],
                                                              qn, etp, gam);
                                apd = ap.d;
                                ape = ap.e;
                                ia = idu;
                                ib = sh.uid[j];
                            }
                            ia = __shfl_sync(FULL, ia, src);
                            ib = __shfl_sync(FULL, ib, src);
                            apd = __shfl_sync(FULL, apd, src);
                            ape = __shfl_sync(FULL, ape, src);
                            const double d64 = warp_dist64(s.D, ia, ib, lane);
                            if (lane == 0) {
                                const double err = fabs((double)apd - d64);
                                const double ratio = err / (double)ape;
                                ++sampled;
                                sum_abs += err;
                                sum_ratio += ratio;
                                max_abs = fmaxf(max_abs, (float)err);
                                max_ratio = fmaxf(max_ratio, (float)ratio);
                                if (d64 != 0.0) {
                                    const double rel = err / fabs(d64);
                                    ++relc;
                                    sum_rel += rel;
                                    max_rel = fmaxf(max_rel, (float)rel);
                                }
                                if (err > (double)ape) ++viol;
                            }
                        }
                    }
                    pmask[part] = pm;
                }
                // append the survivors: one queue atomic per tile
                const uint32_t mine = __popc(pmask[0]) + __popc(pmask[1]);
                uint32_t incl = mine;
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += t;
                }
                if (lane == 31) s_wcnt[warp] = incl;
                __syncthreads();
                if (tid == 0) {
                    unsigned long long tot = 0;
                    for (int w = 0; w < TC_THREADS / 32; ++w) { s_wbase[w] = tot; tot += s_wcnt[w]; }
                    const unsigned long long b0 = tot ? atomicAdd(jq.tail, tot) : 0ull;
                    for (int w = 0; w < TC_THREADS / 32; ++w) s_wbase[w] += b0;
                }
                __syncthreads();
                unsigned long long pos = s_wbase[warp] + incl - mine;
                passed += mine;
                for (int part = 0; part < 2; ++part) {
                    unsigned pm = pmask[part];
                    const uint32_t cb = 64 * half + 32 * part;
                    while (pm) {
                        const int c = __ffs(pm) - 1;
                        pm &= pm - 1;
                        const uint32_t idj = sh.uid[j0 + cb + c];
                        jq.x[pos] = unew ? min(idu, idj) : idj;
                        jq.y[pos] = unew ? max(idu, idj) : idu;
                        jq.n[pos] = n;
                        ++pos;
                    }
                }
                tc::fence_before_sync();
                __syncthreads();   // TMEM and the A tile are free again
            }
        }
        __syncthreads();   // this node's shared arrays are free again
        }
        if (aborted) break;
    }

    if (aborted) tc::mbar_wait(&mbar, phase, TC_WAIT_CYCLES);   // the MMA still in flight, bounded
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_free(tmem, TC_TMEM_COLS);

    for (int o = 16; o; o >>= 1) {
        comps += __shfl_xor_sync(FULL, comps, o);
        passed += __shfl_xor_sync(FULL, passed, o);
        sampled += __shfl_xor_sync(FULL, sampled, o);
        viol += __shfl_xor_sync(FULL, viol, o);
        relc += __shfl_xor_sync(FULL, relc, o);
        sum_abs += __shfl_xor_sync(FULL, sum_abs, o);
        sum_ratio += __shfl_xor_sync(FULL, sum_ratio, o);
        sum_rel += __shfl_xor_sync(FULL, sum_rel, o);
        max_abs = fmaxf(max_abs, __shfl_xor_sync(FULL, max_abs, o));
        max_ratio = fmaxf(max_ratio, __shfl_xor_sync(FULL, max_ratio, o));
        max_rel = fmaxf(max_rel, __shfl_xor_sync(FULL, max_rel, o));
    }
    if (lane == 0) {
        if (comps) { atomicAdd(s.n_comps, comps); atomicAdd(&s.tc->pairs, comps); }
        if (passed) atomicAdd(&s.tc->rechecked, passed);
        if (viol) atomicAdd(&s.tc->violations, viol);
        if (sampled) {
            atomicAdd(&s.tc->sampled, sampled);
            atomicAdd(&s.tc->rel_count, relc);
            atomicAdd(&s.tc->sum_abs, sum_abs);
            atomicAdd(&s.tc->sum_ratio, sum_ratio);
            atomicAdd(&s.tc->sum_rel, sum_rel);
            atomicMax(&s.tc->max_abs_bits, __float_as_uint(max_abs));
            atomicMax(&s.tc->max_ratio_bits, __float_as_uint(max_ratio));
            atomicMax(&s.tc->max_rel_bits, __float_as_uint(max_rel));
        }
    }
}

// Phase 2: the queued pairs, 8 per warp pass: canonical FP32 distance by
// 4-lane groups, the unlocked radius pre-test of both endpoints, then the
// locked inserts (Nhood::parallel_try_insert, kgraph.cpp:723-736) -- the
// CUDA-core join's inner loop, at full occupancy.
__global__ void __launch_bounds__(256) join_insert_kernel(BuildState s, JoinQueue jq) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const unsigned long long total = *jq.tail;
    const unsigned long long w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned long long nw = (gridDim.x * blockDim.x) >> 5;
    InsertTally tally;
    // one contiguous run of entries per warp: a node's pairs share rows
    const unsigned long long chunk = ((total + nw - 1) / nw + 7) & ~7ull;
    const unsigned long long end = min(total, (w0 + 1) * chunk);
    for (unsigned long long base = w0 * chunk; base < end; base += 8) {
        const unsigned long long e = base + g;
        const bool valid = e < end;
        const uint32_t x = valid ? jq.x[e] : 0u, y = valid ? jq.y[e] : 0u, nn = valid ? jq.n[e] : 0u;
        const float dd = pair_dist(s.D, x, y, t, FULL);
        // deferred (the offers to the grouped merge) or locked inserts; the pairs were counted by the filter
        unsigned long long comps = 0;
        bool uu = false;
        settle_pass(s, lane, t, valid, x, y, dd, nn, comps, uu, tally, true);
    }
    if (lane == 0 && tally.attempts) {
        atomicAdd(s.inserts, (unsigned long long)tally.attempts);
        atomicAdd(s.inserts + 1, (unsigned long long)tally.landed);
    }
}

// Upper bound of the pairs node n's join produces: a(a-1)/2 + a*b.
__global__ void join_worst_kernel(BuildState s, uint64_t *worst) {
    for (uint32_t n = blockIdx.x * blockDim.x + threadIdx.x; n <= s.D.n; n += gridDim.x * blockDim.x) {
        uint64_t w = 0;
        if (n < s.D.n) {
            const uint64_t a = min(s.cnt_new[n], s.NEWCAP), b = min(s.cnt_old[n], s.OLDCAP);
            w = a * (a > 0 ? a - 1 : 0) / 2 + a * b;
        }
        worst[n] = w;
    }
}

// Round boundaries: bounds[k] = first node whose exclusive prefix of worst-case
// pairs reaches k * slab (bounds[0] = 0, bounds[R] = N).  A round's pairs are
// then below slab + one node's worst case, which the queue holds.
__global__ void join_bounds_kernel(const uint64_t *pre, uint32_t N, uint64_t slab, uint32_t R, uint32_t *bounds) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k <= R; k += gridDim.x * blockDim.x) {
        uint32_t r;
        if (k == 0) r = 0;
        else if (k == R) r = N;
        else {
            const uint64_t key = (uint64_t)k * slab;
            uint32_t lo = 0, hi = N;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (pre[mid] < key) lo = mid + 1; else hi = mid;
            }
            r = lo;
        }
        bounds[k] = r;
    }
}

size_t join_tc_smem(const BuildState &s, int prec) {
    const size_t Umax = (size_t)s.NEWCAP + s.OLDCAP;
    return 2 * (size_t)TC_M * s.D.ld * (prec ? 1 : 2) + (size_t)s.D.ld * 4 + Umax * 4 * 7;
}

}  // namespace

bool join_tc_supported(const BuildState &s, int prec) {
    return s.D.ld % (prec ? 32 : 16) == 0 && join_tc_smem(s, prec) <= 200 * 1024;
}

uint64_t join_tc_node_max(const BuildState &s) {
    return (uint64_t)s.NEWCAP * (s.NEWCAP - 1) / 2 + (uint64_t)s.NEWCAP * s.OLDCAP;
}

cudaError_t join_tc_worst(cudaStream_t st, const BuildState &s, uint64_t *worst) {
    join_worst_kernel<<<(s.D.n + 256) / 256, 256, 0, st>>>(s, worst);
    return cudaGetLastError();
}

cudaError_t join_tc_bounds(cudaStream_t st, const uint64_t *pre, uint32_t N, uint64_t slab, uint32_t R,
                           uint32_t *bounds) {
    join_bounds_kernel<<<(R + 128) / 128, 128, 0, st>>>(pre, N, slab, R, bounds);
    return cudaGetLastError();
}

cudaError_t launch_join_tc(int num_sms, int grid_insert, cudaStream_t st, const BuildState &s, JoinQueue jq,
                           uint32_t round, int prec) {
    auto kern = prec ? join_tc_kernel<1> : join_tc_kernel<0>;
    size_t smem = join_tc_smem(s, prec);
    if (smem < TC_MIN_SMEM) smem = TC_MIN_SMEM;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    // CTAs per SM from the kernel's registers and shared memory (at most
    // JOIN_TC_MAX_CTAS_PER_SM, which bounds the TMEM columns in use per SM).
    cudaFuncAttributes fa{};
    if ((e = cudaFuncGetAttributes(&fa, kern)) != cudaSuccess) return e;
    int dev = 0, smem_sm = 0, smem_rsv = 0, regs_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    const size_t per_cta_smem = smem + fa.sharedSizeBytes + (size_t)smem_rsv;
    const int regs_cta = ((fa.numRegs + 7) / 8 * 8) * TC_THREADS;
    int occ = JOIN_TC_MAX_CTAS_PER_SM;
    occ = std::min<int>(occ, (int)((size_t)smem_sm / per_cta_smem));
    occ = std::min<int>(occ, regs_cta ? regs_sm / regs_cta : occ);
    if (occ < 1) return cudaErrorInvalidConfiguration;
    cudaMemsetAsync(jq.tail, 0, 8, st);
    cudaMemsetAsync(jq.work, 0, 4, st);
    kern<<<num_sms * occ, TC_THREADS, smem, st>>>(s, s.NEWCAP + s.OLDCAP, jq, round);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cudaFuncSetAttribute(join_insert_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                         (int)cudaSharedmemCarveoutMaxL1);
    join_insert_kernel<<<grid_insert, 256, 0, st>>>(s, jq);
    return cudaGetLastError();
}

}  // namespace kgb
