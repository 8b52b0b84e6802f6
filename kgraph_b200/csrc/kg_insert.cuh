// The per-node locked pool insert shared by both local-join kernels.
#pragma once
#include "kg_build.h"
#include "kg_warp.cuh"

namespace kgb {

constexpr long long LOCK_LIMIT_CYCLES = 4000000000ll;   // ~2 s at 2 GHz, then an error is reported

__device__ __forceinline__ uint32_t cas_acquire(uint32_t *p, uint32_t cmp, uint32_t val) {
    uint32_t old;
    asm volatile("atom.acquire.gpu.global.cas.b32 %0, [%1], %2, %3;" : "=r"(old) : "l"(p), "r"(cmp), "r"(val) : "memory");
    return old;
}
__device__ __forceinline__ void store_release(uint32_t *p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// UpdateKnnListHelper (kgraph.cpp:176-202) on a pool row of Lc <= 128 sorted
// entries with the row held in registers: entry j lives in lane j % 32, slot
// j / 32.  One coalesced read of the row, the position and the duplicate test
// by ballots, one pass of writes.  Same results as warp_update_knn.
__device__ __forceinline__ uint32_t update_knn_regs(volatile float *pd, volatile uint32_t *pi, uint32_t Lc,
                                                    float d, uint32_t idf, int lane) {
    float v[4];
    uint32_t w[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t j = lane + 32 * k;
        v[k] = FLT_MAX;
        w[k] = 0;
        if (j < Lc) { v[k] = pd[j]; w[k] = pi[j]; }
    }
    uint32_t i = 0;   // entries with distance <= d: insert after all of them
#pragma unroll
    for (int k = 0; k < 4; ++k) i += __popc(__ballot_sync(FULL, lane + 32 * k < Lc && v[k] <= d));
    bool dup = false;   // the same id in the run of equal distances before i (kgraph.cpp:187-193)
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t j = lane + 32 * k;
        dup |= j < i && v[k] == d && ((w[k] & ID_MASK) == (idf & ID_MASK));
    }
    if (__any_sync(FULL, dup)) return Lc + 1;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t j = lane + 32 * k;
        if (j >= i && j < Lc) { pd[j + 1] = v[k]; pi[j + 1] = w[k]; }
    }
    if (lane == (int)(i & 31)) { pd[i] = d; pi[i] = idf; }
    return i;
}

// Counts of one warp's inserts: attempts (offers that passed the unlocked
// radius test and took the lock) and landed (entered the list: not a
// duplicate), warp-uniform.
struct InsertTally {
    unsigned long long attempts = 0, landed = 0;
};

// Nhood::parallel_try_insert (kgraph.cpp:723-736) by one warp.  Returns the
// reference's value: pool.size() when the radius test rejects, L+1 for a
// duplicate, else the insert position.  The lock is taken with an acquire
// CAS and released with a release store by lane 0; the warp barriers order
// the other lanes' pool accesses inside that critical section.
__device__ __forceinline__ uint32_t locked_insert(const BuildState &s, uint32_t x, uint32_t y, float d, int lane,
                                                  InsertTally &tally) {
    float rad = 0.f;
    uint32_t Lc = 0;
    if (lane == 0) rad = *reinterpret_cast<volatile float *>(s.radius + x);
    rad = __shfl_sync(FULL, rad, 0);   // one read, the same decision in every lane
    if (d > rad) return s.Lp;
    uint32_t ok = 1;
    if (lane == 0) {
        long long t0 = clock64();
        while (cas_acquire(s.lock + x, 0u, 1u) != 0u) {
            if (clock64() - t0 > LOCK_LIMIT_CYCLES) { ok = 0; raise_error(s.err, ERR_LOCK_TIMEOUT); break; }
            __nanosleep(32);
        }
        if (ok) Lc = *reinterpret_cast<volatile uint32_t *>(s.nodeL + x);
    }
    ok = __shfl_sync(FULL, ok, 0);
    if (!ok) return s.Lp;
    Lc = __shfl_sync(FULL, Lc, 0);
    __syncwarp();
    volatile float *pd = s.pool_d + (size_t)x * s.PS;
    volatile uint32_t *pi = s.pool_i + (size_t)x * s.PS;
    uint32_t r;
    if (s.L <= 128) {
        r = update_knn_regs(pd, pi, Lc, d, y | FLAG_BIT, lane);
    } else {
        r = warp_update_knn(pd, pi, (uint32_t *)nullptr, Lc, d, y | FLAG_BIT, 0u, lane);
    }
    __syncwarp();
    ++tally.attempts;
    if (r <= Lc) ++tally.landed;
    if (lane == 0 && r <= Lc) {
        if (Lc + 1 < s.Lp) *reinterpret_cast<volatile uint32_t *>(s.nodeL + x) = Lc + 1;
        else *reinterpret_cast<volatile float *>(s.radius + x) = pd[Lc - 1];   // after the shift
    }
    if (lane == 0) store_release(s.lock + x, 0u);
    return r;
}

// One pass of 8 pairs (one per 4-lane group: lanes 4p..4p+3 hold pair p's
// x, y and distance, valid marking a pair to evaluate, n the node whose join
// made it): the unlocked radius pre-test for both directions
// (kgraph.cpp:725), then Nhood::parallel_try_insert of the offers that passed
// -- recorded for the deferred merge while the record buffer has room, else
// under the target's lock here.  A locked x <- y insert that lands below K
// (kgraph.cpp:808-810) sets uu, or with set_found the found flag of its pair's
// node directly; comps counts the pairs (the reference's cc).
__device__ __forceinline__ void settle_pass(const BuildState &s, int lane, int t, bool valid, uint32_t x, uint32_t y,
                                            float dd, uint32_t n, unsigned long long &comps, bool &uu,
                                            InsertTally &tally, bool set_found = false) {
    const float rx = (valid && t == 0) ? *reinterpret_cast<volatile float *>(s.radius + x) : 0.f;
    const float ry = (valid && t == 1) ? *reinterpret_cast<volatile float *>(s.radius + y) : 0.f;
    const unsigned vm_all = __ballot_sync(FULL, valid && t == 0);
    unsigned nx = __ballot_sync(FULL, valid && t == 0 && !(dd > rx));
    unsigned ny = __ballot_sync(FULL, valid && t == 1 && !(dd > ry));
    comps += __popc(vm_all);
    if (s.off_lin && (nx | ny)) {
        // deferred: the offers go to the grouped merge after the join (one
        // cursor atomic per pass); those beyond the buffer's capacity are
        // inserted here under the lock
        const unsigned om = nx | ny;
        unsigned long long b0 = 0;
        if (lane == 0) b0 = atomicAdd(s.off_cursor, (unsigned long long)__popc(om));
        b0 = __shfl_sync(FULL, b0, 0);
        const unsigned long long fit = b0 >= s.off_cap ? 0ull : s.off_cap - b0;
        const uint32_t rank = __popc(om & ((1u << lane) - 1u));
        const bool mine = ((om >> lane) & 1u) && rank < fit;
        if (mine) {
            const uint32_t tg = t == 0 ? x : y;
            s.off_lin[b0 + rank] = make_uint4(tg, t == 0 ? y : x, __float_as_uint(dd), n | (t == 0 ? OFFER_UU : 0u));
            atomicAdd(s.off_cnt + tg, 1u);
        }
        const unsigned dm = __ballot_sync(FULL, mine);
        nx &= ~dm;
        ny &= ~dm;
    }
    // only the pairs with an offer that passed a radius test: a pair both endpoints reject
    // inserts nothing and leaves r at pool.size() (>= K)
    unsigned vm = nx | (ny >> 1);
    while (vm) {
        const int src = __ffs(vm) - 1;
        vm &= vm - 1;
        const uint32_t xg = __shfl_sync(FULL, x, src), yg = __shfl_sync(FULL, y, src);
        const float dg = __shfl_sync(FULL, dd, src);
        const uint32_t ng = __shfl_sync(FULL, n, src);
        uint32_t r = s.Lp;
        if (nx & (1u << src)) r = locked_insert(s, xg, yg, dg, lane, tally);
        if (r < s.K) {
            if (!set_found) uu = true;
            else if (lane == 0) s.found[ng] = 1u;
        }
        if (ny & (1u << (src + 1))) locked_insert(s, yg, xg, dg, lane, tally);
    }
}

}  // namespace kgb
