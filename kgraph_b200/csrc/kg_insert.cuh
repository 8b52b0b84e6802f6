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

// Counts of one warp's inserts: attempts (offers that passed the unlocked
// radius test and took the lock) and landed (entered the list: not a
// duplicate), warp-uniform.
struct InsertTally {
    uint32_t attempts = 0, landed = 0;   // per warp and launch: far below 2^32
};

// Nhood::parallel_try_insert (kgraph.cpp:723-736) by one warp, for an offer
// that already passed the reference's unlocked radius test (`dist > radius`,
// kgraph.cpp:724): the callers read the radii of a whole batch of pairs at once
// and call this only for the offers that pass.  Returns the reference's value:
// L+1 for a duplicate, else the insert position.  The lock is taken with an
// acquire CAS and released with a release store by lane 0; the warp barriers
// order the other lanes' pool accesses inside that critical section.  Latency:
// the lock, then ONE round trip for the node's L and its whole pool row (every
// slot is loaded, the ones at or past L masked in registers), then stores only
// -- the new last entry that sets the radius of a full pool comes from the
// registers, not from a reload.
__device__ __forceinline__ uint32_t locked_insert(const BuildState &s, uint32_t x, uint32_t y, float d, int lane,
                                                  InsertTally &tally) {
    uint32_t ok = 1;
    if (lane == 0) {
        long long t0 = clock64();
        while (cas_acquire(s.lock + x, 0u, 1u) != 0u) {
            if (clock64() - t0 > LOCK_LIMIT_CYCLES) { ok = 0; raise_error(s.err, ERR_LOCK_TIMEOUT); break; }
            __nanosleep(32);
        }
    }
    ok = __shfl_sync(FULL, ok, 0);
    if (!ok) return s.Lp;
    volatile float *pd = s.pool_d + (size_t)x * s.PS;
    volatile uint32_t *pi = s.pool_i + (size_t)x * s.PS;
    const uint32_t idf = y | FLAG_BIT;
    uint32_t r, Lc;
    float last = 0.f;   // pool[Lc - 1] after the insert (valid when r <= Lc and Lc >= 1)
    if (s.L <= 128) {
        // L and the row in flight together: slots [0, min(PS, 128))
        uint32_t Lraw = lane == 0 ? *reinterpret_cast<volatile uint32_t *>(s.nodeL + x) : 0u;
        float v[4];
        uint32_t w[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t j = lane + 32 * k;
            v[k] = FLT_MAX;
            w[k] = 0;
            if (j < s.PS && j < 128) { v[k] = pd[j]; w[k] = pi[j]; }
        }
        Lc = __shfl_sync(FULL, Lraw, 0);
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (lane + 32 * k >= Lc) v[k] = FLT_MAX;
        // UpdateKnnListHelper (kgraph.cpp:176-202) on the register-resident row
        uint32_t i = 0;   // entries with distance <= d: insert after all of them
#pragma unroll
        for (int k = 0; k < 4; ++k) i += __popc(__ballot_sync(FULL, lane + 32 * k < Lc && v[k] <= d));
        bool dup = false;   // the same id in the run of equal distances before i (kgraph.cpp:187-193)
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t j = lane + 32 * k;
            dup |= j < i && v[k] == d && ((w[k] & ID_MASK) == (idf & ID_MASK));
        }
        if (__any_sync(FULL, dup)) {
            r = Lc + 1;
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const uint32_t j = lane + 32 * k;
                if (j >= i && j < Lc) { pd[j + 1] = v[k]; pi[j + 1] = w[k]; }
            }
            if (lane == (int)(i & 31)) { pd[i] = d; pi[i] = idf; }
            r = i;
            if (Lc >= 1) {   // new pool[Lc - 1]: d itself, the entry shifted into it, or the old one
                const uint32_t src = (i == Lc - 1) ? 0xFFFFFFFFu : (i < Lc - 1 ? Lc - 2 : Lc - 1);
                const uint32_t sl = src == 0xFFFFFFFFu ? 0u : src;
                float cand = FLT_MAX;
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    if (sl / 32 == (uint32_t)k) cand = __shfl_sync(FULL, v[k], (int)(sl & 31));
                last = src == 0xFFFFFFFFu ? d : cand;
            }
        }
    } else {
        Lc = lane == 0 ? *reinterpret_cast<volatile uint32_t *>(s.nodeL + x) : 0u;
        Lc = __shfl_sync(FULL, Lc, 0);
        r = warp_update_knn(pd, pi, (uint32_t *)nullptr, Lc, d, idf, 0u, lane);
        __syncwarp();
        if (r <= Lc && Lc >= 1) last = pd[Lc - 1];   // after the shift
    }
    __syncwarp();
    ++tally.attempts;
    if (r <= Lc) ++tally.landed;
    if (lane == 0 && r <= Lc) {
        if (Lc + 1 < s.Lp) *reinterpret_cast<volatile uint32_t *>(s.nodeL + x) = Lc + 1;
        else *reinterpret_cast<volatile float *>(s.radius + x) = last;
    }
    if (lane == 0) store_release(s.lock + x, 0u);
    return r;
}

}  // namespace kgb
