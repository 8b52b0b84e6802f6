// Warp-cooperative primitives over sorted (dist, id) lists held in shared or
// global memory: the sorted insert with the reference's duplicate rule, and
// the next-flagged scan of the search walk.
#pragma once
#include "kg_common.cuh"

namespace kgb {

constexpr unsigned FULL = 0xFFFFFFFFu;

// Number of entries in the sorted prefix pd[0, L) with pd[j] <= d, i.e. the
// position UpdateKnnListHelper (kgraph.cpp:180-185) inserts at: after every
// entry of equal distance.  Two probe rounds: 32 evenly spaced probes locate
// the segment, then the segment is counted 32 at a time.
template <typename P>
__device__ __forceinline__ uint32_t warp_upper_bound(P pd, uint32_t L, float d, int lane) {
    if (L == 0) return 0;
    const uint32_t seg = (L + 31) >> 5;
    const uint32_t probe = (uint32_t)lane * seg;
    bool le = probe < L && pd[probe] <= d;
    uint32_t c = __popc(__ballot_sync(FULL, le));
    if (c == 0) return 0;
    uint32_t lo = (c - 1) * seg + 1;
    uint32_t hi = min(c * seg, L);
    uint32_t i = lo;
    for (uint32_t base = lo; base < hi; base += 32) {
        uint32_t j = base + lane;
        bool b = j < hi && pd[j] <= d;
        i += __popc(__ballot_sync(FULL, b));
    }
    return i;
}

// True when an entry with distance == d and id == id (flag bit ignored) sits
// in the run of equal distances that ends at position i-1 (kgraph.cpp:187-193).
template <typename P, typename I>
__device__ __forceinline__ bool warp_dup_before(P pd, I pid, uint32_t i, float d, uint32_t id, int lane) {
    for (int base = (int)i - 32;; base -= 32) {
        int j = base + lane;
        bool eq = j >= 0 && j < (int)i && pd[j] == d;
        bool hit = eq && ((pid[j] & ID_MASK) == (id & ID_MASK));
        if (__any_sync(FULL, hit)) return true;
        // The run continues below this chunk only if the chunk's first entry is still equal.
        bool cont = base > 0 && pd[base] == d;
        if (!__shfl_sync(FULL, cont, 0)) return false;
    }
}

// UpdateKnnListHelper (kgraph.cpp:176-202) by one warp over parallel arrays
// pd/pid/(pm) holding a sorted list of length L with room for entry L.
// Returns the insert position, L + 1 for a duplicate.  pm may be null.
template <typename PD, typename PI>
__device__ __forceinline__ uint32_t warp_update_knn(PD pd, PI pid, uint32_t *pm, uint32_t L, float d,
                                                    uint32_t idf, uint32_t mv, int lane) {
    uint32_t i = warp_upper_bound(pd, L, d, lane);
    if (warp_dup_before(pd, pid, i, d, idf, lane)) return L + 1;
    for (int top = (int)L - 1; top >= (int)i; top -= 32) {
        int j = top - lane;
        float dv = 0.f;
        uint32_t iv = 0, mvv = 0;
        bool act = j >= (int)i;
        if (act) { dv = pd[j]; iv = pid[j]; if (pm) mvv = pm[j]; }
        __syncwarp();
        if (act) { pd[j + 1] = dv; pid[j + 1] = iv; if (pm) pm[j + 1] = mvv; }
        __syncwarp();
    }
    if (lane == 0) { pd[i] = d; pid[i] = idf; if (pm) pm[i] = mv; }
    __syncwarp();
    return i;
}

// n successive UpdateKnnList calls (kgraph.cpp:503-512) by one warp in one
// pass.  The candidates are the lanes set in `mask`, in lane order; each such
// lane holds its candidate's distance di, id-with-flag idf and m|M word pmv
// (ignored when pm is null: a pool without m|M words).
// They are inserted in order into the sorted pool pd/pid/pm of length L whose
// capacity is cap (slot cap-1 is the overflow slot), L growing by one per
// candidate up to cap-1.  Their ids are distinct and absent from the pool (the
// caller's visited set guarantees it), so the duplicate rule never fires.
// Sequential inserts with insert-after-equals and eviction of the last entry
// produce exactly the stable merge of the pool with the candidates ordered by
// (distance, order), truncated to the final length; candidate i's position at
// the moment it is inserted is a_i + #{j < i : d_j <= d_i}, a_i = #pool
// entries <= d_i.  Returns the new L; *min_rank receives the smallest insertion
// position among candidates that entered the list (r < L after the increment),
// or 0xFFFFFFFF.
__device__ __forceinline__ uint32_t warp_batch_insert(float *pd, uint32_t *pid, uint32_t *pm, uint32_t L,
                                                      uint32_t cap, unsigned mask, float di, uint32_t idf,
                                                      uint32_t pmv, uint32_t *min_rank, int lane) {
    const uint32_t n = __popc(mask);
    const bool me = (mask >> lane) & 1u;
    const uint32_t my = __popc(mask & ((1u << lane) - 1u));   // this lane's candidate index
    uint32_t ai = 0;
    if (me) {   // upper bound of di in pd[0, L)
        uint32_t lo = 0, hi = L;
        while (lo < hi) {
            uint32_t mid = (lo + hi) >> 1;
            if (pd[mid] <= di) lo = mid + 1; else hi = mid;
        }
        ai = lo;
    }
    uint32_t e = 0, f = 0, mina = me ? ai : 0xFFFFFFFFu;
    for (unsigned rest = mask; rest; rest &= rest - 1) {
        const int src = __ffs(rest) - 1;
        const float dj = __shfl_sync(FULL, di, src);
        const uint32_t j = __popc(mask & ((1u << src) - 1u));
        if (j < my && dj <= di) ++e;
        if (dj < di || (dj == di && j < my)) ++f;
    }
    const uint32_t r = ai + e;   // position when this candidate is inserted
    const bool ins = me && r < min(L + my + 1, cap - 1);
    uint32_t mr = ins ? r : 0xFFFFFFFFu;
    for (int o = 16; o; o >>= 1) {
        mr = min(mr, __shfl_xor_sync(FULL, mr, o));
        mina = min(mina, __shfl_xor_sync(FULL, mina, o));
    }
    *min_rank = mr;
    const uint32_t Lf = min(L + n, cap - 1);
    // move pool entries q >= mina up by #{j : a_j <= q}, top-down (each chunk's
    // loads precede the next chunk's stores, which reach at most this chunk).
    // For the chunk [top - 31, top]: the candidates with a_j <= top - 31 count
    // for every lane (one ballot); only those with a_j inside the chunk are
    // compared lane by lane.
    for (int top = (int)L - 1; top >= (int)mina; top -= 32) {
        const int q = top - lane;
        const bool act = q >= (int)mina;
        float dv = 0.f;
        uint32_t iv = 0, mv = 0;
        if (act) { dv = pd[q]; iv = pid[q]; if (pm) mv = pm[q]; }
        const int bot = top - 31;
        const unsigned below = __ballot_sync(FULL, me && (int)ai <= bot);
        uint32_t sh = __popc(below);
        for (unsigned rest = __ballot_sync(FULL, me && (int)ai > bot && (int)ai <= top); rest; rest &= rest - 1)
            sh += (__shfl_sync(FULL, ai, __ffs(rest) - 1) <= (uint32_t)q) ? 1u : 0u;
        __syncwarp();
        if (act && (uint32_t)q + sh < Lf) { pd[q + sh] = dv; pid[q + sh] = iv; if (pm) pm[q + sh] = mv; }
    }
    __syncwarp();
    const uint32_t fpos = ai + f;
    if (me && fpos < Lf) { pd[fpos] = di; pid[fpos] = idf; if (pm) pm[fpos] = pmv; }
    __syncwarp();
    return Lf;
}

// First index >= k in [0, L) whose flag bit is set; L if none.
__device__ __forceinline__ uint32_t warp_next_flagged(const uint32_t *pid, uint32_t k, uint32_t L, int lane) {
    for (uint32_t base = k; base < L; base += 32) {
        uint32_t j = base + lane;
        bool f = j < L && (pid[j] & FLAG_BIT);
        unsigned m = __ballot_sync(FULL, f);
        if (m) return base + __ffs(m) - 1;
    }
    return L;
}

}  // namespace kgb
