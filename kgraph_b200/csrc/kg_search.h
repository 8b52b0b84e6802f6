// Launch interface of the batched graph-walk search kernel (kg_search.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "kg_common.cuh"

namespace kgb {

struct SearchArgs {
    DataView D;
    const uint64_t *offsets;    // CSR graph: n+1 offsets
    const uint32_t *nbr;        // neighbour ids
    const uint32_t *Mnode;      // per-node M (KGraphImpl::M)
    const uint32_t *ell;        // optional: the first ell_w neighbours of every node, node-major
    uint32_t ell_w;
    const uint2 *meta;          // optional: per node {M, degree} (saves the offsets loads)
    const float *Q;             // queries, nq rows of q_ld (= D.ld) floats
    uint32_t q_ld, nq;
    const uint32_t *Kq, *Pq;    // optional per-query K and P (null: use K, P)
    uint32_t K, P, Mp, S, T, init;
    float epsilon;
    const uint32_t *seeds;      // concatenated seed lists (T lists of P ids per distinct P)
    const uint32_t *seed_index; // per query: offset of its trial-0 seed list in `seeds`
    const uint32_t *init_ids;   // init > 0: nq rows of out_ld ids
    uint32_t *out_ids;          // nq rows of out_ld
    float *out_dists;           // optional
    uint32_t *out_count;        // nq
    float *out_cost;            // optional, SearchInfo.cost
    uint32_t out_ld;
    uint32_t *visited;          // visited_slots x vwords words
    uint32_t vwords, visited_slots;
    uint32_t *qcounter;         // zeroed before launch
    uint32_t *err;              // device error word
    unsigned long long *work;   // [0] distance evaluations, [1] adjacency entries read, [2] filter
                                //  evaluations on compressed rows, [3] of those skipped (may be null)
    uint32_t prec;              // 0 FP32; 1 BF16, 2 FP8 E4M3 compressed rows filter the walk's candidates
    const void *Xc;             // compressed rows (ld elements each)
    const float4 *cmeta;        // per row {error bound, scale, norm term, 0}
    uint32_t cap, rcap;         // smem capacities: max(K+P+1), max(K+1)
    uint32_t compact_ok;        // the compact pool entry may be used: S >= 1 and every node's expansion
                                //  (actual_M) <= (2^(31 - cp_idbits) - 1) S
    uint32_t cp_idbits;         // compact pool: id bits of a pool word (ids < 2^cp_idbits)
    uint32_t warps_per_block, warp_smem_bytes;   // filled by launch_search
};

// Launch shape of the search kernel: the D-split (lanes per distance, 2/4/8;
// 32/split candidates per pass), the query tile (warps = queries per block,
// 1/2/4/8; 0 = as many as fit, at most 8), the L2 prefetch depth (0 or 2
// neighbour batches), the register budget per thread (64; 80 for the FP32
// walk; 56 for the compact FP32 walk in blocks of at most 4 warps; 0 = 64)
// and the pool entry (compact = 1: 8 bytes instead of 12, FP32 walk only,
// where SearchArgs::compact_ok).  Every shape computes the same bits.
struct SearchShape {
    uint32_t split = 4, warps_per_block = 0, prefetch = 2, regs = 64, compact = 1;
};
bool search_shape_valid(const SearchShape &sh);
// Whether a launch of shape sh with arguments a runs the compact pool entry.
bool search_uses_compact(const SearchArgs &a, const SearchShape &sh);

size_t search_warp_smem_bytes(uint32_t ld, uint32_t cap, uint32_t rcap, bool compact = false);
// Upper bound of concurrently resident warps (= visited slots needed).
uint32_t search_max_slots(const SearchArgs &a, const SearchShape &sh, int num_sms);
cudaError_t launch_search(SearchArgs &a, const SearchShape &sh, int num_sms, cudaStream_t st, uint32_t *grid_out);
// Filter lower bounds and canonical distances of `per` rows (ids) per query of a.Q
// (rows of a.q_ld floats, a.D.ld <= 256), with the compressed rows of a.prec.
cudaError_t launch_filter_bounds(const SearchArgs &a, const uint32_t *ids, uint32_t per, float *lb, float *dist,
                                 cudaStream_t st);

}  // namespace kgb
