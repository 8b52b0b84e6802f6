// Library context: one GPU, one stream, the dataset and the graph in HBM.
#pragma once
#include <algorithm>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>
#include <cuda_runtime.h>
#include "kg_common.cuh"
#include "kg_search.h"
#include "../../include/kgraph_b200.h"

namespace kgb {

struct RouterState;
void router_release(RouterState *r);

// A device buffer that only grows.
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    cudaError_t reserve(size_t b) {
        if (b <= bytes) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        size_t nb = b < 256 ? 256 : b;
        cudaError_t e = cudaMalloc(&p, nb);
        if (e == cudaSuccess) bytes = nb;
        return e;
    }
    void release() { if (p) cudaFree(p); p = nullptr; bytes = 0; }
    template <typename T> T *as() const { return reinterpret_cast<T *>(p); }
};

struct Error {
    int code;
    std::string msg;
};

}  // namespace kgb

struct kg_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::mutex mu;
    std::string err;
    float last_build_ms = 0.f, last_search_ms = 0.f, last_router_ms = 0.f;
    unsigned last_build_graph_launches = 0;   // CUDA graph launches of the last build's iterations
    unsigned long long last_build_work[3] = {0, 0, 0};   // join pairs, join list entries, iterations
    std::vector<kg_build_iteration> last_build_iters;    // per-iteration counters and device time
    unsigned long long last_work[4] = {0, 0, 0, 0};   // evaluations, adjacency reads, filter: approx, skipped

    // dataset
    kgb::DevBuf X, norms;
    uint32_t n = 0, d = 0, ld = 0;
    int metric = 0;
    bool has_data = false;
    uint64_t data_version = 0;       // bumped whenever the dataset changes

    // reduced-precision copy for the search's distance filter (kg_precision.cu)
    int search_prec = KG_SEARCH_FP32, prec_built = KG_SEARCH_FP32;
    uint64_t prec_data_version = ~0ull;
    kgb::DevBuf Xc, cmeta, cstats;
    double prec_max_rel = 0.0, prec_mean_rel = 0.0;

    // graph, CSR
    kgb::DevBuf offsets, nbr, nbr_d, Mnode;
    uint64_t E = 0;
    uint32_t gn = 0;
    bool has_graph = false;
    bool no_dist = false;
    uint64_t graph_version = 0;      // bumped whenever the graph changes

    // search-side copy of the graph: ELL rows of the first ell_w neighbours + {M, degree}
    kgb::DevBuf ell, meta;
    uint32_t ell_w = 0;
    uint32_t max_degree = 0, max_mdeg = 0;   // largest degree and largest min(M, degree) of the graph
    kgb::SearchShape search_shape;   // launch shape of the search kernel (kg_search_autotune)
    kgb::SearchShape last_shape;     // the shape the last kg_search_batch launched (kg_last_search_shape)
    uint64_t layout_version = ~0ull;

    // scratch
    kgb::DevBuf errw, counter, visited, qbuf, kbuf, pbuf, seeds, seed_index, init_ids, out_ids, out_d,
        out_cnt, out_cost;
    std::vector<uint32_t> h_stage_u32;

    kgb::DevBuf build_scratch[25];   // NN-descent state (kg_build.cu)
    kgb::DevBuf rev_scratch[17];     // reverse-edge completion work space (kg_graph.cu), kept between builds
    int join_mode = KG_JOIN_AUTO;
    kgb::DevBuf tcstat;              // tensor-core join counters
    kgb::DevBuf joinq, joinaux, joinb;   // tensor-core join: candidate queue, worst-case prefix, round bounds
    kgb::DevBuf offer_lin, offer_grp, offer_aux, offer_scan;   // deferred join inserts (kg_build.cu)
    int join_inserts = KG_INSERTS_AUTO;
    size_t offer_cap = 0;             // record-buffer capacity of deferred inserts, in offers (0: automatic)
    bool join_tile = true;            // FP32 join with each node's lists staged in shared memory
    kg_join_stats last_join{};
    // tensor-core brute force (kg_bruteforce.cu): BF16 centred rows, row terms, mean + extents, work space
    kgb::DevBuf bf_rows, bf_meta, bf_aux, bf_work;
    uint64_t bf_data_version = ~0ull;
    float bf_ext[5] = {0, 0, 0, 0, 0};
    int bf_mode = KG_BRUTEFORCE_AUTO;
    unsigned long long *bf_stats_dev = nullptr;
    kg_bruteforce_stats last_bf{};
    kgb::RouterState *router = nullptr;   // learned entry router (kg_router.cu)
    void *noalloc_scratch = nullptr;      // device address of kg_search_batch_noalloc's static array
    kgb::DevBuf rseeds;                   // router seeds handed to the search (kg_router_search)
};

namespace kgb {

// Helpers shared by the entry-point files.
int set_error(kg_ctx *ctx, int code, const std::string &msg);
int cuda_fail(kg_ctx *ctx, cudaError_t e, const char *what);
bool is_device_ptr(const void *p);
// Reads and clears the device error word; returns KG_OK or sets the message.
int check_device_error(kg_ctx *ctx, const char *what);
// kg_search_batch with the context lock held (kg_ctx.cu); init_dev, when not
// null, holds the starting points (device rows of init_ld ids).
int search_locked(kg_ctx *ctx, const float *queries, size_t nq, size_t q_stride_bytes,
                  const kg_search_params *params, const uint32_t *K_per_q, const uint32_t *P_per_q, size_t out_ld,
                  uint32_t *ids, float *dists, uint32_t *counts, float *costs, const SearchShape &sh,
                  const uint32_t *init_dev, size_t init_ld);
// The id bits of a compact pool word for N nodes (ids 0 .. N-1).
inline uint32_t compact_id_bits(uint32_t N) {
    uint32_t b = 1;
    while (b < 31 && (N - 1) >> b) ++b;
    return b;
}
// Whether the search may use the compact 8-byte pool entry on the current
// graph (its search layout built): S >= 1 and every node's expansion,
// min(max(M, Mp), degree), at most 2^(31 - id bits) - 1 batches of S.
inline uint32_t compact_pool_ok(const kg_ctx *ctx, uint32_t N, uint32_t S, uint32_t Mp) {
    if (ctx->layout_version != ctx->graph_version || S == 0 || N == 0) return 0;
    const uint32_t pbits = 31 - compact_id_bits(N);
    // min(max(M_i, Mp), deg_i) <= max(min(M_i, deg_i), min(Mp, deg_i))
    const uint64_t em = std::max<uint64_t>(ctx->max_mdeg, std::min<uint64_t>(Mp, ctx->max_degree));
    return pbits >= 1 && em <= ((1ull << pbits) - 1) * S ? 1u : 0u;
}
// Builds the compressed rows of ctx->search_prec if the dataset changed since.
int ensure_search_precision(kg_ctx *ctx);
// Exact top-K brute force of `nq` dataset rows (LinearSearch, kgraph.cpp:212-229)
// used for the build's control nodes.
cudaError_t launch_linear_search(kg_ctx *ctx, const uint32_t *rows, uint32_t nq, uint32_t K, uint32_t *out_ids,
                                 float *out_d);

}  // namespace kgb
