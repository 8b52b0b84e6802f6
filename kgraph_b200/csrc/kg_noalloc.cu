// kg_search_batch_noalloc: the batched graph-walk search without any device
// allocation.
//
// Who needs it.  Some callers cannot call cudaMalloc at search time: a
// serving thread that must never block on the allocator (cudaMalloc can
// synchronise the device), an application that hands out all GPU memory up
// front through its own pool and forbids libraries to allocate behind its
// back, or an embedding that runs under a fixed memory budget.  kg_search_batch
// grows per-context device buffers on demand (query staging, seed table,
// per-warp visited sets); this entry point allocates nothing.
//
// How.  Its scratch -- the query counter, error word and work counters, the
// seed table, the per-query seed index and the per-warp visited sets -- lives
// in one file-scope static __device__ array of KG_NOALLOC_SCRATCH_BYTES that
// every GPU loading the library holds until the process exits.  Host code
// cannot use the array's name as a device address (it is a host-side stand-in),
// so the first call through a context resolves the address on the context's
// device with cudaGetSymbolAddress while that device is current, and keeps it
// in the context.  That first call should therefore come before any stream
// capture.  Keeping the address per context (not per process) means a context
// created after a device reset looks it up again; a context that outlives a
// reset is unusable anyway, since its dataset and graph buffers are gone.  The
// dataset and graph are the context's (kg_set_data / kg_build /
// kg_graph_import allocate as usual, beforehand); queries and outputs are the
// caller's DEVICE buffers.  When an earlier kg_search_batch has already built
// the context's search-side copy of the graph or the compressed rows of its
// distance filter, this entry point uses them too (same results, faster);
// otherwise it walks the CSR graph in FP32 and builds nothing.
//
// Limits.  The whole scratch is shared by every call in the process: calls
// whose kernels overlap on the GPU race on it, so callers serialise them (one
// stream, or events).  Each call zeroes the counters it needs first; the
// visited sets are cleared per query by the kernel.  Fewer visited sets fit than
// kg_search_batch would use when N is large, so large-N batches run on fewer
// resident warps (the same results, lower throughput).
#include <algorithm>
#include <ctime>
#include <mutex>
#include <random>
#include "kg_ctx.h"
#include "kg_search.h"

namespace kgb {
void gen_random(std::mt19937 &rng, uint32_t *addr, uint32_t size, uint32_t N);
}

using namespace kgb;

namespace {

constexpr size_t SCRATCH_BYTES = KG_NOALLOC_SCRATCH_BYTES;
constexpr size_t HEADER_BYTES = 256;   // counter (4), error word (4), work counters (16)
static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

// Device address of the static scratch on the context's device (which the
// caller has made current), looked up once per context.
cudaError_t scratch_address(kg_ctx *ctx, unsigned char **out) {
    if (!ctx->noalloc_scratch) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        ctx->noalloc_scratch = p;
    }
    *out = static_cast<unsigned char *>(ctx->noalloc_scratch);
    return cudaSuccess;
}

}  // namespace

extern "C" size_t kg_noalloc_scratch_bytes(void) { return SCRATCH_BYTES; }

extern "C" int kg_search_batch_noalloc(kg_ctx *ctx, const float *queries, size_t nq, size_t q_stride_bytes,
                                       const kg_search_params *params, size_t out_ld, uint32_t *ids, float *dists,
                                       uint32_t *counts, float *costs) {
    if (!ctx) return KG_E_INVALID;
    std::lock_guard<std::mutex> lk(ctx->mu);
    cudaSetDevice(ctx->device);
    if (!ctx->has_data) return set_error(ctx, KG_E_RUNTIME, "no dataset");
    if (!params || !ids || !counts || (nq && !queries)) return set_error(ctx, KG_E_INVALID, "bad arguments");
    if (nq == 0) return KG_OK;
    const bool graph = ctx->has_graph;
    const uint32_t N = graph ? ctx->gn : ctx->n;
    const uint32_t ld = ctx->ld;
    if (graph && ctx->gn > ctx->n) return set_error(ctx, KG_E_RUNTIME, "dataset larger than index");
    if (params->init && params->T > 1) return set_error(ctx, KG_E_RUNTIME, "when init > 0, T must be 1.");
    if (params->K > out_ld || params->init > out_ld) return set_error(ctx, KG_E_INVALID, "out_ld smaller than K");
    // Everything the kernel touches must already be on the device.
    if (!is_device_ptr(queries) || !is_device_ptr(ids) || !is_device_ptr(counts) || (dists && !is_device_ptr(dists)) ||
        (costs && !is_device_ptr(costs)))
        return set_error(ctx, KG_E_INVALID, "kg_search_batch_noalloc needs device buffers for queries and outputs");
    if (q_stride_bytes != (size_t)ld * sizeof(float) || (reinterpret_cast<uintptr_t>(queries) & 15))
        return set_error(ctx, KG_E_INVALID,
                         "kg_search_batch_noalloc needs 16-byte aligned query rows padded to a multiple of 16 floats");

    unsigned char *base = nullptr;
    cudaError_t e = scratch_address(ctx, &base);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "noalloc scratch address");

    // Layout inside the static array.
    const bool walk = graph && params->P < N;
    const uint32_t T = params->T ? params->T : 1;
    const size_t seed_words = walk && params->init == 0 ? (size_t)T * params->P : 1;
    size_t off = HEADER_BYTES;
    uint32_t *seeds = reinterpret_cast<uint32_t *>(base + off);
    off += (seed_words * 4 + 255) / 256 * 256;
    uint32_t *seed_index = reinterpret_cast<uint32_t *>(base + off);
    off += (nq * 4 + 255) / 256 * 256;
    if (off >= SCRATCH_BYTES)
        return set_error(ctx, KG_E_INVALID, "kg_search_batch_noalloc: P*T seeds and nq queries exceed the " +
                                                 std::to_string(SCRATCH_BYTES >> 20) + " MiB scratch");

    SearchArgs a{};
    a.D = DataView{ctx->X.as<float>(), ctx->norms.as<float>(), N, ctx->d, ld, ctx->metric};
    a.offsets = graph ? ctx->offsets.as<uint64_t>() : nullptr;
    a.nbr = graph ? ctx->nbr.as<uint32_t>() : nullptr;
    a.Mnode = graph ? ctx->Mnode.as<uint32_t>() : nullptr;
    if (graph && ctx->layout_version == ctx->graph_version && ctx->ell.p) {   // already built: reuse, build nothing
        a.ell = ctx->ell.as<uint32_t>();
        a.ell_w = ctx->ell_w;
        a.meta = ctx->meta.as<uint2>();
        a.compact_ok = compact_pool_ok(ctx, N, params->S, params->M);
        a.cp_idbits = compact_id_bits(N);
    }
    if (graph && ctx->search_prec != KG_SEARCH_FP32 && ctx->prec_built == ctx->search_prec &&
        ctx->prec_data_version == ctx->data_version) {
        a.prec = (uint32_t)ctx->search_prec;
        a.Xc = ctx->Xc.p;
        a.cmeta = ctx->cmeta.as<float4>();
    }
    a.Q = queries;
    a.q_ld = ld;
    a.nq = (uint32_t)nq;
    a.K = params->K; a.P = graph ? params->P : N; a.Mp = params->M; a.S = params->S; a.T = params->T;
    a.init = graph ? params->init : 0u;
    a.epsilon = params->epsilon;
    a.seeds = seeds;
    a.seed_index = seed_index;
    a.init_ids = a.init ? ids : nullptr;   // each warp reads its row's starting points before writing results
    a.out_ids = ids;
    a.out_dists = dists;
    a.out_count = counts;
    a.out_cost = costs;
    a.out_ld = (uint32_t)out_ld;
    a.cap = walk ? params->K + params->P + 1 : params->K + 1;
    a.rcap = params->K + 1;
    if (search_warp_smem_bytes(ld, a.cap, a.rcap) > 200 * 1024)
        return set_error(ctx, KG_E_INVALID, "K + P too large for one query's shared-memory pool");
    a.qcounter = reinterpret_cast<uint32_t *>(base);
    a.err = reinterpret_cast<uint32_t *>(base + 4);
    a.work = reinterpret_cast<unsigned long long *>(base + 8);

    // Visited sets: as many as fit in what is left, at least one SM's worth of warps.
    a.vwords = ((N + 31) / 32 + 3) / 4 * 4;
    const size_t per_slot = (size_t)a.vwords * 4;
    const size_t fit = (SCRATCH_BYTES - off) / per_slot;
    const uint32_t per_sm_slots = search_max_slots(a, ctx->search_shape, 1);
    if (fit < per_sm_slots)
        return set_error(ctx, KG_E_INVALID, "kg_search_batch_noalloc: N = " + std::to_string(N) +
                                                 " needs more visited-set scratch than the " +
                                                 std::to_string(SCRATCH_BYTES >> 20) + " MiB static array holds");
    const int sms = (int)std::min<size_t>((size_t)ctx->num_sms, fit / per_sm_slots);
    a.visited = reinterpret_cast<uint32_t *>(base + off);
    a.visited_slots = (uint32_t)std::min<size_t>(fit, (size_t)sms * per_sm_slots);

    // Seed table from the host mt19937 (kgraph.cpp:444-453), staged through a stack buffer.
    cudaStream_t st = ctx->stream;
    if (walk && params->init == 0) {
        unsigned seed = params->seed ? params->seed : (unsigned)time(NULL);
        std::mt19937 rng(seed);
        uint32_t chunk[4096];
        if (params->P > 4096) return set_error(ctx, KG_E_INVALID, "kg_search_batch_noalloc supports P <= 4096");
        for (uint32_t t = 0; t < T; ++t) {
            kgb::gen_random(rng, chunk, params->P, N);
            if ((e = cudaMemcpyAsync(seeds + (size_t)t * params->P, chunk, params->P * 4, cudaMemcpyHostToDevice,
                                     st)) != cudaSuccess)
                return cuda_fail(ctx, e, "noalloc seeds");
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "noalloc seeds");
        }
    }
    cudaMemsetAsync(base, 0, HEADER_BYTES, st);        // counter, error word, work counters start at zero
    cudaMemsetAsync(seed_index, 0, nq * 4, st);         // one P for the batch: every query uses list 0
    cudaEventRecord(ctx->ev0, st);
    if ((e = launch_search(a, ctx->search_shape, sms, st, nullptr)) != cudaSuccess) return cuda_fail(ctx, e, "noalloc search launch");
    cudaEventRecord(ctx->ev1, st);
    uint32_t err = 0;
    cudaMemcpyAsync(&err, a.err, 4, cudaMemcpyDeviceToHost, st);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "noalloc search");
    cudaEventElapsedTime(&ctx->last_search_ms, ctx->ev0, ctx->ev1);
    if (err & ERR_INIT_K) return set_error(ctx, KG_E_INVALID, "L < params.K");
    if (err) return set_error(ctx, KG_E_DEVICE, "search: device reported error bits " + std::to_string(err));
    return KG_OK;
}
