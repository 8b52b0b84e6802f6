// Graph post-processing on the GPU: reverse-edge completion
// (KGraphImpl::reverse, kgraph.cpp:667-702) and pruning (kgraph.cpp:584-665).
//
// reverse.  The reference appends, for every node i in increasing order and
// every kept forward edge j, the edge to ng[i] and its reverse to ng[e.id],
// then std::sort's each list by distance and drops ADJACENT duplicate ids.
// std::sort is not stable, so the final order of equal distances -- and which
// duplicates end up adjacent -- depends on the list's push order and on the
// GNU introsort.  Here the push order is rebuilt exactly (reverse edges
// grouped by target with a stable radix sort of (target) over edges numbered
// in (i, j) order, the node's own forward edges spliced in at i == x), and
// each list is sorted by the same introsort (kg_sort.h), one thread per node.
// The result is the reference's graph bit for bit.
#include <cub/cub.cuh>
#include <iostream>
#include <vector>
#include "kg_ctx.h"
#include "kg_sort.h"

namespace kgb {

cudaError_t scan_counts64(kg_ctx *ctx, const uint64_t *in, uint64_t *out, uint32_t n);

namespace {

__global__ void rev_count_kernel(uint32_t N, const uint64_t *off, const uint32_t *M, int rev_k, uint64_t *kcnt) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        uint32_t deg = (uint32_t)(off[i + 1] - off[i]);
        uint32_t k = rev_k > 0 ? min((uint32_t)rev_k, deg) : min(M[i], deg);
        kcnt[i] = k;
    }
}

// One entry per kept forward edge, numbered in (i, j) order: its target and index.
__global__ void rev_edges_kernel(uint32_t N, const uint64_t *off, const uint32_t *nbr, const uint64_t *koff,
                                 uint32_t *key, uint32_t *val, uint64_t *rc, uint32_t *err) {
    const int lane = threadIdx.x & 31;
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = w; i < N; i += nw) {
        const uint64_t b = koff[i];
        const uint32_t k = (uint32_t)(koff[i + 1] - b);
        for (uint32_t j = lane; j < k; j += 32) {
            uint32_t t = nbr[off[i] + j];
            if (t >= N) { atomicOr(err, 4u); t = i; }
            key[b + j] = t;
            val[b + j] = (uint32_t)(b + j);
            atomicAdd(reinterpret_cast<unsigned long long *>(rc + t), 1ull);
        }
    }
}

__global__ void rev_degree_kernel(uint32_t N, const uint64_t *kcnt, const uint64_t *rc, uint64_t *deg) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) deg[i] = kcnt[i] + rc[i];
}

// Upper bound of edge index e in the (i, j) numbering -> source node i.
__device__ __forceinline__ uint32_t source_of(const uint64_t *koff, uint32_t N, uint64_t e) {
    uint32_t lo = 0, hi = N;   // first i with koff[i+1] > e
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (koff[mid + 1] > e) hi = mid; else lo = mid + 1;
    }
    return lo;
}

struct ListAcc {
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

// Rebuilds node x's list in the reference's push order, sorts it with the
// GNU introsort, removes adjacent duplicate ids; writes its final length.
__global__ void rev_assemble_kernel(uint32_t N, const uint64_t *off, const uint32_t *nbr, const float *nbr_d,
                                    const uint64_t *koff, const uint64_t *toff, const uint32_t *sorted_val,
                                    const uint64_t *noff, uint32_t *out_i, float *out_d, uint64_t *fdeg) {
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < N; x += gridDim.x * blockDim.x) {
        uint32_t *oi = out_i + noff[x];
        float *od = out_d + noff[x];
        uint32_t p = 0;
        uint64_t q = toff[x];
        const uint64_t qe = toff[x + 1];
        const uint32_t kx = (uint32_t)(koff[x + 1] - koff[x]);
        // reverse edges from sources i < x
        while (q < qe) {
            uint64_t e = sorted_val[q];
            uint32_t src = source_of(koff, N, e);
            if (src >= x) break;
            oi[p] = src;
            od[p] = nbr_d[off[src] + (e - koff[src])];
            ++p; ++q;
        }
        // own forward edges; a self loop's reverse edge follows its forward edge
        for (uint32_t j = 0; j < kx; ++j) {
            oi[p] = nbr[off[x] + j];
            od[p] = nbr_d[off[x] + j];
            ++p;
            while (q < qe) {
                uint64_t e = sorted_val[q];
                if (source_of(koff, N, e) != x || e - koff[x] != j) break;
                oi[p] = x;
                od[p] = nbr_d[off[x] + j];
                ++p; ++q;
            }
        }
        // reverse edges from sources i > x
        while (q < qe) {
            uint64_t e = sorted_val[q];
            uint32_t src = source_of(koff, N, e);
            oi[p] = src;
            od[p] = nbr_d[off[src] + (e - koff[src])];
            ++p; ++q;
        }
        ListAcc acc{od, oi};
        gnu_sort(acc, 0, (int)p);   // kgraph.cpp:697
        uint32_t m = 0;             // std::unique by id (kgraph.cpp:698)
        for (uint32_t r = 0; r < p; ++r) {
            if (m > 0 && oi[m - 1] == oi[r]) continue;
            oi[m] = oi[r];
            od[m] = od[r];
            ++m;
        }
        fdeg[x] = m;
    }
}

__global__ void compact_kernel(uint32_t N, const uint64_t *src_off, const uint64_t *dst_off, const uint32_t *si,
                               const float *sd, uint32_t *di, float *dd, uint32_t *M, int set_M) {
    const int lane = threadIdx.x & 31;
    const uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t x = w; x < N; x += nw) {
        const uint64_t a = src_off[x], b = dst_off[x];
        const uint32_t c = (uint32_t)(dst_off[x + 1] - b);
        for (uint32_t r = lane; r < c; r += 32) {
            di[b + r] = si[a + r];
            if (sd) dd[b + r] = sd[a + r];
        }
        if (set_M && lane == 0) M[x] = c;
    }
}

__global__ void prune1_count_kernel(uint32_t N, const uint64_t *off, const uint32_t *M, uint64_t *cnt) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        uint32_t deg = (uint32_t)(off[i + 1] - off[i]);
        cnt[i] = deg > M[i] ? M[i] : deg;
    }
}

}  // namespace

// Installs (off, ids, dists) of n nodes as the context's graph, taking ownership
// of the three scratch buffers by swapping them in.
static void swap_graph(kg_ctx *ctx, DevBuf &off, DevBuf &ids, DevBuf &dists) {
    std::swap(ctx->offsets, off);
    std::swap(ctx->nbr, ids);
    std::swap(ctx->nbr_d, dists);
}

int graph_reverse(kg_ctx *ctx, int rev_k) {
    if (rev_k == 0) return KG_OK;
    if (!ctx->has_graph) return set_error(ctx, KG_E_RUNTIME, "no index");
    if (ctx->no_dist) return set_error(ctx, KG_E_RUNTIME, "Need distance information to reverse graph");
    std::cerr << "Graph completion with reverse edges..." << std::endl;
    const uint32_t N = ctx->gn;
    const size_t n = N;
    cudaStream_t st = ctx->stream;
    cudaError_t e;
    // Work space kept in the context between calls: a build reverses once per call, and freeing and
    // re-allocating ~2 GB (1M nodes) each time costs device-synchronising cudaFree / cudaMalloc calls whose
    // time varied from build to build.  Buffers grow with 1/8 slack.
    DevBuf *R = ctx->rev_scratch;
    DevBuf &kcnt = R[0], &koff = R[1], &rc = R[2], &toff = R[3], &deg = R[4], &noff = R[5], &fdeg = R[6],
           &foff = R[7], &key = R[8], &val = R[9], &skey = R[10], &sval = R[11], &tmp = R[12], &ai = R[13],
           &ad = R[14], &fi = R[15], &fd = R[16];
    auto grow = [](DevBuf &b, size_t bytes) { return b.reserve(bytes <= b.bytes ? bytes : bytes + bytes / 8); };
    auto fail = [&](const char *w) { return cuda_fail(ctx, e, w); };
    if ((e = grow(kcnt, (n + 1) * 8)) != cudaSuccess || (e = grow(koff, (n + 1) * 8)) != cudaSuccess ||
        (e = grow(rc, (n + 1) * 8)) != cudaSuccess || (e = grow(toff, (n + 1) * 8)) != cudaSuccess ||
        (e = grow(deg, (n + 1) * 8)) != cudaSuccess || (e = grow(noff, (n + 1) * 8)) != cudaSuccess ||
        (e = grow(fdeg, (n + 1) * 8)) != cudaSuccess || (e = grow(foff, (n + 1) * 8)) != cudaSuccess)
        return fail("alloc reverse");
    cudaMemsetAsync(kcnt.p, 0, (n + 1) * 8, st);
    cudaMemsetAsync(rc.p, 0, (n + 1) * 8, st);
    cudaMemsetAsync(deg.p, 0, (n + 1) * 8, st);
    cudaMemsetAsync(fdeg.p, 0, (n + 1) * 8, st);
    const int grid = ctx->num_sms * 4;
    rev_count_kernel<<<grid, 256, 0, st>>>(N, ctx->offsets.as<uint64_t>(), ctx->Mnode.as<uint32_t>(), rev_k,
                                           kcnt.as<uint64_t>());
    if ((e = scan_counts64(ctx, kcnt.as<uint64_t>(), koff.as<uint64_t>(), N)) != cudaSuccess) return fail("scan");
    uint64_t Ef = 0;
    cudaMemcpyAsync(&Ef, koff.as<uint64_t>() + N, 8, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    if (Ef >= 0xFFFFFFFFull) { e = cudaErrorInvalidValue; return fail("graph too large to reverse"); }
    if ((e = grow(key, Ef * 4 + 4)) != cudaSuccess || (e = grow(val, Ef * 4 + 4)) != cudaSuccess ||
        (e = grow(skey, Ef * 4 + 4)) != cudaSuccess || (e = grow(sval, Ef * 4 + 4)) != cudaSuccess)
        return fail("alloc reverse");
    rev_edges_kernel<<<grid * 2, 256, 0, st>>>(N, ctx->offsets.as<uint64_t>(), ctx->nbr.as<uint32_t>(),
                                               koff.as<uint64_t>(), key.as<uint32_t>(), val.as<uint32_t>(),
                                               rc.as<uint64_t>(), ctx->errw.as<uint32_t>());
    // stable radix sort by target keeps the (i, j) order within each target
    int end_bit = 1;
    while (end_bit < 32 && (1ull << end_bit) < n) ++end_bit;
    size_t tb = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, tb, key.as<uint32_t>(), skey.as<uint32_t>(), val.as<uint32_t>(),
                                    sval.as<uint32_t>(), (int64_t)Ef, 0, end_bit, st);
    if ((e = grow(tmp, tb)) != cudaSuccess) return fail("alloc sort");
    if ((e = cub::DeviceRadixSort::SortPairs(tmp.p, tb, key.as<uint32_t>(), skey.as<uint32_t>(), val.as<uint32_t>(),
                                             sval.as<uint32_t>(), (int64_t)Ef, 0, end_bit, st)) != cudaSuccess)
        return fail("sort");
    if ((e = scan_counts64(ctx, rc.as<uint64_t>(), toff.as<uint64_t>(), N)) != cudaSuccess) return fail("scan");
    rev_degree_kernel<<<grid, 256, 0, st>>>(N, kcnt.as<uint64_t>(), rc.as<uint64_t>(), deg.as<uint64_t>());
    if ((e = scan_counts64(ctx, deg.as<uint64_t>(), noff.as<uint64_t>(), N)) != cudaSuccess) return fail("scan");
    const uint64_t E2 = 2 * Ef;
    if ((e = grow(ai, E2 * 4 + 4)) != cudaSuccess || (e = grow(ad, E2 * 4 + 4)) != cudaSuccess)
        return fail("alloc reverse");
    std::cerr << "Reranking edges..." << std::endl;
    rev_assemble_kernel<<<(N + 127) / 128, 128, 0, st>>>(
        N, ctx->offsets.as<uint64_t>(), ctx->nbr.as<uint32_t>(), ctx->nbr_d.as<float>(), koff.as<uint64_t>(),
        toff.as<uint64_t>(), sval.as<uint32_t>(), noff.as<uint64_t>(), ai.as<uint32_t>(), ad.as<float>(),
        fdeg.as<uint64_t>());
    if ((e = cudaGetLastError()) != cudaSuccess) return fail("reverse");
    if ((e = scan_counts64(ctx, fdeg.as<uint64_t>(), foff.as<uint64_t>(), N)) != cudaSuccess) return fail("scan");
    uint64_t Efin = 0;
    cudaMemcpyAsync(&Efin, foff.as<uint64_t>() + N, 8, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    if ((e = grow(fi, Efin * 4 + 4)) != cudaSuccess || (e = grow(fd, Efin * 4 + 4)) != cudaSuccess)
        return fail("alloc reverse");
    compact_kernel<<<grid * 2, 256, 0, st>>>(N, noff.as<uint64_t>(), foff.as<uint64_t>(), ai.as<uint32_t>(),
                                             ad.as<float>(), fi.as<uint32_t>(), fd.as<float>(),
                                             ctx->Mnode.as<uint32_t>(), 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return fail("reverse");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail("reverse");
    swap_graph(ctx, foff, fi, fd);
    ctx->E = Efin;
    ++ctx->graph_version;
    return check_device_error(ctx, "reverse");
}

// prune1 (kgraph.cpp:584-590) on the GPU.
static int prune1(kg_ctx *ctx) {
    const uint32_t N = ctx->gn;
    const size_t n = N;
    cudaStream_t st = ctx->stream;
    cudaError_t e;
    DevBuf cnt, noff, ni, nd;
    if ((e = cnt.reserve((n + 1) * 8)) != cudaSuccess || (e = noff.reserve((n + 1) * 8)) != cudaSuccess)
        return cuda_fail(ctx, e, "alloc prune");
    cudaMemsetAsync(cnt.p, 0, (n + 1) * 8, st);
    prune1_count_kernel<<<ctx->num_sms * 4, 256, 0, st>>>(N, ctx->offsets.as<uint64_t>(), ctx->Mnode.as<uint32_t>(),
                                                           cnt.as<uint64_t>());
    if ((e = scan_counts64(ctx, cnt.as<uint64_t>(), noff.as<uint64_t>(), N)) != cudaSuccess) return cuda_fail(ctx, e, "scan");
    uint64_t E = 0;
    cudaMemcpyAsync(&E, noff.as<uint64_t>() + N, 8, cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    if ((e = ni.reserve(E * 4 + 4)) != cudaSuccess || (e = nd.reserve(E * 4 + 4)) != cudaSuccess)
        return cuda_fail(ctx, e, "alloc prune");
    compact_kernel<<<ctx->num_sms * 8, 256, 0, st>>>(N, ctx->offsets.as<uint64_t>(), noff.as<uint64_t>(),
                                                     ctx->nbr.as<uint32_t>(), ctx->no_dist ? nullptr : ctx->nbr_d.as<float>(),
                                                     ni.as<uint32_t>(), nd.as<float>(), nullptr, 0);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_fail(ctx, e, "prune");
    swap_graph(ctx, noff, ni, nd);
    ctx->E = E;
    ++ctx->graph_version;
    return KG_OK;
}

// prune2 (kgraph.cpp:593-656): a sequential level-by-level pass whose every
// step reads the edits of the steps before it (reverse lists and flags of
// other nodes), so it runs on the host, in the reference's order, on the
// graph copied out of HBM; the result goes back to HBM.  It is maintenance
// of a finished index, not part of build or search.
static int prune2(kg_ctx *ctx) {
    const uint32_t N = ctx->gn;
    std::vector<uint64_t> off(N + 1);
    std::vector<uint32_t> ids(ctx->E), M(N);
    std::vector<float> ds(ctx->no_dist ? 0 : ctx->E);
    cudaMemcpy(off.data(), ctx->offsets.p, (N + 1) * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(ids.data(), ctx->nbr.p, ctx->E * 4, cudaMemcpyDeviceToHost);
    if (!ctx->no_dist) cudaMemcpy(ds.data(), ctx->nbr_d.p, ctx->E * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(M.data(), ctx->Mnode.p, N * 4, cudaMemcpyDeviceToHost);
    std::vector<uint8_t> flag(ctx->E, 0);
    std::vector<std::vector<uint32_t>> rev(N);
    std::vector<uint32_t> newL(N, 0), todo(N), next;
    for (uint32_t i = 0; i < N; ++i) todo[i] = i;
    auto at = [&](uint32_t node, uint32_t k) { return off[node] + k; };
    for (uint32_t l = 0; !todo.empty(); ++l) {
        next.clear();
        for (uint32_t i : todo) {
            if (l >= M[i]) continue;
            next.push_back(i);
            if (l >= off[i + 1] - off[i]) return set_error(ctx, KG_E_RUNTIME, "M larger than the list");
            if (flag[at(i, l)]) continue;
            flag[at(i, l)] = 1;
            uint32_t T;
            {
                uint32_t &nl = newL[i];
                T = ids[at(i, nl)] = ids[at(i, l)];
                if (!ds.empty()) ds[at(i, nl)] = ds[at(i, l)];
                ++nl;
            }
            rev[T].push_back(i);
            for (uint32_t ll = l + 1; ll < M[i]; ++ll) {
                if (flag[at(i, ll)]) continue;
                for (uint32_t j = 0; j < newL[T]; ++j)
                    if (ids[at(i, ll)] == ids[at(T, j)]) { flag[at(i, ll)] = 1; break; }
            }
            for (uint32_t r : rev[i])
                for (uint32_t ll = l; ll < M[r]; ++ll)
                    if (ids[at(r, ll)] == T) flag[at(r, ll)] = 1;
        }
        todo.swap(next);
    }
    cudaMemcpy(ctx->nbr.p, ids.data(), ctx->E * 4, cudaMemcpyHostToDevice);
    if (!ctx->no_dist) cudaMemcpy(ctx->nbr_d.p, ds.data(), ctx->E * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(ctx->Mnode.p, newL.data(), N * 4, cudaMemcpyHostToDevice);
    ++ctx->graph_version;
    return prune1(ctx);
}

int graph_prune(kg_ctx *ctx, unsigned level) {
    if (!ctx->has_graph) return set_error(ctx, KG_E_RUNTIME, "no index");
    if (level & 1) {
        int r = prune1(ctx);
        if (r != KG_OK) return r;
    }
    if (level & 2) {
        int r = prune2(ctx);
        if (r != KG_OK) return r;
    }
    return KG_OK;
}

}  // namespace kgb

extern "C" int kg_reverse(kg_ctx *ctx, int rev_k) {
    if (!ctx) return KG_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return kgb::graph_reverse(ctx, rev_k);
}

extern "C" int kg_prune(kg_ctx *ctx, unsigned level) {
    if (!ctx) return KG_E_INVALID;
    std::lock_guard<std::mutex> g(ctx->mu);
    cudaSetDevice(ctx->device);
    return kgb::graph_prune(ctx, level);
}
