// kgraph::KGraph for the B200 build: the reference's C++ API (kgraph.h) on
// top of the C-ABI (kgraph_b200.h).  Host-side logic kept from the
// reference: parameter handling, the index file format (kgraph.cpp:291-373),
// get_nn (kgraph.cpp:566-582) and the error types.  All compute goes through
// kg_* calls to the GPU.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include "../../include/kgraph.h"
#include "../../include/kgraph_b200.h"

namespace kgraph {

unsigned verbosity = default_verbosity;

namespace {

char const *KGRAPH_MAGIC = "KNNGRAPH";
constexpr unsigned KGRAPH_MAGIC_SIZE = 8;
constexpr uint32_t SIGNATURE_VERSION = 2;

// On-disk neighbour record (kgraph.cpp:67-74): {u32 id; f32 dist; bool flag; 3 pad}.
struct DiskNeighbor {
    uint32_t id;
    float dist;
    uint8_t flag;
    uint8_t pad[3];
};
static_assert(sizeof(DiskNeighbor) == 12, "neighbour record must be 12 bytes");

[[noreturn]] void throw_code(int code, std::string const &msg) {
    switch (code) {
        case KG_E_INVALID: throw invalid_argument(msg);
        case KG_E_IO: throw io_error(msg);
        default: throw runtime_error(msg);
    }
}

void check(kg_ctx *ctx, int code) {
    if (code != KG_OK) throw_code(code, kg_last_error(ctx));
}

kg_ctx *new_ctx() {
    kg_ctx *c = nullptr;
    int r = kg_ctx_create(0, &c);
    if (r != KG_OK || !c) throw runtime_error("no CUDA device available for kgraph-b200");
    return c;
}

struct Binding {
    float const *rows = nullptr;
    unsigned n = 0, d = 0;
    size_t stride = 0;
    int metric = -1;
    bool same(DenseView const &v) const {
        return rows == v.rows && n == v.n && d == v.d && stride == v.stride && metric == v.metric;
    }
};

void bind(kg_ctx *ctx, Binding &b, DenseView const &v, bool force) {
    if (v.metric < 0 || v.metric > 2) throw invalid_argument("metric not supported by the GPU oracles");
    if (!force && b.same(v)) return;
    check(ctx, kg_set_data(ctx, v.rows, v.n, v.d, v.stride, v.metric));
    b.rows = v.rows; b.n = v.n; b.d = v.d; b.stride = v.stride; b.metric = v.metric;
}

kg_search_params to_c(KGraph::SearchParams const &p) {
    kg_search_params c;
    c.K = p.K; c.M = p.M; c.P = p.P; c.S = p.S; c.T = p.T; c.epsilon = p.epsilon; c.seed = p.seed; c.init = p.init;
    return c;
}

class KGraphB200 : public KGraph {
    kg_ctx *ctx;
    mutable Binding binding;
    mutable std::mutex mu;
    // Host mirror of the graph for save / get_nn, refreshed lazily.
    mutable bool mirror_ok = false;
    mutable std::vector<uint64_t> off;
    mutable std::vector<uint32_t> ids, Ms;
    mutable std::vector<float> dists;
    bool has_graph = false;
    bool no_dist = false;

    void refresh() const {
        if (mirror_ok) return;
        size_t n = 0, E = 0;
        check(ctx, kg_graph_size(ctx, &n, &E));
        off.resize(n + 1);
        ids.resize(E);
        Ms.resize(n);
        dists.assign(no_dist ? 0 : E, 0.f);
        check(ctx, kg_graph_export(ctx, off.data(), ids.data(), no_dist ? nullptr : dists.data(), Ms.data()));
        mirror_ok = true;
    }

public:
    KGraphB200() : ctx(new_ctx()) {}
    ~KGraphB200() override { kg_ctx_destroy(ctx); }

    void load(char const *path) override {
        std::lock_guard<std::mutex> g(mu);
        std::ifstream is(path, std::ios::binary);
        if (!is) throw io_error(std::string("cannot open ") + path);
        char magic[KGRAPH_MAGIC_SIZE];
        uint32_t sig_version = 0, sig_cap = 0, N = 0;
        is.read(magic, sizeof(magic));
        is.read(reinterpret_cast<char *>(&sig_version), sizeof(sig_version));
        is.read(reinterpret_cast<char *>(&sig_cap), sizeof(sig_cap));
        if (sig_version != SIGNATURE_VERSION) throw runtime_error("data version not supported.");
        is.read(reinterpret_cast<char *>(&N), sizeof(N));
        if (!is) throw io_error("error reading index file.");
        // kgraph.cpp:304-306 checks the magic but never throws; kept lenient.
        bool nd = sig_cap & FORMAT_NO_DIST;
        std::vector<uint64_t> o(N + 1, 0);
        std::vector<uint32_t> id, M(N);
        std::vector<float> ds;
        std::vector<DiskNeighbor> rec;
        for (uint32_t i = 0; i < N; ++i) {
            uint32_t K = 0;
            is.read(reinterpret_cast<char *>(&M[i]), sizeof(M[i]));
            is.read(reinterpret_cast<char *>(&K), sizeof(K));
            if (!is) throw io_error("error reading index file.");
            size_t base = id.size();
            id.resize(base + K);
            if (nd) {
                is.read(reinterpret_cast<char *>(id.data() + base), K * sizeof(uint32_t));
            } else {
                rec.resize(K);
                is.read(reinterpret_cast<char *>(rec.data()), K * sizeof(DiskNeighbor));
                ds.resize(base + K);
                for (uint32_t k = 0; k < K; ++k) { id[base + k] = rec[k].id; ds[base + k] = rec[k].dist; }
            }
            if (!is) throw io_error("error reading index file.");
            o[i + 1] = o[i] + K;
        }
        for (uint32_t v : id)
            if (v >= N) throw io_error("index corrupted.");
        check(ctx, kg_graph_import(ctx, N, o.data(), id.data(), nd ? nullptr : ds.data(), M.data()));
        has_graph = true;
        no_dist = nd;
        mirror_ok = false;
    }

    void save(char const *path, int format) const override {
        std::lock_guard<std::mutex> g(mu);
        refresh();
        uint32_t N = (uint32_t)Ms.size();
        if (format == FORMAT_TEXT) {   // kgraph.cpp:334-348
            std::cerr << "Saving to text file; you won't be able to load text file." << std::endl;
            std::ofstream os(path);
            os << N << std::endl;
            for (uint32_t i = 0; i < N; ++i) {
                uint32_t K = (uint32_t)(off[i + 1] - off[i]);
                os << K;
                for (uint64_t e = off[i]; e < off[i + 1]; ++e) os << ' ' << ids[e] << ' ' << (no_dist ? 0.f : dists[e]);
                os << std::endl;
            }
            return;
        }
        std::ofstream os(path, std::ios::binary);
        if (!os) throw io_error(std::string("cannot open ") + path);
        os.write(KGRAPH_MAGIC, KGRAPH_MAGIC_SIZE);
        os.write(reinterpret_cast<char const *>(&SIGNATURE_VERSION), sizeof(SIGNATURE_VERSION));
        uint32_t sig_cap = format;
        os.write(reinterpret_cast<char const *>(&sig_cap), sizeof(sig_cap));
        os.write(reinterpret_cast<char const *>(&N), sizeof(N));
        std::vector<DiskNeighbor> rec;
        for (uint32_t i = 0; i < N; ++i) {
            uint32_t K = (uint32_t)(off[i + 1] - off[i]);
            os.write(reinterpret_cast<char const *>(&Ms[i]), sizeof(Ms[i]));
            os.write(reinterpret_cast<char const *>(&K), sizeof(K));
            if (format & FORMAT_NO_DIST) {
                os.write(reinterpret_cast<char const *>(ids.data() + off[i]), K * sizeof(uint32_t));
            } else {
                rec.assign(K, DiskNeighbor{0, 0.f, 0, {0, 0, 0}});
                for (uint32_t k = 0; k < K; ++k) {
                    rec[k].id = ids[off[i] + k];
                    rec[k].dist = no_dist ? 0.f : dists[off[i] + k];
                }
                os.write(reinterpret_cast<char const *>(rec.data()), K * sizeof(DiskNeighbor));
            }
        }
        if (!os) throw io_error(std::string("error writing ") + path);
    }

    void build(IndexOracle const &oracle, IndexParams const &params, IndexInfo *info) override {
        std::lock_guard<std::mutex> g(mu);
        auto const *dense = dynamic_cast<DenseIndexOracle const *>(&oracle);
        if (!dense)
            throw invalid_argument("kgraph-b200 builds on the GPU and needs a dense oracle (MatrixOracle or "
                                   "DenseMatrixOracle); this oracle has no dense view");
        bind(ctx, binding, dense->dense(), true);
        kg_index_params p;
        p.iterations = params.iterations; p.L = params.L; p.K = params.K; p.S = params.S; p.R = params.R;
        p.controls = params.controls; p.seed = params.seed; p.delta = params.delta; p.recall = params.recall;
        p.prune = params.prune; p.reverse = params.reverse;
        kg_set_verbosity(verbosity);
        kg_index_info ci;
        check(ctx, kg_build(ctx, &p, &ci));
        if (info) {
            info->stop_condition = (IndexInfo::StopCondition)ci.stop_condition;
            info->iterations = ci.iterations;
            info->cost = ci.cost; info->recall = ci.recall; info->accuracy = ci.accuracy;
            info->delta = ci.delta; info->M = ci.M;
        }
        has_graph = true;
        no_dist = false;
        mirror_ok = false;
    }

    void prune(IndexOracle const &, unsigned level) override {
        std::lock_guard<std::mutex> g(mu);
        check(ctx, kg_prune(ctx, level));
        mirror_ok = false;
    }

    unsigned search(SearchOracle const &oracle, SearchParams const &params, unsigned *out_ids, float *out_dists,
                    SearchInfo *pinfo) const override {
        std::lock_guard<std::mutex> g(mu);
        auto const *dense = dynamic_cast<DenseSearchOracle const *>(&oracle);
        if (!dense)
            throw invalid_argument("kgraph-b200 searches on the GPU and needs a dense search oracle");
        DenseView v = dense->dense();
        bind(ctx, const_cast<Binding &>(binding), v, false);
        kg_search_params p = to_c(params);
        unsigned cnt = 0;
        float cost = 0.f;
        std::vector<uint32_t> ibuf(params.K ? params.K : 1);
        if (params.init && out_ids)
            for (unsigned l = 0; l < params.init && l < ibuf.size(); ++l) ibuf[l] = out_ids[l];
        std::vector<float> dbuf(params.K ? params.K : 1);
        int r = kg_search_batch(ctx, dense->query(), 1, v.d * sizeof(float), &p, nullptr, nullptr,
                                params.K ? params.K : 1, ibuf.data(), dbuf.data(), &cnt, &cost);
        if (r != KG_OK) throw_code(r, kg_last_error(ctx));
        if (out_ids) for (unsigned k = 0; k < cnt; ++k) out_ids[k] = ibuf[k];
        if (out_dists) for (unsigned k = 0; k < cnt; ++k) out_dists[k] = dbuf[k];
        if (pinfo) { pinfo->cost = cost; pinfo->updates = 0; }
        return cnt;
    }

    void search_batch(IndexOracle const &oracle, float const *queries, unsigned nq, size_t qstride,
                      SearchParams const &params, unsigned *out_ids, float *out_dists, unsigned *counts,
                      float *costs) const override {
        std::lock_guard<std::mutex> g(mu);
        auto const *dense = dynamic_cast<DenseIndexOracle const *>(&oracle);
        if (!dense) throw invalid_argument("kgraph-b200 searches on the GPU and needs a dense oracle");
        bind(ctx, const_cast<Binding &>(binding), dense->dense(), false);
        kg_search_params p = to_c(params);
        std::vector<uint32_t> cbuf;
        if (!counts) { cbuf.resize(nq); counts = cbuf.data(); }
        int r = kg_search_batch(ctx, queries, nq, qstride, &p, nullptr, nullptr, params.K, out_ids, out_dists,
                                counts, costs);
        if (r != KG_OK) throw_code(r, kg_last_error(ctx));
    }

    void *native_context(IndexOracle const &oracle) override {
        std::lock_guard<std::mutex> g(mu);
        auto const *dense = dynamic_cast<DenseIndexOracle const *>(&oracle);
        if (!dense) throw invalid_argument("kgraph-b200 needs a dense oracle");
        bind(ctx, binding, dense->dense(), false);
        return ctx;
    }

    void get_nn(unsigned id, unsigned *nns, float *dist, unsigned *pM, unsigned *pL) const override {
        std::lock_guard<std::mutex> g(mu);
        refresh();
        if (!(id < Ms.size())) throw invalid_argument("id too big");
        *pM = Ms[id];
        *pL = (unsigned)(off[id + 1] - off[id]);
        if (nns) for (uint64_t e = off[id]; e < off[id + 1]; ++e) nns[e - off[id]] = ids[e];
        if (dist) {
            if (no_dist) throw runtime_error("distance information is not available");
            for (uint64_t e = off[id]; e < off[id + 1]; ++e) dist[e - off[id]] = dists[e];
        }
    }

    void reverse(int rev_k) override {
        std::lock_guard<std::mutex> g(mu);
        if (rev_k == 0) return;
        if (no_dist) throw runtime_error("Need distance information to reverse graph");
        check(ctx, kg_reverse(ctx, rev_k));
        mirror_ok = false;
    }
};

// One process-wide context for SearchOracle::search on dense oracles.
kg_ctx *shared_ctx() {
    static std::once_flag once;
    static kg_ctx *c = nullptr;
    std::call_once(once, [] { c = new_ctx(); });
    return c;
}

}  // namespace

KGraph *KGraph::create() { return new KGraphB200; }

char const *KGraph::version() { return kg_version(); }

// SearchOracle::search (kgraph.cpp:231-252): exact brute force on the GPU.
unsigned SearchOracle::search(unsigned K, float epsilon, unsigned *ids, float *dists) const {
    auto const *dense = dynamic_cast<DenseSearchOracle const *>(this);
    if (!dense) throw invalid_argument("brute-force search needs a dense search oracle on the GPU build");
    static std::mutex mu;
    std::lock_guard<std::mutex> g(mu);
    static Binding b;
    kg_ctx *c = shared_ctx();
    DenseView v = dense->dense();
    bind(c, b, v, false);
    kg_search_params p;
    kg_search_params_default(&p);
    p.K = K;
    p.epsilon = epsilon;
    std::vector<uint32_t> ib(K ? K : 1);
    std::vector<float> db(K ? K : 1);
    unsigned cnt = 0;
    int r = kg_search_batch(c, dense->query(), 1, v.d * sizeof(float), &p, nullptr, nullptr, K ? K : 1, ib.data(),
                            db.data(), &cnt, nullptr);
    if (r != KG_OK) throw_code(r, kg_last_error(c));
    for (unsigned k = 0; k < cnt; ++k) {
        if (ids) ids[k] = ib[k];
        if (dists) dists[k] = db[k];
    }
    return cnt;
}

}  // namespace kgraph
