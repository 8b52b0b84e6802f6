// Python module of the B200 build: the reference's `kgraph.KGraph(data,
// metric)` class (python-api.cpp:331-450) with the same methods, keyword
// arguments, defaults and errors, over the C++ API in kgraph.h.
//
// Extensions (no counterpart in the reference's module): search(..., router=m)
// seeds the walk with m learned entry nodes (train_router first);
// set_search_precision() and autotune() reach the distance filter and the
// search autotuner of the C-ABI.
//
// Differences, by design: search() runs all queries of one call in a single
// GPU launch (the reference loops over queries with OpenMP,
// python-api.cpp:291-301); blas=True takes the exact GPU brute force in place
// of the reference's optional OpenBLAS path (python-api.cpp:131-205); float64
// input is rejected ("data type not supported.") because the GPU kernels
// compute in float32.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>
#include "../../include/kgraph.h"
#include "../../include/kgraph-data.h"
#include "../../include/kgraph_b200.h"

namespace py = pybind11;

namespace {

struct AlignedRows {   // the reference's AlignedMatrix (python-api.cpp:72-85)
    float *p = nullptr;
    unsigned n = 0, d = 0;
    size_t stride = 0;
    AlignedRows(float const *src, unsigned rows, unsigned cols, size_t src_stride) : n(rows), d(cols) {
        stride = (cols * sizeof(float) + 63) / 64 * 64;
        size_t bytes = (size_t)rows * stride;
        p = (float *)aligned_alloc(64, bytes ? bytes : 64);
        if (!p) throw std::runtime_error("memalign");
        std::memset(p, 0, bytes);
        for (unsigned i = 0; i < rows; ++i)
            std::memcpy(reinterpret_cast<char *>(p) + stride * i, reinterpret_cast<char const *>(src) + src_stride * i,
                        cols * sizeof(float));
    }
    ~AlignedRows() { free(p); }
    AlignedRows(AlignedRows const &) = delete;
    AlignedRows &operator=(AlignedRows const &) = delete;
};

py::array_t<float, py::array::c_style | py::array::forcecast> as_f32_2d(py::object obj, bool strict) {
    py::array a = py::array::ensure(obj);
    if (!a) throw kgraph::invalid_argument("bad array");
    if (strict && !py::isinstance<py::array_t<float>>(a)) throw std::runtime_error("data type not supported.");
    auto f = py::array_t<float, py::array::c_style | py::array::forcecast>::ensure(a);
    if (!f || f.ndim() != 2) throw kgraph::invalid_argument("expecting a 2-D array");
    return f;
}

class PyKGraph {
    std::unique_ptr<AlignedRows> data;
    std::unique_ptr<kgraph::DenseMatrixOracle> oracle;
    std::unique_ptr<kgraph::KGraph> index;
    std::unique_ptr<kgraph::KGraph> brute;   // graph-less instance: exact brute force
    bool hasIndex = false;

public:
    PyKGraph(py::object obj, std::string const &metric) {
        int code;
        if (metric == "euclidean") code = 0;
        else if (metric == "angular") code = 1;
        else throw std::runtime_error("metric not supported");
        auto arr = as_f32_2d(obj, true);
        data.reset(new AlignedRows(arr.data(), (unsigned)arr.shape(0), (unsigned)arr.shape(1),
                                   (size_t)arr.shape(1) * sizeof(float)));
        oracle.reset(new kgraph::DenseMatrixOracle(data->p, data->n, data->d, data->stride, code));
        index.reset(kgraph::KGraph::create());
    }

    void load(char const *path) { index->load(path); hasIndex = true; }
    void save(char const *path) const { index->save(path); }
    void save_text(char const *path) const { index->save(path, kgraph::KGraph::FORMAT_TEXT); }

    void build(unsigned iterations, unsigned L, unsigned K, unsigned S, unsigned controls, float delta, float recall,
               unsigned prune, int reverse) {
        kgraph::KGraph::IndexParams params;   // R and seed keep their defaults, as in python-api.cpp:378-388
        params.iterations = iterations;
        params.L = L;
        params.K = K;
        params.S = S;
        params.controls = controls;
        params.delta = delta;
        params.recall = recall;
        params.prune = prune;
        params.reverse = reverse;
        {
            py::gil_scoped_release nogil;
            index->build(*oracle, params, nullptr);
        }
        hasIndex = true;
    }

    // ---- extensions of this library (no counterpart in the reference's module)

    // The index's C-ABI context with this object's dataset bound to it.
    kg_ctx *native() {
        if (!hasIndex) throw kgraph::runtime_error("no index: build or load one first");
        auto *c = static_cast<kg_ctx *>(index->native_context(*oracle));
        if (!c) throw kgraph::runtime_error("no native context");
        return c;
    }

    static void check_c(kg_ctx *c, int r) {
        if (r == KG_OK) return;
        if (r == KG_E_INVALID) throw kgraph::invalid_argument(kg_last_error(c));
        throw kgraph::runtime_error(kg_last_error(c));
    }

    // Learned entry router on the index (kg_router_train): trained on queries
    // from the same distribution as the ones it will seed.
    py::dict train_router(py::object queries, unsigned clusters, unsigned hidden, unsigned kmeans_iters,
                          unsigned label_P, unsigned epochs, unsigned batch, float lr, unsigned seed,
                          unsigned entries, unsigned probe, unsigned refine, unsigned refine_P) {
        kg_ctx *c = native();
        auto q = as_f32_2d(queries, false);
        if ((unsigned)q.shape(1) != data->d) throw kgraph::invalid_argument("query dimension mismatch");
        kg_router_params p;
        kg_router_params_default(&p);
        p.clusters = clusters; p.hidden = hidden; p.kmeans_iters = kmeans_iters; p.label_P = label_P;
        p.epochs = epochs; p.batch = batch; p.lr = lr; p.seed = seed; p.entries = entries; p.probe = probe;
        p.refine = refine; p.refine_P = refine_P;
        kg_router_info info{};
        int r;
        {
            py::gil_scoped_release nogil;
            r = kg_router_train(c, &p, q.data(), (size_t)q.shape(0), (size_t)q.shape(1) * sizeof(float), &info);
        }
        check_c(c, r);
        py::dict d;
        d["steps"] = info.steps;
        d["final_loss"] = info.final_loss;
        d["train_accuracy"] = info.train_accuracy;
        d["empty_clusters"] = info.empty_clusters;
        d["entries"] = info.entries;
        d["relabelled"] = info.relabelled;
        return d;
    }

    // Distance filter of the walk (kg_set_search_precision): "fp32", "bf16" or "fp8".
    void set_search_precision(std::string const &mode) {
        int m;
        if (mode == "fp32") m = KG_SEARCH_FP32;
        else if (mode == "bf16") m = KG_SEARCH_BF16;
        else if (mode == "fp8") m = KG_SEARCH_FP8;
        else throw kgraph::invalid_argument("precision must be fp32, bf16 or fp8");
        kg_ctx *c = native();
        check_c(c, kg_set_search_precision(c, m));
    }

    // Search autotuner (kg_search_autotune) on a sample of queries at K, P.
    py::dict autotune(py::object query, unsigned K, unsigned P) {
        kg_ctx *c = native();
        auto q = as_f32_2d(query, false);
        if ((unsigned)q.shape(1) != data->d) throw kgraph::invalid_argument("query dimension mismatch");
        kg_search_params p;
        kg_search_params_default(&p);
        p.K = K;
        p.P = P;
        kg_search_tuning t{};
        int r;
        {
            py::gil_scoped_release nogil;
            r = kg_search_autotune(c, q.data(), (size_t)q.shape(0), (size_t)q.shape(1) * sizeof(float), &p, nullptr,
                                   nullptr, nullptr, 0, &t);
        }
        check_c(c, r);
        py::dict d;
        d["split"] = t.split;
        d["warps_per_block"] = t.warps_per_block;
        d["prefetch"] = t.prefetch;
        d["regs"] = t.regs;
        d["compact"] = t.compact;
        d["ms"] = t.ms;
        d["default_ms"] = t.default_ms;
        return d;
    }

    py::object search(py::object query, unsigned K, unsigned P, unsigned M, unsigned S, unsigned T,
                      unsigned threads, bool withDistance, bool blas, unsigned router) {
        (void)threads;   // one launch covers every query; the reference's thread knob has no effect here
        auto q = as_f32_2d(query, false);
        if ((unsigned)q.shape(1) != data->d) throw kgraph::invalid_argument("query dimension mismatch");
        size_t nq = (size_t)q.shape(0);
        py::array_t<uint32_t> result({nq, (size_t)K});
        py::array_t<float> distance({nq, (size_t)K});
        std::memset(result.mutable_data(), 0, nq * K * sizeof(uint32_t));
        std::memset(distance.mutable_data(), 0, nq * K * sizeof(float));
        kgraph::KGraph::SearchParams params;
        params.K = K;
        params.P = P;
        params.M = M;
        params.S = S;
        params.T = T;
        if (nq) {
            uint32_t *ids = result.mutable_data();
            float *dists = distance.mutable_data();
            float const *qp = q.data();
            size_t qstride = (size_t)q.shape(1) * sizeof(float);
            kg_ctx *rc = router ? native() : nullptr;   // router seeds: kg_router_search on the index
            py::gil_scoped_release nogil;
            if (router) {
                kg_search_params p;
                kg_search_params_default(&p);
                p.K = K; p.P = P; p.M = M; p.S = S; p.T = T; p.init = router;
                std::vector<uint32_t> counts(nq);
                int r = kg_router_search(rc, qp, nq, qstride, &p, K, ids, dists, counts.data(), nullptr);
                if (r != KG_OK) {
                    py::gil_scoped_acquire gil;
                    check_c(rc, r);
                }
            } else if (hasIndex && !blas) {
                index->search_batch(*oracle, qp, (unsigned)nq, qstride, params, ids, dists, nullptr, nullptr);
            } else {
                if (!brute) brute.reset(kgraph::KGraph::create());
                brute->search_batch(*oracle, qp, (unsigned)nq, qstride, params, ids, dists, nullptr, nullptr);
            }
        }
        if (withDistance) return py::make_tuple(result, distance);
        return result;
    }
};

}  // namespace

PYBIND11_MODULE(_kgraph, module) {
    py::dict arch;
    arch["name"] = "sm_100a";
    arch["alignment"] = 64;
    module.doc() = "KGraph (NN-descent k-NN graph + graph search) on NVIDIA B200";
    module.attr("git_commit") = "kgraph-b200";
    module.attr("arch") = arch;
    module.attr("version") = kgraph::KGraph::version();
    py::class_<PyKGraph>(module, "KGraph")
        .def(py::init<py::object, std::string const &>())
        .def("load", &PyKGraph::load, "load")
        .def("save", &PyKGraph::save, "save")
        .def("save_text", &PyKGraph::save_text, "save_text")
        .def("build", &PyKGraph::build, "build", py::arg("iterations") = kgraph::default_iterations,
             py::arg("L") = kgraph::default_L, py::arg("K") = kgraph::default_K, py::arg("S") = kgraph::default_S,
             py::arg("controls") = kgraph::default_controls, py::arg("delta") = kgraph::default_delta,
             py::arg("recall") = kgraph::default_recall, py::arg("prune") = kgraph::default_prune,
             py::arg("reverse") = kgraph::default_reverse)
        .def("search", &PyKGraph::search, "search", py::arg("query"), py::arg("K") = kgraph::default_K,
             py::arg("P") = kgraph::default_P, py::arg("M") = kgraph::default_M, py::arg("S") = kgraph::default_S,
             py::arg("T") = kgraph::default_T, py::arg("threads") = 0, py::arg("withDistance") = false,
             py::arg("blas") = false, py::arg("router") = 0)
        // extensions of this library
        .def("train_router", &PyKGraph::train_router, "learned entry router (kg_router_train)", py::arg("queries"),
             py::arg("clusters") = 1024, py::arg("hidden") = 256, py::arg("kmeans_iters") = 8,
             py::arg("label_P") = 1000, py::arg("epochs") = 4, py::arg("batch") = 1024, py::arg("lr") = 2e-3f,
             py::arg("seed") = 1998, py::arg("entries") = 8, py::arg("probe") = 8, py::arg("refine") = 2,
             py::arg("refine_P") = 50)
        .def("set_search_precision", &PyKGraph::set_search_precision,
             "distance filter of the walk: 'fp32', 'bf16' or 'fp8' (identical results)", py::arg("mode"))
        .def("autotune", &PyKGraph::autotune, "search autotuner (kg_search_autotune)", py::arg("query"),
             py::arg("K") = 10, py::arg("P") = kgraph::default_P);
}
