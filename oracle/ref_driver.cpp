// C entry points over the REFERENCE's own C++ API, for ctypes callers in the
// tests and in the CPU baseline.  This file is project code; it is compiled
// together with the reference's kgraph.cpp (see oracle/Makefile) and calls
// only the reference's public interface:
//   KGraph::create / build / search / save / load      (kgraph.h:155-228)
//   MatrixOracle<Matrix<float>, metric::l2sqr>           (kgraph-data.h:302-331)
// Test infrastructure only: never linked into the product library.
#include <cstring>
#include <cstdio>
#include <memory>
#include <stdexcept>
#include <string>
#include <omp.h>
#include "kgraph.h"
#include "kgraph-data.h"

using kgraph::KGraph;
typedef kgraph::MatrixOracle<float, kgraph::metric::l2sqr> L2Oracle;

static thread_local std::string g_err;

static void fill_matrix(kgraph::Matrix<float> &m, const float *data, unsigned n, unsigned d) {
    m.resize(n, d);
    m.zero();
    for (unsigned i = 0; i < n; ++i) std::memcpy(m[i], data + (size_t)i * d, sizeof(float) * d);
}

extern "C" {

const char *kgref_last_error() { return g_err.c_str(); }

void kgref_set_verbosity(unsigned v) { kgraph::verbosity = v; }

void kgref_set_threads(int t) { if (t > 0) omp_set_num_threads(t); }

// Builds an index over rows `data` (n x d, dense) with the C++ MatrixOracle
// (full squared L2) and saves it to `index_path`.  info_out (7 floats):
// stop_condition, iterations, cost, recall, accuracy, delta, M.
int kgref_build_l2sqr(const float *data, unsigned n, unsigned d,
                      unsigned iterations, unsigned L, unsigned K, unsigned S, unsigned R,
                      unsigned controls, unsigned seed, float delta, float recall,
                      unsigned prune, int reverse, const char *index_path, float *info_out) {
    try {
        kgraph::Matrix<float> m;
        fill_matrix(m, data, n, d);
        L2Oracle oracle(m);
        KGraph::IndexParams p;
        p.iterations = iterations; p.L = L; p.K = K; p.S = S; p.R = R;
        p.controls = controls; p.seed = seed; p.delta = delta; p.recall = recall;
        p.prune = prune; p.reverse = reverse;
        KGraph::IndexInfo info;
        std::unique_ptr<KGraph> index(KGraph::create());
        index->build(oracle, p, &info);
        index->save(index_path);
        if (info_out) {
            info_out[0] = (float)info.stop_condition; info_out[1] = (float)info.iterations;
            info_out[2] = info.cost; info_out[3] = info.recall; info_out[4] = info.accuracy;
            info_out[5] = info.delta; info_out[6] = info.M;
        }
        return 0;
    } catch (std::exception const &e) { g_err = e.what(); return 1; }
}

// Searches nq queries against an index file with MatrixOracle (full squared
// L2).  Output rows are K wide; counts[q] = returned results, costs[q] =
// SearchInfo.cost.  ids is also the input of `init` starting points.
int kgref_search_l2sqr(const float *data, unsigned n, unsigned d, const char *index_path,
                       const float *queries, unsigned nq,
                       unsigned K, unsigned P, unsigned M, unsigned S, unsigned T,
                       float epsilon, unsigned seed, unsigned init,
                       unsigned *ids, float *dists, unsigned *counts, float *costs, int threads) {
    try {
        kgraph::Matrix<float> m, q;
        fill_matrix(m, data, n, d);
        fill_matrix(q, queries, nq, d);
        L2Oracle oracle(m);
        std::unique_ptr<KGraph> index(KGraph::create());
        index->load(index_path);
        KGraph::SearchParams p;
        p.K = K; p.P = P; p.M = M; p.S = S; p.T = T; p.epsilon = epsilon; p.seed = seed; p.init = init;
        int err = 0;
        std::string msg;
        if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 16)
        for (unsigned i = 0; i < nq; ++i) {
            try {
                KGraph::SearchInfo info;
                counts[i] = index->search(oracle.query(q[i]), p, ids + (size_t)i * K,
                                          dists + (size_t)i * K, &info);
                costs[i] = info.cost;
            } catch (std::exception const &e) {
#pragma omp critical
                { err = 1; msg = e.what(); }
            }
        }
        if (err) { g_err = msg; return 1; }
        return 0;
    } catch (std::exception const &e) { g_err = e.what(); return 1; }
}

// LSHKIT matrix I/O through the reference's own Matrix<float>
// (kgraph-data.h:193-218): write n x d rows, or read a file's shape (data ==
// NULL) and then its rows.
int kgref_save_lshkit(const float *data, unsigned n, unsigned d, const char *path) {
    try {
        kgraph::Matrix<float> m;
        fill_matrix(m, data, n, d);
        m.save_lshkit(path);
        return 0;
    } catch (std::exception const &e) { g_err = e.what(); return 1; }
}
int kgref_load_lshkit(const char *path, float *data, unsigned *n, unsigned *d) {
    try {
        kgraph::Matrix<float> m;
        m.load_lshkit(path);
        *n = m.size();
        *d = m.dim();
        if (data)
            for (unsigned i = 0; i < m.size(); ++i) std::memcpy(data + (size_t)i * m.dim(), m[i], sizeof(float) * m.dim());
        return 0;
    } catch (std::exception const &e) { g_err = e.what(); return 1; }
}

// Loads an index file with the reference's loader and saves it again with its
// saver in `format` (KGraph::FORMAT_DEFAULT / FORMAT_NO_DIST / FORMAT_TEXT,
// kgraph.cpp:291-373): the reference's own files in every format it writes.
int kgref_resave(const char *in_path, const char *out_path, int format) {
    try {
        std::unique_ptr<KGraph> index(KGraph::create());
        index->load(in_path);
        index->save(out_path, format);
        return 0;
    } catch (std::exception const &e) { g_err = e.what(); return 1; }
}

// Reads an index file through the reference's loader and returns its CSR
// form: offsets[n+1], ids/dists[E], M[n].  Call once with ids == NULL to get
// n and E.
int kgref_load_graph(const char *index_path, unsigned *n_out, unsigned long long *e_out,
                     unsigned long long *offsets, unsigned *ids, float *dists, unsigned *Ms) {
    try {
        std::unique_ptr<KGraph> index(KGraph::create());
        index->load(index_path);
        // get_nn reports L per node; walk to find n.
        unsigned n = 0;
        unsigned long long e = 0;
        std::vector<unsigned> tmp_ids(1 << 20);
        std::vector<float> tmp_d(1 << 20);
        for (;; ++n) {
            unsigned Mv, Lv;
            try { index->get_nn(n, nullptr, nullptr, &Mv, &Lv); }
            catch (std::exception const &) { break; }
            if (offsets) offsets[n] = e;
            if (ids) {
                index->get_nn(n, ids + e, dists ? dists + e : nullptr, &Mv, &Lv);
                Ms[n] = Mv;
            }
            e += Lv;
        }
        if (offsets) offsets[n] = e;
        *n_out = n; *e_out = e;
        return 0;
    } catch (std::exception const &e) { g_err = e.what(); return 1; }
}

}
