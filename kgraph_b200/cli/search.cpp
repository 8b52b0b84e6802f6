// `search`: k-NN search of a query file against a saved index -- the
// reference's search tool (search.cpp) with the same options, input and
// output formats and summary line, on kgraph-b200's C++ API: the whole query
// file is one batched GPU search (KGraph::search_batch) instead of one
// OpenMP thread per query (search.cpp:139-146).
//
//   search [OPTIONS] DATA INDEX QUERY [OUTPUT]
//
// DATA and QUERY are LSHKIT float32 matrices; OUTPUT (optional) receives the
// result ids as an LSHKIT uint32 matrix of K columns.  --eval GS scores the
// result against a gold-standard LSHKIT uint32 matrix by distance value
// (AverageRecall); --linear runs the exact brute force instead of the graph
// (SearchOracle::search, cost 1); --init takes starting points from an
// LSHKIT uint32 matrix -- as in the reference, its column count becomes
// SearchParams.init and must be >= K (search.cpp:97-98), which the search
// then rejects (init must be < K, kgraph.cpp:461-463): the reference tool's
// behaviour, kept.  The oracle is MatrixOracle<float, metric::l2sqr>.
#include <kgraph.h>
#include <kgraph-data.h>
#include <kgraph_b200.h>
#include <algorithm>
#include <chrono>
#include <iostream>
#include <memory>
#include <vector>
#include "cli_args.h"

using namespace kgraph;

static void usage() {
    std::cout << "search <data> <index> <query> [output]\n"
                 "General options:\n"
                 "  -h [ --help ]         produce help message.\n"
                 "  -v [ --version ]      print version number.\n"
                 "  --data arg            input path\n  --index arg           index path\n"
                 "  --query arg           query path\n  --output arg          output path\n"
                 "  --init arg            init path\n  --eval arg            eval path\n"
                 "  -K arg (=25)\n  -M arg (=0)\n  -P arg (=100)\n  -S arg (=10)\n  -T arg (=1)\n"
                 "  --linear\n"
                 "  --l2norm              l2-normalize data, so as to mimic cosine similarity\n";
}

int main(int argc, char **argv) {
    kgcli::Args a;
    try {
        a = kgcli::parse(argc, argv, {"data", "index", "query", "output", "init", "eval", "K", "M", "P", "S", "T"},
                         {{"h", "help"}, {"v", "version"}}, {"help", "version", "linear", "l2norm"});
    } catch (std::exception const &e) {
        std::cerr << e.what() << std::endl;
        return 1;
    }
    const char *pos_names[] = {"data", "index", "query", "output"};
    for (size_t p = 0; p < a.positional.size() && p < 4; ++p)
        if (!a.has(pos_names[p])) a.values[pos_names[p]] = a.positional[p];
    if (a.has("version")) {
        std::cout << "KGraph version " << KGraph::version() << std::endl;
        return 0;
    }
    if (a.has("help") || !a.has("data") || !a.has("index") || !a.has("query")) {
        usage();
        return 0;
    }
    unsigned K = a.u("K", default_K), M = a.u("M", default_M), P = a.u("P", default_P), S = a.u("S", default_S),
             T = a.u("T", default_T);
    if (P < K) P = K;   // search.cpp:81-83
    try {
        Matrix<float> data, query;
        Matrix<unsigned> result;
        unsigned init = 0;
        data.load_lshkit(a.str("data"));
        query.load_lshkit(a.str("query"));
        if (a.has("init")) {
            result.load_lshkit(a.str("init"));
            if (result.size() != query.size()) throw invalid_argument("init rows != query rows");
            init = result.dim();
            if (init < K) throw invalid_argument("init columns must be >= K");
        }
        if (a.has("l2norm")) {
            std::cerr << "L2-normalizing data..." << std::endl;
            data.normalize2();
            query.normalize2();
        }
        MatrixOracle<float, metric::l2sqr> oracle(data);
        const unsigned nq = query.size();
        std::vector<unsigned> ids((size_t)nq * K, 0), counts(nq, 0);
        std::vector<float> costs(nq, 0.f);
        float cost = 0, recall = 0;
        double time = 0;
        if (a.has("linear")) {   // exact brute force on the GPU: a context with the dataset and no graph
            kg_ctx *ctx = nullptr;
            if (kg_ctx_create(0, &ctx) != KG_OK) throw runtime_error("cannot create a GPU context");
            std::unique_ptr<kg_ctx, void (*)(kg_ctx *)> hold(ctx, kg_ctx_destroy);
            if (kg_set_data(ctx, data[0], data.size(), data.dim(), data.step(), KG_METRIC_L2SQR) != KG_OK)
                throw runtime_error(kg_last_error(ctx));
            kg_search_params sp;
            kg_search_params_default(&sp);
            sp.K = K;
            const auto t0 = std::chrono::steady_clock::now();
            if (kg_search_batch(ctx, query[0], nq, query.step(), &sp, nullptr, nullptr, K, ids.data(), nullptr,
                                counts.data(), nullptr) != KG_OK)
                throw runtime_error(kg_last_error(ctx));
            time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            cost = 1.0f;
        } else {
            KGraph::SearchParams params;
            params.K = K; params.M = M; params.P = P; params.S = S; params.T = T; params.init = init;
            std::unique_ptr<KGraph> index(KGraph::create());
            index->load(a.str("index").c_str());
            if (init)   // the starting points ride in the ids buffer (the reference passes result rows)
                for (unsigned i = 0; i < nq; ++i)
                    for (unsigned k = 0; k < K; ++k) ids[(size_t)i * K + k] = result[i][k];
            std::cerr << "Searching..." << std::endl;
            const auto t0 = std::chrono::steady_clock::now();
            index->search_batch(oracle, query[0], nq, query.step(), params, ids.data(), nullptr, counts.data(),
                                costs.data());
            time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            double c = 0;
            for (float x : costs) c += x;
            cost = nq ? (float)(c / nq) : 0.f;
        }
        result.resize(nq, K);
        for (unsigned i = 0; i < nq; ++i)
            for (unsigned k = 0; k < K; ++k) result[i][k] = ids[(size_t)i * K + k];
        if (a.has("output")) result.save_lshkit(a.str("output"));
        if (a.has("eval")) {   // search.cpp:157-182: recall by distance value
            Matrix<unsigned> gs;
            gs.load_lshkit(a.str("eval"));
            if (gs.dim() < K || gs.size() < nq) throw invalid_argument("gold standard too small");
            Matrix<float> gs_dist(nq, K), result_dist(nq, K);
            for (unsigned i = 0; i < nq; ++i) {
                auto Q = oracle.query(query[i]);
                for (unsigned k = 0; k < K; ++k) {
                    gs_dist[i][k] = Q(gs[i][k]);
                    result_dist[i][k] = Q(result[i][k]);
                }
                std::sort(gs_dist[i], gs_dist[i] + K);
                std::sort(result_dist[i], result_dist[i] + K);
            }
            recall = AverageRecall(gs_dist, result_dist, K);
        }
        std::cout << "Time: " << time << " Recall: " << recall << " Cost: " << cost << std::endl;
    } catch (std::exception const &e) {
        std::cerr << "error: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
