// `index`: builds a k-NN graph index with the GPU NN-descent and saves it --
// the reference's index tool (index.cpp) with the same options, defaults,
// input formats and output, on kgraph-b200's C++ API (include/kgraph.h).
//
//   index [OPTIONS] INPUT [OUTPUT]
//
// INPUT is an LSHKIT matrix (header: element size, rows, cols; then rows of
// float32), or with --raw a headerless float32 file read with --dim, --skip and
// --gap (kgraph-data.h Matrix::load); --synthetic N generates N uniform
// [-1, 1) rows of --dim instead (std::default_random_engine(seed), as
// index.cpp:117-131).  --noise adds Gaussian noise of noise x the data's
// standard deviation (index.cpp:135-157), --l2norm L2-normalises every row.
// The oracle is MatrixOracle<float, metric::l2sqr>, the reference tool's.
#include <kgraph.h>
#include <kgraph-data.h>
#include <chrono>
#include <cmath>
#include <fstream>
#include <iostream>
#include <memory>
#include <random>
#include "cli_args.h"

using namespace kgraph;

static void usage() {
    std::cout << "Usage: index [OTHER OPTIONS]... INPUT [OUTPUT]\n"
                 "General options:\n"
                 "  -h [ --help ]            produce help message.\n"
                 "  -v [ --version ]         print version information.\n"
                 "  --data arg               input path\n"
                 "  --output arg             output path\n"
                 "  -K arg (=25)             number of nearest neighbor\n"
                 "  -C [ --controls ] arg (=100) number of control points\n"
                 "Expert options:\n"
                 "  -I [ --iterations ] arg (=30)\n"
                 "  -S arg (=10)\n  -R arg (=100)\n  -L arg (=100)\n"
                 "  --delta arg (=0.002)\n  --recall arg (=0.99)\n  --prune arg (=0)\n  --reverse arg (=0)\n"
                 "  --noise arg (=0)         noise\n  --seed arg (=1998)\n"
                 "  -D [ --dim ] arg         dimension, see format\n"
                 "  --skip arg (=0)          see format\n  --gap arg (=0)           see format\n"
                 "  --raw                    read raw binary file, need to specify D.\n"
                 "  --synthetic arg (=0)     generate synthetic data, for performance evaluation only, specify "
                 "number of points\n"
                 "  --l2norm                 l2-normalize data, so as to mimic cosine similarity\n";
}

int main(int argc, char **argv) {
    kgcli::Args a;
    try {
        a = kgcli::parse(argc, argv,
                         {"data", "output", "K", "controls", "iterations", "S", "R", "L", "delta", "recall", "prune",
                          "reverse", "noise", "seed", "dim", "skip", "gap", "synthetic"},
                         {{"h", "help"}, {"v", "version"}, {"C", "controls"}, {"I", "iterations"}, {"D", "dim"}},
                         {"help", "version", "raw", "l2norm"});
    } catch (std::exception const &e) {
        std::cerr << e.what() << std::endl;
        return 1;
    }
    if (!a.positional.empty() && !a.has("data")) a.values["data"] = a.positional[0];
    if (a.positional.size() > 1 && !a.has("output")) a.values["output"] = a.positional[1];
    const bool lshkit = !a.has("raw");
    if (a.has("version")) {
        std::cout << "KGraph version " << KGraph::version() << std::endl;
        return 0;
    }
    KGraph::IndexParams params;
    params.K = a.u("K", default_K);
    params.controls = a.u("controls", default_controls);
    params.iterations = a.u("iterations", default_iterations);
    params.S = a.u("S", default_S);
    params.R = a.u("R", default_R);
    params.L = a.u("L", default_L);
    params.delta = a.f("delta", default_delta);
    params.recall = a.f("recall", default_recall);
    params.prune = a.u("prune", default_prune);
    params.reverse = a.i("reverse", default_reverse);
    params.seed = a.u("seed", default_seed);
    const float noise = a.f("noise", 0.f);
    const unsigned synthetic = a.u("synthetic", 0);
    unsigned D = a.u("dim", 0), skip = a.u("skip", 0), gap = a.u("gap", 0);
    const std::string data_path = a.str("data"), output_path = a.str("output");
    if (a.has("help") || (synthetic && (!a.has("dim") || a.has("data"))) ||
        (!synthetic && (!a.has("data") || (!a.has("dim") && !lshkit)))) {
        usage();
        return 0;
    }
    if (params.S == 0) params.S = params.K;   // index.cpp:101-103
    try {
        Matrix<float> data;
        if (synthetic) {
            data.resize(synthetic, D);
            std::cerr << "Generating synthetic data..." << std::endl;
            std::default_random_engine rng(params.seed);
            std::uniform_real_distribution<double> distribution(-1.0, 1.0);
            data.zero();
            for (unsigned i = 0; i < synthetic; ++i)
                for (unsigned j = 0; j < D; ++j) data[i][j] = distribution(rng);
        } else if (lshkit) {
            data.load_lshkit(data_path);
        } else {
            data.load(data_path, D, skip, gap);
        }
        if (noise != 0) {
            std::default_random_engine rng;
            double sum = 0, sum2 = 0;
            for (unsigned i = 0; i < data.size(); ++i)
                for (unsigned j = 0; j < data.dim(); ++j) {
                    double v = data[i][j];
                    sum += v;
                    sum2 += v * v;
                }
            const double total = double(data.size()) * data.dim();
            const double avg2 = sum2 / total, avg = sum / total;
            const double dev = std::sqrt(avg2 - avg * avg);
            std::cerr << "Adding Gaussian noise w/ " << noise << "x sigma(" << dev << ")..." << std::endl;
            std::normal_distribution<double> gaussian(0, noise * dev);
            for (unsigned i = 0; i < data.size(); ++i)
                for (unsigned j = 0; j < data.dim(); ++j) data[i][j] += gaussian(rng);
        }
        if (a.has("l2norm")) {
            std::cerr << "L2-normalizing data..." << std::endl;
            data.normalize2();
        }
        MatrixOracle<float, metric::l2sqr> oracle(data);
        KGraph::IndexInfo info;
        std::unique_ptr<KGraph> index(KGraph::create());
        const auto t0 = std::chrono::steady_clock::now();
        index->build(oracle, params, &info);
        std::cerr << info.stop_condition << std::endl;
        const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::cerr << " " << wall << "s wall" << std::endl;
        if (!output_path.empty()) index->save(output_path.c_str());
    } catch (std::exception const &e) {
        std::cerr << "error: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
