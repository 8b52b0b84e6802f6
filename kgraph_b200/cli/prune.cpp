// `prune`: loads an index, prunes it and saves it -- the reference's prune
// tool (prune.cpp), same options and defaults, on kgraph-b200's C++ API.
//
//   prune [OPTIONS] DATA INPUT [OUTPUT]
//
// DATA is an LSHKIT float32 matrix (or, with --raw, a headerless file read
// with --dim, --skip, --gap); the index is pruned with KGraph::prune
// (kgraph.cpp:584-665).  The default level is the reference tool's
// PRUNE_LEVEL_1 & PRUNE_LEVEL_2, which is 0 (no pruning) -- kept as it is.
#include <kgraph.h>
#include <kgraph-data.h>
#include <chrono>
#include <iostream>
#include <memory>
#include "cli_args.h"

using namespace kgraph;

int main(int argc, char **argv) {
    kgcli::Args a;
    try {
        a = kgcli::parse(argc, argv, {"data", "input", "output", "prune", "dim", "skip", "gap"},
                         {{"h", "help"}, {"D", "dim"}}, {"help", "raw"});
    } catch (std::exception const &e) {
        std::cerr << e.what() << std::endl;
        return 1;
    }
    const char *pos_names[] = {"data", "input", "output"};
    for (size_t p = 0; p < a.positional.size() && p < 3; ++p)
        if (!a.has(pos_names[p])) a.values[pos_names[p]] = a.positional[p];
    if (a.has("help") || !a.has("input")) {
        std::cout << "Usage: prune [OTHER OPTIONS]... DATA INPUT [OUTPUT]\n"
                     "General options:\n  -h [ --help ]         produce help message.\n"
                     "  --data arg            input path\n  --input arg           input index path\n"
                     "  --output arg          output index path\n  --prune arg (=0)      prune level\n"
                     "Expert options:\n  -D [ --dim ] arg      dimension, see format\n"
                     "  --skip arg (=0)       see format\n  --gap arg (=0)        see format\n"
                     "  --raw                 read raw binary file, need to specify D.\n";
        return 0;
    }
    const unsigned level = a.u("prune", PRUNE_LEVEL_1 & PRUNE_LEVEL_2);
    try {
        Matrix<float> data;
        if (a.has("raw")) data.load(a.str("data"), a.u("dim", 0), a.u("skip", 0), a.u("gap", 0));
        else data.load_lshkit(a.str("data"));
        MatrixOracle<float, metric::l2sqr> oracle(data);
        std::unique_ptr<KGraph> index(KGraph::create());
        index->load(a.str("input").c_str());
        const auto t0 = std::chrono::steady_clock::now();
        index->prune(oracle, level);
        std::cerr << " " << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() << "s wall"
                  << std::endl;
        if (a.has("output")) index->save(a.str("output").c_str());
    } catch (std::exception const &e) {
        std::cerr << "error: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
