// `resave`: loads an index and saves it again, optionally pruned and/or
// without distances -- the reference's resave tool (resave.cpp), same options,
// on kgraph-b200's C++ API.
//
//   resave [--prune LEVEL] [--no-dist] INPUT [OUTPUT]
//
// Pruning needs only the graph's own distances (KGraph::prune,
// kgraph.cpp:584-665); as in the reference tool, no dataset is read.
#include <kgraph.h>
#include <iostream>
#include <memory>
#include "cli_args.h"

using namespace kgraph;

namespace {
// The reference tool prunes through an oracle that must never be called.
class NoDataOracle : public IndexOracle {
public:
    unsigned size() const override { throw runtime_error("resave: no dataset"); }
    float operator()(unsigned, unsigned) const override { throw runtime_error("resave: no dataset"); }
};
}  // namespace

int main(int argc, char **argv) {
    kgcli::Args a;
    try {
        a = kgcli::parse(argc, argv, {"input", "output", "prune"}, {{"h", "help"}}, {"help", "no-dist"});
    } catch (std::exception const &e) {
        std::cerr << e.what() << std::endl;
        return 1;
    }
    const char *pos_names[] = {"input", "output"};
    for (size_t p = 0; p < a.positional.size() && p < 2; ++p)
        if (!a.has(pos_names[p])) a.values[pos_names[p]] = a.positional[p];
    if (a.has("help") || !a.has("input")) {
        std::cout << "General options:\n  -h [ --help ]         produce help message.\n  --input arg\n  --output arg\n"
                     "  --prune arg\n  --no-dist\n";
        return 0;
    }
    int format = KGraph::FORMAT_DEFAULT;
    if (a.has("no-dist")) format |= KGraph::FORMAT_NO_DIST;
    try {
        std::unique_ptr<KGraph> index(KGraph::create());
        index->load(a.str("input").c_str());
        if (a.has("prune")) {
            NoDataOracle o;
            index->prune(o, a.u("prune", 0));
        }
        if (a.has("output")) index->save(a.str("output").c_str(), format);
    } catch (std::exception const &e) {
        std::cerr << "error: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
