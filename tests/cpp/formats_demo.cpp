// Index file formats through kgraph-b200's C++ API (KGraph::save / load,
// kgraph.cpp:291-373 of the reference):
//   argv[1] an index file in the default format (written by the reference)
//   argv[2] <- that index saved as FORMAT_TEXT
//   argv[3] <- that index saved as FORMAT_NO_DIST
//   argv[4] an index file in FORMAT_NO_DIST (written by the reference)
//   argv[5] <- argv[4] loaded and saved again as FORMAT_NO_DIST
//   argv[6] dataset (raw float32, n x d), argv[7] n, argv[8] d,
//   argv[9] queries (raw float32, nq x d), argv[10] nq, argv[11] K, argv[12] P
//   argv[13] <- ids (raw uint32, nq x K) of a search of argv[4]'s graph
// Prints which operations a graph without distances refuses.
#include <kgraph.h>
#include <kgraph-data.h>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <vector>

static std::vector<float> read_f32(const char *path, size_t count) {
    std::vector<float> v(count);
    std::ifstream is(path, std::ios::binary);
    is.read(reinterpret_cast<char *>(v.data()), count * sizeof(float));
    return v;
}

int main(int argc, char **argv) {
    if (argc < 14) return 2;
    using kgraph::KGraph;
    std::unique_ptr<KGraph> a(KGraph::create());
    a->load(argv[1]);
    a->save(argv[2], KGraph::FORMAT_TEXT);
    a->save(argv[3], KGraph::FORMAT_NO_DIST);
    std::unique_ptr<KGraph> b(KGraph::create());
    b->load(argv[4]);
    b->save(argv[5], KGraph::FORMAT_NO_DIST);
    const unsigned n = (unsigned)std::atoi(argv[7]), d = (unsigned)std::atoi(argv[8]);
    const unsigned nq = (unsigned)std::atoi(argv[10]), K = (unsigned)std::atoi(argv[11]), P = (unsigned)std::atoi(argv[12]);
    std::vector<float> X = read_f32(argv[6], (size_t)n * d), Q = read_f32(argv[9], (size_t)nq * d);
    kgraph::DenseMatrixOracle oracle(X.data(), n, d, d * sizeof(float), 0);
    KGraph::SearchParams sp;
    sp.K = K;
    sp.P = P;
    std::vector<unsigned> ids((size_t)nq * K, 0);
    b->search_batch(oracle, Q.data(), nq, d * sizeof(float), sp, ids.data(), nullptr, nullptr, nullptr);
    std::ofstream os(argv[13], std::ios::binary);
    os.write(reinterpret_cast<const char *>(ids.data()), ids.size() * sizeof(unsigned));
    bool no_dists = false, no_reverse = false;
    unsigned M, L;
    std::vector<unsigned> nn(4096);
    std::vector<float> dd(4096);
    try { b->get_nn(0, nn.data(), dd.data(), &M, &L); } catch (kgraph::runtime_error const &) { no_dists = true; }
    try { b->reverse(-1); } catch (kgraph::runtime_error const &) { no_reverse = true; }
    b->get_nn(0, nn.data(), &M, &L);   // ids alone are available
    std::printf("refuses_dists=%d refuses_reverse=%d L0=%u\n", (int)no_dists, (int)no_reverse, L);
    return 0;
}
