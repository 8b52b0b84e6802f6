// Uses kgraph-b200 exactly as code written for the reference's C++ API would:
// kgraph.h / kgraph-data.h, KGraph::create, build, search, save, load, get_nn.
// Prints one line of results for the test to compare.
#include <kgraph.h>
#include <kgraph-data.h>
#include <cstdio>
#include <memory>
#include <random>
#include <vector>

int main(int argc, char **argv) {
    const char *path = argc > 1 ? argv[1] : "/tmp/api_demo.kgraph";
    unsigned n = 5000, d = 24;
    kgraph::Matrix<float> data(n, d);
    std::mt19937 rng(7);
    std::uniform_real_distribution<float> u(0, 1);
    for (unsigned i = 0; i < n; ++i)
        for (unsigned j = 0; j < d; ++j) data[i][j] = u(rng);
    kgraph::MatrixOracle<float, kgraph::metric::l2sqr> oracle(data);
    kgraph::verbosity = 0;
    std::unique_ptr<kgraph::KGraph> index(kgraph::KGraph::create());
    kgraph::KGraph::IndexParams ip;
    ip.K = 10; ip.L = 30; ip.S = 8; ip.reverse = -1;
    kgraph::KGraph::IndexInfo info;
    index->build(oracle, ip, &info);
    index->save(path);
    std::unique_ptr<kgraph::KGraph> again(kgraph::KGraph::create());
    again->load(path);
    kgraph::KGraph::SearchParams sp;
    sp.K = 5; sp.P = 40;
    std::vector<unsigned> ids(sp.K), ids2(sp.K), bf(sp.K);
    std::vector<float> ds(sp.K), bd(sp.K);
    kgraph::KGraph::SearchInfo si;
    unsigned c1 = index->search(oracle.query(data[17]), sp, ids.data(), ds.data(), &si);
    unsigned c2 = again->search(oracle.query(data[17]), sp, ids2.data(), nullptr, nullptr);
    unsigned c3 = oracle.query(data[17]).search(sp.K, 1e30f, bf.data(), bd.data());
    unsigned M, L;
    std::vector<unsigned> nn(1000);
    again->get_nn(17, nn.data(), &M, &L);
    bool bad_oracle = false;
    try {
        std::vector<std::vector<float>> v(10, std::vector<float>(4, 0.f));
        kgraph::VectorOracle<std::vector<std::vector<float>>, std::vector<float>> vo(
            v, [](std::vector<float> const &, std::vector<float> const &) { return 0.f; });
        index->build(vo, ip);
    } catch (kgraph::invalid_argument const &) { bad_oracle = true; }
    std::printf("iterations=%u stop=%d c1=%u c2=%u c3=%u first=%u,%u,%u self_dist=%g cost=%g M=%u L=%u "
                "same=%d rejects_vector_oracle=%d\n",
                info.iterations, (int)info.stop_condition, c1, c2, c3, ids[0], ids2[0], bf[0], ds[0], si.cost, M, L,
                (int)(ids == ids2 && ids == bf), (int)bad_oracle);
    return 0;
}
