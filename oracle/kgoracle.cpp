// CPU restatement of KGraph's hot paths -- TEST INFRASTRUCTURE ONLY (the
// checker).  See kgoracle.h for the contract and the parity pin.  Compiled
// with -ffp-contract=off so that every fused multiply-add below is an explicit
// std::fma where the reference's compiled code performs one, and nothing else
// is fused.
#include "kgoracle.h"
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <limits>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

std::string g_err;

// ---------------------------------------------------------------- distances
// xsimd avx512f reduce_add (xsimd_avx512f.hpp: four 128-bit quarters added
// pairwise, then the sse3 hadd pair): lane k of the 4-wide sum is
// (x_k + x_{k+4}) + (x_{k+8} + x_{k+12}); the result (t0 + t1) + (t2 + t3).
inline float reduce16(const float *x) {
    float t[4];
    for (int k = 0; k < 4; ++k) t[k] = (x[k] + x[k + 4]) + (x[k + 8] + x[k + 12]);
    return (t[0] + t[1]) + (t[2] + t[3]);
}

// kgraph-data.h:65-83
float dot_impl(const float *a, const float *b, unsigned d) {
    float acc[16] = {0};
    unsigned vs = d - d % 16, i = 0;
    for (; i < vs; i += 16)
        for (int l = 0; l < 16; ++l) acc[l] = acc[l] + a[i + l] * b[i + l];
    float r = reduce16(acc);
    if (d - i >= 8)   // the compiler vectorises 8 tail products: rounded, added in order
        for (unsigned e = i + 8; i < e; ++i) r = r + a[i] * b[i];
    for (; i < d; ++i) r = std::fma(a[i], b[i], r);
    return r;
}

// kgraph-data.h:87-103
float norm2_impl(const float *a, unsigned d) {
    float acc[16] = {0};
    unsigned vs = d - d % 16, i = 0;
    for (; i < vs; i += 16)
        for (int l = 0; l < 16; ++l) acc[l] = acc[l] + a[i + l] * a[i + l];
    float r = reduce16(acc);
    if (d - i >= 8)
        for (unsigned e = i + 8; i < e; ++i) r = r + a[i] * a[i];
    for (; i < d; ++i) r = std::fma(a[i], a[i], r);
    return r;
}

// kgraph-data.h:41-61
float l2sqr_impl(const float *a, const float *b, unsigned d) {
    float acc[16] = {0};
    unsigned vs = d - d % 16, i = 0;
    for (; i < vs; i += 16)
        for (int l = 0; l < 16; ++l) {
            float t = a[i + l] - b[i + l];
            acc[l] = acc[l] + t * t;
        }
    float r = reduce16(acc);
    if (d - i >= 8)
        for (unsigned e = i + 8; i < e; ++i) {
            float t = a[i] - b[i];
            r = r + t * t;
        }
    for (; i < d; ++i) {
        float t = a[i] - b[i];
        r = std::fma(t, t, r);
    }
    return r;
}

// python-api.cpp:51-69 norm / dist
inline float metric_norm(const float *x, unsigned d, int metric) {
    if (metric == KGO_EUCLIDEAN) return norm2_impl(x, d) / 2;
    if (metric == KGO_ANGULAR) return std::sqrt(norm2_impl(x, d));
    return 0.0f;
}
inline float metric_dist(float dot, float n1, float n2, int metric) {
    if (metric == KGO_EUCLIDEAN) return (n1 + n2) - dot;
    // -dot / (n1*n2 + eps): the product and the add are fused (FP contraction).
    return -dot / std::fma(n1, n2, std::numeric_limits<float>::epsilon());
}

struct Data {
    const float *X; const float *norms; unsigned n, d; int metric;
    const float *row(unsigned i) const { return X + (size_t)i * d; }
    float operator()(unsigned i, unsigned j) const {
        if (metric == KGO_L2SQR) return l2sqr_impl(row(i), row(j), d);
        return metric_dist(dot_impl(row(i), row(j), d), norms[i], norms[j], metric);
    }
};
struct Query {
    const Data &D; const float *q; float qn;
    float operator()(unsigned i) const {
        if (D.metric == KGO_L2SQR) return l2sqr_impl(D.row(i), q, D.d);
        return metric_dist(dot_impl(D.row(i), q, D.d), D.norms[i], qn, D.metric);
    }
};

// ---------------------------------------------------------------- lists
struct Neighbor { uint32_t id; float dist; bool flag; };
struct NeighborX { uint32_t id; float dist; bool flag; uint16_t m; uint16_t M; };

// Entries no insert has written yet (the reference leaves them
// indeterminate): defined here as an id no node has and +FLT_MAX.
inline Neighbor unset_neighbor() { return Neighbor{0xFFFFFFFFu, FLT_MAX, false}; }

inline bool less_dist(const Neighbor &a, const Neighbor &b) { return a.dist < b.dist; }

// UpdateKnnListHelper, kgraph.cpp:176-202
template <typename T>
unsigned update_knn_list(T *addr, unsigned K, T nn) {
    unsigned j, i = K;
    while (i > 0) {
        j = i - 1;
        if (addr[j].dist <= nn.dist) break;
        i = j;
    }
    unsigned l = i;
    while (l > 0) {
        j = l - 1;
        if (addr[j].dist < nn.dist) break;
        if (addr[j].id == nn.id) return K + 1;
        l = j;
    }
    j = K;
    while (j > i) { addr[j] = addr[j - 1]; --j; }
    addr[i] = nn;
    return i;
}

// GenRandom, kgraph.cpp:44-65
template <typename RNG>
void gen_random(RNG &rng, unsigned *addr, unsigned size, unsigned N) {
    if (N == size) {
        for (unsigned i = 0; i < size; ++i) addr[i] = i;
        return;
    }
    for (unsigned i = 0; i < size; ++i) addr[i] = rng() % (N - size);
    std::sort(addr, addr + size);
    for (unsigned i = 1; i < size; ++i)
        if (addr[i] <= addr[i - 1]) addr[i] = addr[i - 1] + 1;
    unsigned off = rng() % N;
    for (unsigned i = 0; i < size; ++i) addr[i] = (addr[i] + off) % N;
}

struct Graph {
    std::vector<std::vector<Neighbor>> adj;
    std::vector<uint32_t> M;
};
Graph g_result;

uint64_t store_result(Graph &&g) { g_result = std::move(g); uint64_t e = 0; for (auto &v : g_result.adj) e += v.size(); return e; }

// KGraphImpl::reverse, kgraph.cpp:667-702
void reverse_graph(Graph &g, int rev_k) {
    if (rev_k == 0) return;
    unsigned N = g.adj.size();
    std::vector<std::vector<Neighbor>> ng(N);
    for (unsigned i = 0; i < N; ++i) {
        auto const &v = g.adj[i];
        unsigned K = g.M[i];
        if (rev_k > 0) { K = rev_k; if (K > v.size()) K = v.size(); }
        for (unsigned j = 0; j < K; ++j) {
            auto const &e = v[j];
            auto re = e;
            re.id = i;
            ng[i].push_back(e);
            ng[e.id].push_back(re);
        }
    }
    g.adj.swap(ng);
    for (unsigned i = 0; i < N; ++i) {
        auto &v = g.adj[i];
        std::sort(v.begin(), v.end(), less_dist);
        v.resize(std::unique(v.begin(), v.end(),
                             [](const Neighbor &a, const Neighbor &b) { return a.id == b.id; }) - v.begin());
        g.M[i] = v.size();
    }
}

// prune1 / prune2, kgraph.cpp:584-656
void prune1(Graph &g) {
    for (unsigned i = 0; i < g.adj.size(); ++i)
        if (g.adj[i].size() > g.M[i]) g.adj[i].resize(g.M[i]);
}
void prune2(Graph &g) {
    unsigned N = g.adj.size();
    std::vector<std::vector<unsigned>> rev(N);
    std::vector<uint32_t> new_L(N, 0);
    for (unsigned i = 0; i < N; ++i)
        for (auto &e : g.adj[i]) e.flag = false;
    std::vector<unsigned> todo(N), new_todo;
    for (unsigned i = 0; i < N; ++i) todo[i] = i;
    for (unsigned l = 0; todo.size(); ++l) {
        new_todo.clear();
        for (unsigned i : todo) {
            if (l >= g.M[i]) continue;
            new_todo.push_back(i);
            auto &v = g.adj[i];
            if (v[l].flag) continue;
            v[l].flag = true;
            unsigned T;
            {
                auto &nl = new_L[i];
                T = v[nl].id = v[l].id;
                v[nl].dist = v[l].dist;
                ++nl;
            }
            rev[T].push_back(i);
            {
                auto const &u = g.adj[T];
                for (unsigned ll = l + 1; ll < g.M[i]; ++ll) {
                    if (v[ll].flag) continue;
                    for (unsigned j = 0; j < new_L[T]; ++j)
                        if (v[ll].id == u[j].id) { v[ll].flag = true; break; }
                }
            }
            for (auto r : rev[i]) {
                auto &u = g.adj[r];
                for (unsigned ll = l; ll < g.M[r]; ++ll)
                    if (u[ll].id == T) u[ll].flag = true;
            }
        }
        todo.swap(new_todo);
    }
    g.M.swap(new_L);
    prune1(g);
}

Graph graph_from_csr(unsigned n, const uint64_t *offsets, const uint32_t *ids, const float *dists,
                     const uint32_t *M) {
    Graph g;
    g.adj.resize(n);
    g.M.assign(M, M + n);
    for (unsigned i = 0; i < n; ++i)
        for (uint64_t e = offsets[i]; e < offsets[i + 1]; ++e)
            g.adj[i].push_back(Neighbor{ids[e], dists ? dists[e] : 0.0f, false});
    return g;
}

// ---------------------------------------------------------------- build
struct Nhood {
    float radius, radiusM;
    std::vector<Neighbor> pool;
    unsigned L, M;
    bool found;
    std::vector<unsigned> nn_old, nn_new, rnn_old, rnn_new;

    // Nhood::parallel_try_insert, kgraph.cpp:723-736
    unsigned try_insert(unsigned id, float dist) {
        if (dist > radius) return pool.size();
        unsigned l = update_knn_list(&pool[0], L, Neighbor{id, dist, true});
        if (l <= L) {
            if (L + 1 < pool.size()) ++L;
            else radius = pool[L - 1].dist;
        }
        return l;
    }
};

struct Control { unsigned id; std::vector<Neighbor> neighbors; };

// kgraph.cpp:96-156
bool evaluate_recall(const std::vector<Neighbor> &pool, const std::vector<Neighbor> &knn, float *out) {
    if (knn.empty()) { *out = 1.0f; return true; }
    unsigned found = 0, n_p = 0, n_k = 0;
    for (;;) {
        if (n_p >= pool.size()) break;
        if (n_k >= knn.size()) break;
        if (knn[n_k].dist < pool[n_p].dist) ++n_k;
        else if (knn[n_k].dist == pool[n_p].dist) { ++found; ++n_k; ++n_p; }
        else return false;
    }
    *out = float(found) / knn.size();
    return true;
}
float evaluate_accuracy(const std::vector<Neighbor> &pool, const std::vector<Neighbor> &knn) {
    unsigned m = std::min(pool.size(), knn.size());
    float sum = 0;
    unsigned cnt = 0;
    for (unsigned i = 0; i < m; ++i)
        if (knn[i].dist > 0) { sum += std::abs(pool[i].dist - knn[i].dist) / knn[i].dist; ++cnt; }
    return cnt > 0 ? sum / cnt : 0;
}
float evaluate_delta(const std::vector<Neighbor> &pool, unsigned K) {
    unsigned c = 0, N = K;
    if (pool.size() < N) N = pool.size();
    for (unsigned i = 0; i < N; ++i) if (pool[i].flag) ++c;
    return float(c) / K;
}

// LinearSearch, kgraph.cpp:212-229
void linear_search(const Data &D, unsigned i, unsigned K, std::vector<Neighbor> *out) {
    std::vector<Neighbor> nns(K + 1, unset_neighbor());
    Neighbor nn{0, 0.0f, true};
    unsigned k = 0;
    while (nn.id < D.n) {
        if (nn.id != i) {
            nn.dist = D(i, nn.id);
            update_knn_list(&nns[0], k, nn);
            if (k < K) ++k;
        }
        ++nn.id;
    }
    nns.resize(K);
    out->swap(nns);
}

// Float mean as the boost accumulator the reference uses: float running sum / count.
struct Mean { float s = 0; size_t c = 0; void operator()(float x) { s += x; ++c; } float get() const { return s / c; } };

}  // namespace

extern "C" {

const char *kgo_last_error(void) { return g_err.c_str(); }

float kgo_dot(const float *a, const float *b, unsigned d) { return dot_impl(a, b, d); }
float kgo_norm2(const float *a, unsigned d) { return norm2_impl(a, d); }
float kgo_l2sqr(const float *a, const float *b, unsigned d) { return l2sqr_impl(a, b, d); }

void kgo_norms(const float *X, unsigned n, unsigned d, int metric, float *norms) {
    for (unsigned i = 0; i < n; ++i) norms[i] = metric_norm(X + (size_t)i * d, d, metric);
}
float kgo_query_norm(const float *q, unsigned d, int metric) { return metric_norm(q, d, metric); }

float kgo_pair(const float *X, const float *norms, unsigned d, int metric, unsigned i, unsigned j) {
    Data D{X, norms, 0, d, metric};
    return D(i, j);
}
float kgo_query_dist(const float *X, const float *norms, unsigned d, int metric,
                     const float *q, float qnorm, unsigned i) {
    Data D{X, norms, 0, d, metric};
    return Query{D, q, qnorm}(i);
}

unsigned kgo_bruteforce(const float *X, const float *norms, unsigned n, unsigned d, int metric,
                        const float *q, unsigned K, float epsilon, uint32_t *ids, float *dists) {
    Data D{X, norms, n, d, metric};
    Query Q{D, q, metric_norm(q, d, metric)};
    std::vector<Neighbor> nns(K + 1, unset_neighbor());
    unsigned L = 0;
    for (unsigned k = 0; k < n; ++k) {
        float kd = Q(k);
        if (kd > epsilon) continue;
        update_knn_list(&nns[0], L, Neighbor{k, kd, true});
        if (L < K) ++L;
    }
    for (unsigned k = 0; k < L; ++k) { if (ids) ids[k] = nns[k].id; if (dists) dists[k] = nns[k].dist; }
    return L;
}

void kgo_linear_search(const float *X, const float *norms, unsigned n, unsigned d, int metric,
                       unsigned i, unsigned K, uint32_t *ids, float *dists) {
    Data D{X, norms, n, d, metric};
    std::vector<Neighbor> out;
    linear_search(D, i, K, &out);
    for (unsigned k = 0; k < K; ++k) { ids[k] = out[k].id; dists[k] = out[k].dist; }
}

void kgo_genrandom(unsigned seed, unsigned size, unsigned N, unsigned calls, uint32_t *out) {
    std::mt19937 rng(seed);
    std::vector<unsigned> tmp(size + 1);
    for (unsigned c = 0; c < calls; ++c) gen_random(rng, tmp.data(), size, N);
    gen_random(rng, tmp.data(), size, N);
    std::copy(tmp.begin(), tmp.begin() + size, out);
}

void kgo_std_sort_pairs(float *dists, uint32_t *ids, unsigned n) {
    std::vector<Neighbor> v(n);
    for (unsigned i = 0; i < n; ++i) v[i] = Neighbor{ids[i], dists[i], false};
    std::sort(v.begin(), v.end(), less_dist);
    for (unsigned i = 0; i < n; ++i) { ids[i] = v[i].id; dists[i] = v[i].dist; }
}

unsigned kgo_search(const float *X, const float *norms, unsigned n, unsigned d, int metric,
                    const uint64_t *offsets, const uint32_t *nbr, const uint32_t *Mn,
                    const float *q, unsigned K, unsigned P, unsigned Mp, unsigned S, unsigned T,
                    float epsilon, unsigned seed_in, unsigned init,
                    uint32_t *ids, float *dists, float *cost) {
    Data D{X, norms, n, d, metric};
    Query oracle{D, q, metric_norm(q, d, metric)};
    const unsigned N = n;
    auto actual_M = [&](unsigned pM, unsigned i) -> unsigned {
        unsigned deg = (unsigned)(offsets[i + 1] - offsets[i]);
        return std::min(std::max(Mn[i], pM), deg);
    };
    if (P >= N) {   // kgraph.cpp:427-433
        if (cost) *cost = 1.0f;
        return kgo_bruteforce(X, norms, n, d, metric, q, K, epsilon, ids, dists);
    }
    std::vector<NeighborX> knn(K + P + 1, NeighborX{0xFFFFFFFFu, FLT_MAX, false, 0, 0});
    std::vector<NeighborX> results;
    std::vector<bool> flags(N, false);
    if (init && T > 1) { g_err = "when init > 0, T must be 1."; return 0xFFFFFFFFu; }
    unsigned seed = seed_in;
    if (seed == 0) seed = time(NULL);
    std::mt19937 rng(seed);
    unsigned n_comps = 0;
    for (unsigned trial = 0; trial < T; ++trial) {
        unsigned L = init;
        if (L == 0) {
            std::vector<unsigned> random(P + 1);
            gen_random(rng, &random[0], P, N);
            for (unsigned i = 0; i < P; ++i) {
                unsigned s = random[i];
                if (!flags[s]) knn[L++].id = s;
            }
        } else {
            if (!ids) { g_err = "no initial data provided via ids"; return 0xFFFFFFFFu; }
            if (!(L < K)) { g_err = "L < params.K"; return 0xFFFFFFFFu; }
            for (unsigned l = 0; l < L; ++l) knn[l].id = ids[l];
        }
        for (unsigned k = 0; k < L; ++k) {
            auto &e = knn[k];
            flags[e.id] = true;
            e.flag = true;
            e.dist = oracle(e.id);
            e.m = 0;
            e.M = actual_M(Mp, e.id);
        }
        std::sort(knn.begin(), knn.begin() + L,
                  [](const NeighborX &a, const NeighborX &b) { return a.dist < b.dist; });
        unsigned k = 0;
        while (k < L) {
            auto &e = knn[k];
            if (!e.flag) { ++k; continue; }
            unsigned beginM = e.m;
            unsigned endM = beginM + S;
            if (endM > e.M) { e.flag = false; endM = e.M; }
            e.m = endM;
            unsigned node = e.id;
            for (unsigned m = beginM; m < endM; ++m) {
                unsigned id = nbr[offsets[node] + m];
                if (flags[id]) continue;
                flags[id] = true;
                ++n_comps;
                float dist = oracle(id);
                NeighborX nn{id, dist, true, 0, 0};
                unsigned r = update_knn_list(&knn[0], L, nn);
                if (L + 1 < knn.size()) ++L;
                if (r < L) {
                    knn[r].M = actual_M(Mp, id);
                    if (r < k) k = r;
                }
            }
        }
        if (L > K) L = K;
        if (results.empty()) {
            results.reserve(K + 1);
            results.resize(L + 1, NeighborX{0xFFFFFFFFu, FLT_MAX, false, 0, 0});
            std::copy(knn.begin(), knn.begin() + L, results.begin());
        } else {
            for (unsigned l = 0; l < L; ++l) {
                unsigned r = update_knn_list(&results[0], results.size() - 1, knn[l]);
                if (r < results.size() && results.size() < (K + 1))
                    results.resize(results.size() + 1, NeighborX{0xFFFFFFFFu, FLT_MAX, false, 0, 0});
            }
        }
    }
    results.pop_back();
    for (unsigned l = 0; l < results.size(); ++l)
        if (results[l].dist > epsilon) { results.resize(l); break; }
    unsigned L = results.size();
    for (unsigned k = 0; k < L; ++k) { if (ids) ids[k] = results[k].id; if (dists) dists[k] = results[k].dist; }
    if (cost) *cost = float(n_comps) / N;
    return L;
}

int kgo_build(const float *X, const float *norms, unsigned n, unsigned d, int metric,
              unsigned iterations, unsigned Lp, unsigned Kp, unsigned Sp, unsigned R,
              unsigned controls_n, unsigned seed, float delta_stop, float recall_stop,
              unsigned prune, int reverse, unsigned rand_seed,
              uint64_t *E, float *info_out, float *log, unsigned log_cap) {
    try {
        Data D{X, norms, n, d, metric};
        const unsigned N = n;
        unsigned L = Lp, K = Kp, S = Sp, C = controls_n;
        // kgraph.cpp:893-905
        if (N <= K) throw std::runtime_error("K larger than dataset size");
        if (N < C) C = N;
        if (N <= L) L = N - 1;
        if (N <= S) S = N - 1;
        std::srand(rand_seed);
        // GenerateControl, kgraph.cpp:254-270
        std::vector<Control> controls(C);
        {
            std::vector<unsigned> index(N);
            for (unsigned i = 0; i < N; ++i) index[i] = i;
            std::random_shuffle(index.begin(), index.end());
            for (unsigned i = 0; i < C; ++i) { controls[i].id = index[i]; linear_search(D, index[i], K, &controls[i].neighbors); }
        }
        // init, kgraph.cpp:760-796 (one OpenMP thread: rng = mt19937(seed ^ 0))
        std::vector<Nhood> nhoods(N);
        for (auto &nh : nhoods) {
            nh.nn_new.resize(S * 2);
            nh.pool.assign(L + 1, unset_neighbor());
            nh.radius = std::numeric_limits<float>::max();
        }
        {
            std::mt19937 rng(seed ^ 0);
            std::vector<unsigned> random(S + 1);
            for (unsigned nn = 0; nn < N; ++nn) {
                auto &nh = nhoods[nn];
                gen_random(rng, &nh.nn_new[0], nh.nn_new.size(), N);
                gen_random(rng, &random[0], random.size(), N);
                nh.L = S;
                nh.M = S;
                unsigned i = 0;
                for (unsigned l = 0; l < nh.L; ++l) {
                    if (random[i] == nn) ++i;
                    auto &e = nh.pool[l];
                    e.id = random[i++];
                    e.dist = D(e.id, nn);
                    e.flag = true;
                }
                std::sort(nh.pool.begin(), nh.pool.begin() + nh.L, less_dist);
            }
        }
        float total = N * float(N - 1) / 2;
        size_t n_comps = 0;
        int stop = 0;
        unsigned info_it = 0;
        float info_cost = 0, info_recall = 0, info_acc = std::numeric_limits<float>::max(), info_delta = 1.0f, info_M = 0;
        for (unsigned it = 0; (iterations <= 0) || (it < iterations); ++it) {
            ++info_it;
            // join, kgraph.cpp:797-815 (one thread: nodes in order)
            size_t cc = 0;
            for (unsigned nn = 0; nn < N; ++nn) {
                size_t uu = 0;
                nhoods[nn].found = false;
                auto cb = [&](unsigned i, unsigned j) {
                    float dist = D(i, j);
                    ++cc;
                    unsigned r = nhoods[i].try_insert(j, dist);
                    if (r < K) ++uu;
                    nhoods[j].try_insert(i, dist);
                    if (r < K) ++uu;
                };
                const auto &nh = nhoods[nn];
                std::vector<unsigned> nw = nh.nn_new, od = nh.nn_old;   // join reads a stable copy
                for (unsigned i : nw) {
                    for (unsigned j : nw) if (i < j) cb(i, j);
                    for (unsigned j : od) cb(i, j);
                }
                nhoods[nn].found = uu > 0;
            }
            n_comps += cc;
            // statistics, kgraph.cpp:927-963
            info_cost = n_comps / total;
            Mean one_exact, one_approx, one_recall, recall, accuracy, Mm, delta;
            for (auto const &nh : nhoods) { Mm(nh.M); delta(evaluate_delta(nh.pool, K)); }
            for (auto const &c : controls) {
                one_approx(nhoods[c.id].pool[0].dist);
                one_exact(c.neighbors[0].dist);
                one_recall(nhoods[c.id].pool[0].dist == c.neighbors[0].dist ? 1.0f : 0.0f);
                float rr;
                if (!evaluate_recall(nhoods[c.id].pool, c.neighbors, &rr)) throw std::runtime_error("distance is unstable");
                recall(rr);
                accuracy(evaluate_accuracy(nhoods[c.id].pool, c.neighbors));
            }
            info_delta = delta.get();
            info_recall = recall.get();
            info_acc = accuracy.get();
            info_M = Mm.get();
            if (log && info_it <= log_cap) {
                float *row = log + (size_t)(info_it - 1) * 9;
                row[0] = info_it; row[1] = info_recall; row[2] = info_acc; row[3] = info_cost;
                row[4] = info_M; row[5] = info_delta; row[6] = one_recall.get();
                row[7] = one_approx.get() / one_exact.get(); row[8] = 0;
            }
            if (info_delta <= delta_stop) { stop = 1; break; }
            if (info_recall >= recall_stop) { stop = 2; break; }
            // update, kgraph.cpp:816-883
            for (auto &nh : nhoods) {
                nh.nn_new.clear(); nh.nn_old.clear(); nh.rnn_new.clear(); nh.rnn_old.clear();
                nh.radius = nh.pool.back().dist;
            }
            for (unsigned nn = 0; nn < N; ++nn) {
                auto &nh = nhoods[nn];
                if (nh.found) {
                    unsigned maxl = std::min(nh.M + S, nh.L);
                    unsigned c = 0, l = 0;
                    while ((l < maxl) && (c < S)) { if (nh.pool[l].flag) ++c; ++l; }
                    nh.M = l;
                }
                nh.radiusM = nh.pool[nh.M - 1].dist;
            }
            for (unsigned nn = 0; nn < N; ++nn) {
                auto &nh = nhoods[nn];
                for (unsigned l = 0; l < nh.M; ++l) {
                    auto &e = nh.pool[l];
                    auto &other = nhoods[e.id];
                    if (e.flag) {
                        nh.nn_new.push_back(e.id);
                        if (e.dist > other.radiusM) other.rnn_new.push_back(nn);
                        e.flag = false;
                    } else {
                        nh.nn_old.push_back(e.id);
                        if (e.dist > other.radiusM) other.rnn_old.push_back(nn);
                    }
                }
            }
            for (unsigned i = 0; i < N; ++i) {
                auto &nh = nhoods[i];
                if (R && nh.rnn_new.size() > R) { std::random_shuffle(nh.rnn_new.begin(), nh.rnn_new.end()); nh.rnn_new.resize(R); }
                nh.nn_new.insert(nh.nn_new.end(), nh.rnn_new.begin(), nh.rnn_new.end());
                if (R && nh.rnn_old.size() > R) { std::random_shuffle(nh.rnn_old.begin(), nh.rnn_old.end()); nh.rnn_old.resize(R); }
                nh.nn_old.insert(nh.nn_old.end(), nh.rnn_old.begin(), nh.rnn_old.end());
            }
        }
        // finalize, kgraph.cpp:975-988 (only entries an insert has written)
        if (prune > 2) throw std::runtime_error("prune level not supported.");
        Graph g;
        g.adj.resize(N);
        g.M.resize(N);
        for (unsigned nn = 0; nn < N; ++nn) {
            g.M[nn] = nhoods[nn].M;
            unsigned cnt = std::min(L, nhoods[nn].L);
            g.adj[nn].assign(nhoods[nn].pool.begin(), nhoods[nn].pool.begin() + cnt);
            for (auto &e : g.adj[nn]) e.flag = false;
        }
        nhoods.clear();
        if (reverse) reverse_graph(g, reverse);
        if (prune & 1) prune1(g);
        if (prune & 2) prune2(g);
        *E = store_result(std::move(g));
        if (info_out) {
            info_out[0] = stop; info_out[1] = info_it; info_out[2] = info_cost; info_out[3] = info_recall;
            info_out[4] = info_acc; info_out[5] = info_delta; info_out[6] = info_M;
        }
        return 0;
    } catch (std::exception const &e) {
        g_err = e.what();
        return 1;
    }
}

void kgo_build_result(uint64_t *offsets, uint32_t *ids, float *dists, uint32_t *M) {
    uint64_t e = 0;
    for (unsigned i = 0; i < g_result.adj.size(); ++i) {
        offsets[i] = e;
        for (auto &x : g_result.adj[i]) { ids[e] = x.id; if (dists) dists[e] = x.dist; ++e; }
        M[i] = g_result.M[i];
    }
    offsets[g_result.adj.size()] = e;
}

uint64_t kgo_reverse(unsigned n, const uint64_t *offsets, const uint32_t *ids, const float *dists,
                     const uint32_t *M, int rev_k) {
    Graph g = graph_from_csr(n, offsets, ids, dists, M);
    reverse_graph(g, rev_k);
    return store_result(std::move(g));
}

uint64_t kgo_prune(unsigned n, const uint64_t *offsets, const uint32_t *ids, const float *dists,
                   const uint32_t *M, unsigned level) {
    Graph g = graph_from_csr(n, offsets, ids, dists, M);
    if (level & 1) prune1(g);
    if (level & 2) prune2(g);
    return store_result(std::move(g));
}

void kgo_serial_inserts(unsigned Lp, float *pool_d, uint32_t *pool_i, unsigned *L, float *radius, unsigned n_off,
                        const uint32_t *cand, const float *dist, uint32_t *r_out) {
    Nhood nh;
    nh.pool.resize(Lp);
    for (unsigned j = 0; j < Lp; ++j)
        nh.pool[j] = Neighbor{pool_i[j] & 0x7FFFFFFFu, pool_d[j], (pool_i[j] & 0x80000000u) != 0};
    nh.L = *L;
    nh.radius = *radius;
    for (unsigned k = 0; k < n_off; ++k) r_out[k] = nh.try_insert(cand[k], dist[k]);
    for (unsigned j = 0; j < Lp; ++j) {
        pool_d[j] = nh.pool[j].dist;
        pool_i[j] = nh.pool[j].id | (nh.pool[j].flag ? 0x80000000u : 0u);
    }
    *L = nh.L;
    *radius = nh.radius;
}

}  // extern "C"
