// Dense datasets and the built-in oracles, B200 build.
//
// Same classes as the reference's kgraph-data.h (Matrix, MatrixProxy,
// metric::l2sqr / l2, MatrixOracle, AverageRecall; kgraph-data.h:31-367),
// plus DenseMatrixOracle, the euclidean / angular oracle of the Python module
// (python-api.cpp:51-129) for C++ users.  Every oracle here carries the
// DenseIndexOracle / DenseSearchOracle mix-in, which is how KGraph::build
// and KGraph::search hand the matrix to the GPU.
//
// The CPU operator() of each oracle returns the same bits as the GPU kernels:
// 16-lane accumulation (rounded product, rounded add), the reference's
// 16->4->1 reduction tree, then the D % 16 tail in order (with 8 or more tail
// elements the first 8 as rounded product + add, the others fused).
#ifndef WDONG_KGRAPH_DATA
#define WDONG_KGRAPH_DATA

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>
#include "kgraph.h"

namespace kgraph {

static constexpr size_t KGRAPH_MATRIX_ALIGN = 64;

namespace detail {
    inline float reduce16(float const *x) {
        float t[4];
        for (int k = 0; k < 4; ++k) t[k] = (x[k] + x[k + 4]) + (x[k + 8] + x[k + 12]);
        return (t[0] + t[1]) + (t[2] + t[3]);
    }
    // mode 0: dot, 1: squared difference
    inline float canonical_sum(float const *a, float const *b, unsigned d, int mode) {
        float acc[16] = {0};
        unsigned vs = d - d % 16, i = 0;
        for (; i < vs; i += 16)
            for (int l = 0; l < 16; ++l) {
                volatile float p;
                if (mode) { float t = a[i + l] - b[i + l]; p = t * t; }
                else p = a[i + l] * b[i + l];
                acc[l] = acc[l] + p;
            }
        float r = reduce16(acc);
        if (d - i >= 8)
            for (unsigned e = i + 8; i < e; ++i) {
                volatile float p;
                if (mode) { float t = a[i] - b[i]; p = t * t; }
                else p = a[i] * b[i];
                r = r + p;
            }
        for (; i < d; ++i) {
            if (mode) { float t = a[i] - b[i]; r = std::fma(t, t, r); }
            else r = std::fma(a[i], b[i], r);
        }
        return r;
    }
}

namespace metric {
    /// Squared L2 distance (reference kgraph-data.h:38-104).
    struct l2sqr {
        static constexpr int code = 2;
        template <typename T>
        static T apply(T const *t1, T const *t2, unsigned size) { return detail::canonical_sum(t1, t2, size, 1); }
        template <typename T>
        static T dot(T const *t1, T const *t2, unsigned size) { return detail::canonical_sum(t1, t2, size, 0); }
        template <typename T>
        static float norm2(T const *t1, unsigned size) { return detail::canonical_sum(t1, t1, size, 0); }
    };
    /// L2 distance (reference kgraph-data.h:106-111).  Not a GPU metric.
    struct l2 {
        static constexpr int code = -1;
        template <typename T>
        static T apply(T const *t1, T const *t2, unsigned dim) { return std::sqrt(l2sqr::apply<T>(t1, t2, dim)); }
    };
}

/// Row-major matrix with rows padded to A bytes (reference kgraph-data.h:114-219).
template <typename T, unsigned A = KGRAPH_MATRIX_ALIGN>
class Matrix {
    unsigned col;
    unsigned row;
    size_t stride;
    char *data;
protected:
    void reset(unsigned r, unsigned c) {
        row = r;
        col = c;
        stride = (sizeof(T) * c + A - 1) / A * A;
        if (data) free(data);
        data = (char *)aligned_alloc(A, (row * stride + A - 1) / A * A + A);
        if (!data) throw runtime_error("memalign");
    }
public:
    Matrix() : col(0), row(0), stride(0), data(0) {}
    Matrix(unsigned r, unsigned c) : data(0) { reset(r, c); }
    Matrix(Matrix const &) = delete;
    Matrix &operator=(Matrix const &) = delete;
    ~Matrix() { if (data) free(data); }
    unsigned size() const { return row; }
    unsigned dim() const { return col; }
    size_t step() const { return stride; }
    void resize(unsigned r, unsigned c) { reset(r, c); }
    T const *operator[](unsigned i) const { return reinterpret_cast<T const *>(&data[stride * i]); }
    T *operator[](unsigned i) { return reinterpret_cast<T *>(&data[stride * i]); }
    void zero() { memset(data, 0, row * stride); }
    void normalize2() {
        for (unsigned i = 0; i < row; ++i) {
            T *p = operator[](i);
            double sum = metric::l2sqr::norm2(p, col);
            sum = std::sqrt(sum);
            for (unsigned j = 0; j < col; ++j) p[j] /= sum;
        }
    }
    void load(const std::string &path, unsigned dim, unsigned skip = 0, unsigned gap = 0) {
        std::ifstream is(path.c_str(), std::ios::binary);
        if (!is) throw io_error(path);
        is.seekg(0, std::ios::end);
        size_t size = is.tellg();
        size -= skip;
        unsigned line = sizeof(T) * dim + gap;
        unsigned N = size / line;
        reset(N, dim);
        zero();
        is.seekg(skip, std::ios::beg);
        for (unsigned i = 0; i < N; ++i) {
            is.read(&data[stride * i], sizeof(T) * dim);
            is.seekg(gap, std::ios::cur);
        }
        if (!is) throw io_error(path);
    }
    void load_lshkit(std::string const &path) {
        std::ifstream is(path.c_str(), std::ios::binary);
        unsigned header[3];   // element size, rows, cols
        is.read((char *)header, sizeof header);
        if (!is) throw io_error(path);
        if (header[0] != sizeof(T)) throw io_error(path);
        is.close();
        load(path, header[2], 3 * sizeof(unsigned), 0);
    }
    void save_lshkit(std::string const &path) {
        std::ofstream os(path.c_str(), std::ios::binary);
        unsigned header[3] = {(unsigned)sizeof(T), row, col};
        os.write((const char *)header, sizeof(header));
        for (unsigned i = 0; i < row; ++i) os.write(&data[stride * i], sizeof(T) * col);
    }
};

/// Non-owning view of a row-major matrix (reference kgraph-data.h:221-296).
template <typename DATA_TYPE, unsigned A = KGRAPH_MATRIX_ALIGN>
class MatrixProxy {
    unsigned rows;
    unsigned cols;
    size_t stride;
    uint8_t const *data;
public:
    MatrixProxy(Matrix<DATA_TYPE> const &m)
        : rows(m.size()), cols(m.dim()), stride(m.step()), data(reinterpret_cast<uint8_t const *>(m[0])) {}
    MatrixProxy(DATA_TYPE const *p, unsigned r, unsigned c, size_t s)
        : rows(r), cols(c), stride(s), data(reinterpret_cast<uint8_t const *>(p)) {
        if (!(stride >= cols * sizeof(DATA_TYPE))) throw invalid_argument("bad stride");
    }
    unsigned size() const { return rows; }
    unsigned dim() const { return cols; }
    size_t step() const { return stride; }
    DATA_TYPE const *operator[](unsigned i) const { return reinterpret_cast<DATA_TYPE const *>(data + stride * i); }
};

/// Oracle over a Matrix / MatrixProxy with a metric of namespace metric
/// (reference kgraph-data.h:298-331).  Dense: usable by the GPU build.
template <typename DATA_TYPE, typename DIST_TYPE>
class MatrixOracle : public IndexOracle, public DenseIndexOracle {
    MatrixProxy<DATA_TYPE> proxy;
public:
    class SearchOracle : public kgraph::SearchOracle, public DenseSearchOracle {
        MatrixProxy<DATA_TYPE> proxy;
        DATA_TYPE const *q;
    public:
        SearchOracle(MatrixProxy<DATA_TYPE> const &p, DATA_TYPE const *query) : proxy(p), q(query) {}
        virtual unsigned size() const { return proxy.size(); }
        virtual float operator()(unsigned i) const { return DIST_TYPE::apply(proxy[i], q, proxy.dim()); }
        virtual DenseView dense() const {
            return DenseView{reinterpret_cast<float const *>(proxy[0]), proxy.size(), proxy.dim(), proxy.step(),
                             DIST_TYPE::code};
        }
        virtual float const *query() const { return reinterpret_cast<float const *>(q); }
    };
    template <typename MATRIX_TYPE>
    MatrixOracle(MATRIX_TYPE const &m) : proxy(m) {}
    virtual unsigned size() const { return proxy.size(); }
    virtual float operator()(unsigned i, unsigned j) const { return DIST_TYPE::apply(proxy[i], proxy[j], proxy.dim()); }
    SearchOracle query(DATA_TYPE const *q) const { return SearchOracle(proxy, q); }
    virtual DenseView dense() const {
        return DenseView{reinterpret_cast<float const *>(proxy[0]), proxy.size(), proxy.dim(), proxy.step(),
                         DIST_TYPE::code};
    }
};

/// Euclidean (half squared L2 by expansion) or angular (-cos) oracle over a
/// dense float matrix: the oracles of the reference's Python module
/// (python-api.cpp:51-129), usable from C++.  metric: 0 euclidean, 1 angular.
class DenseMatrixOracle : public IndexOracle, public DenseIndexOracle {
    float const *rows;
    unsigned n, d;
    size_t stride;
    int metric;
    std::vector<float> n2;
    float const *row(unsigned i) const { return reinterpret_cast<float const *>(reinterpret_cast<char const *>(rows) + stride * i); }
    static float norm_of(float const *x, unsigned d, int metric) {
        float s = detail::canonical_sum(x, x, d, 0);
        return metric == 0 ? s / 2 : std::sqrt(s);
    }
    static float combine(float dot, float a, float b, int metric) {
        if (metric == 0) return (a + b) - dot;
        return -dot / std::fma(a, b, std::numeric_limits<float>::epsilon());
    }
public:
    class SearchOracle : public kgraph::SearchOracle, public DenseSearchOracle {
        DenseMatrixOracle const &o;
        float const *q;
        float qn;
    public:
        SearchOracle(DenseMatrixOracle const &oracle, float const *query)
            : o(oracle), q(query), qn(norm_of(query, oracle.d, oracle.metric)) {}
        virtual unsigned size() const { return o.n; }
        virtual float operator()(unsigned i) const {
            return combine(detail::canonical_sum(o.row(i), q, o.d, 0), o.n2[i], qn, o.metric);
        }
        virtual DenseView dense() const { return o.dense(); }
        virtual float const *query() const { return q; }
    };
    DenseMatrixOracle(float const *data, unsigned rows_, unsigned dim, size_t stride_bytes, int metric_)
        : rows(data), n(rows_), d(dim), stride(stride_bytes), metric(metric_) {
        if (metric != 0 && metric != 1) throw runtime_error("metric not supported");
        if (stride < d * sizeof(float)) throw invalid_argument("bad stride");
        n2.resize(n);
        for (unsigned i = 0; i < n; ++i) n2[i] = norm_of(row(i), d, metric);
    }
    virtual unsigned size() const { return n; }
    virtual float operator()(unsigned i, unsigned j) const {
        return combine(detail::canonical_sum(row(i), row(j), d, 0), n2[i], n2[j], metric);
    }
    SearchOracle query(float const *q) const { return SearchOracle(*this, q); }
    virtual DenseView dense() const { return DenseView{rows, n, d, stride, metric}; }
};

/// Mean recall of `result` against gold standard `gs`, matching by distance
/// value (reference kgraph-data.h:333-364).
inline float AverageRecall(Matrix<float> const &gs, Matrix<float> const &result, unsigned K = 0) {
    if (K == 0) K = result.dim();
    if (!(gs.dim() >= K)) throw invalid_argument("gs.dim() >= K");
    if (!(result.dim() >= K)) throw invalid_argument("result.dim() >= K");
    if (!(gs.size() >= result.size())) throw invalid_argument("gs.size() > result.size()");
    float sum = 0;
    for (unsigned i = 0; i < result.size(); ++i) {
        float const *gs_row = gs[i];
        float const *re_row = result[i];
        unsigned found = 0, gs_n = 0, re_n = 0;
        while ((gs_n < K) && (re_n < K)) {
            if (gs_row[gs_n] < re_row[re_n]) ++gs_n;
            else if (gs_row[gs_n] == re_row[re_n]) { ++found; ++gs_n; ++re_n; }
            else throw runtime_error("distance is unstable");
        }
        sum += float(found) / K;
    }
    return sum / result.size();
}

}  // namespace kgraph

#endif
