// GPU tests of the linalg_backend::B200 operator specializations, written
// against the reference's own template API (include/linalg_b200/
// reference_api.h) the way its GPU test suite exercises CUDA_BLAS: device
// buffers, caller-owned workspace, non-default streams, argument validation.
// Built by __graft_entry__.build() / tests/cpp/build.sh; run by
// tests/test_cpp_api_gpu.py on a B200.  Prints one PASS/FAIL line per case.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <stdexcept>
#include <utility>
#include <vector>

#include "linalg_b200/backend_b200.h"

using linalg::linalg_backend;
constexpr auto B = linalg_backend::B200;

static int g_fail = 0;
#define CHECK(cond, name)                                                                          \
    do                                                                                             \
    {                                                                                              \
        if (cond)                                                                                  \
            std::printf("PASS %s\n", name);                                                        \
        else                                                                                       \
        {                                                                                          \
            std::printf("FAIL %s (%s:%d)\n", name, __FILE__, __LINE__);                            \
            ++g_fail;                                                                              \
        }                                                                                          \
    } while (0)

template <typename T> struct dbuf
{
    T*     p = nullptr;
    size_t n = 0;
    explicit dbuf(size_t count) : n(count)
    {
        if (cudaMalloc(&p, sizeof(T) * (count ? count : 1)) != cudaSuccess)
            throw std::runtime_error("cudaMalloc");
    }
    ~dbuf() { cudaFree(p); }
    void up(const std::vector<T>& h) { cudaMemcpy(p, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice); }
    std::vector<T> down() const
    {
        std::vector<T> h(n);
        cudaMemcpy(h.data(), p, sizeof(T) * n, cudaMemcpyDeviceToHost);
        return h;
    }
};

static std::vector<double> random_matrix(int rows, int cols, unsigned seed, double lo = -5, double hi = 5)
{
    std::mt19937_64                        g(seed);
    std::uniform_real_distribution<double> u(lo, hi);
    std::vector<double>                    a((size_t)rows * cols);
    for (auto& v : a) v = u(g);
    return a;
}

static void test_lu()
{
    const int           n = 17;
    std::vector<double> a = random_matrix(n, n, 1);
    dbuf<double>        m(n * n);
    dbuf<linalg_int>    piv(n);
    m.up(a);
    const size_t ws_bytes = linalg::lu_decomposition<double, B>::workspace_size(n);
    dbuf<unsigned char> ws(ws_bytes);
    int                 info = -1;
    const bool ok = linalg::lu_decomposition<double, B>::apply(m.p, n, piv.p, ws.p, ws_bytes, &info);
    auto lu = m.down();
    auto p  = piv.down();
    bool pivots_ok = true;
    for (int i = 0; i < n; ++i) pivots_ok = pivots_ok && p[i] >= i + 1 && p[i] <= n;
    // P A = L U
    std::vector<double> pa = a;
    for (int i = 0; i < n; ++i)
        if (p[i] - 1 != i)
            for (int j = 0; j < n; ++j) std::swap(pa[i * n + j], pa[(p[i] - 1) * n + j]);
    double err = 0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
            double s = 0;
            for (int k = 0; k <= std::min(i, j); ++k)
                s += (k == i ? 1.0 : lu[i * n + k]) * (k <= j ? lu[k * n + j] : 0.0);
            err = std::max(err, std::fabs(s - pa[i * n + j]));
        }
    CHECK(ok && info == 0, "lu_decomposition returns true, info 0");
    CHECK(pivots_ok, "lu_decomposition pivots in [i+1, n]");
    CHECK(err <= 1e-9 * n, "lu_decomposition P*A == L*U");
}

static void test_linear_solver()
{
    const int           n = 1024;
    std::vector<double> r = random_matrix(n, n, 2, -1, 1);
    std::vector<double> a((size_t)n * n, 0.0), x_true(n), b(n, 0.0);
    // symmetric positive definite: R R^T + 2n I
    for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j)
        {
            double s = 0;
            for (int k = 0; k < n; ++k) s += r[i * n + k] * r[j * n + k];
            a[i * n + j] = a[j * n + i] = s + (i == j ? 2.0 * n : 0.0);
        }
    std::mt19937_64 g(3);
    std::uniform_real_distribution<double> u(-1, 1);
    for (auto& v : x_true) v = u(g);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) b[i] += a[i * n + j] * x_true[j];
    for (auto mode : {linalg::linear_solver_type::LU_LINEAR_SOLVER,
             linalg::linear_solver_type::CHOLESKY_LINEAR_SOLVER})
    {
        const bool chol = mode == linalg::linear_solver_type::CHOLESKY_LINEAR_SOLVER;
        dbuf<double>     m(n * n), x(n);
        dbuf<linalg_int> piv(n);
        m.up(a);
        x.up(b);
        cudaStream_t s;
        cudaStreamCreate(&s);
        const size_t        bytes = linalg::linear_solver<double, B>::workspace_size(n, mode);
        dbuf<unsigned char> ws(bytes);
        linalg::linear_solver<double, B>::apply(m.p, piv.p, n, x.p, mode, ws.p, bytes, s);
        cudaStreamSynchronize(s);
        auto xs = x.down();
        double e = 0;
        for (int i = 0; i < n; ++i) e = std::max(e, std::fabs(xs[i] - x_true[i]));
        CHECK(e <= 1e-9 * n, chol ? "linear_solver CHOLESKY on a stream" : "linear_solver LU on a stream");
        // the UPFRONT modes reuse the factors (and, for LU, the pivots)
        x.up(b);
        linalg::linear_solver<double, B>::apply(m.p, chol ? nullptr : piv.p, n, x.p,
            chol ? linalg::linear_solver_type::CHOLESKY_UPFRONT_LINEAR_SOLVER
                 : linalg::linear_solver_type::LU_UPFRONT_LINEAR_SOLVER,
            ws.p, bytes, s);
        cudaStreamSynchronize(s);
        xs = x.down();
        e  = 0;
        for (int i = 0; i < n; ++i) e = std::max(e, std::fabs(xs[i] - x_true[i]));
        CHECK(e <= 1e-9 * n, chol ? "linear_solver CHOLESKY_UPFRONT reuses the factor"
                                  : "linear_solver LU_UPFRONT reuses pivots");
        cudaStreamDestroy(s);
    }
}

static void test_triangular()
{
    const int n = 35, nrhs = 9, lda = n + 2, ldb = nrhs + 1, ldx = nrhs + 3;
    bool      all_ok = true;
    for (bool upper : {false, true})
        for (bool transpose : {false, true})
            for (bool unit : {false, true})
            {
                std::vector<double> a((size_t)n * lda, NAN), b((size_t)n * ldb, -123.0), ex((size_t)n * ldx, -123.0);
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j < n; ++j)
                        if (upper ? j >= i : j <= i)
                            a[i * lda + j] = i == j ? (unit ? NAN : 2.0 + 0.02 * i) : 0.01 * std::sin(double(i * n + j + 1));
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j < nrhs; ++j) ex[i * ldx + j] = std::sin(double(i * nrhs + j + 1));
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j < nrhs; ++j)
                    {
                        double s = 0;
                        for (int k = 0; k < n; ++k)
                        {
                            const int row = transpose ? k : i, col = transpose ? i : k;
                            if (upper ? col < row : col > row) continue;
                            s += (unit && row == col ? 1.0 : a[row * lda + col]) * ex[k * ldx + j];
                        }
                        b[i * ldb + j] = s;
                    }
                dbuf<double> da(a.size()), db(b.size()), dx((size_t)n * ldx);
                da.up(a);
                db.up(b);
                dx.up(std::vector<double>((size_t)n * ldx, -123.0));
                linalg::triangular_solver<double, B>::apply(upper, transpose, unit, n, nrhs, da.p, lda, db.p, ldb, dx.p, ldx, nullptr, 0);
                cudaDeviceSynchronize();
                auto x = dx.down();
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j < ldx; ++j)
                        all_ok = all_ok && (j < nrhs ? std::fabs(x[i * ldx + j] - ex[i * ldx + j]) <= 1e-12 : x[i * ldx + j] == -123.0);
            }
    CHECK(all_ok, "triangular_solver known answers, padding preserved");
}

static void test_multiplication()
{
    const int rows = 256, cols = 128, depth = 128;
    bool      all_ok = true;
    for (bool ta : {false, true})
        for (bool tb : {false, true})
        {
            auto a = random_matrix(ta ? depth : rows, ta ? rows : depth, 4);
            auto b = random_matrix(tb ? cols : depth, tb ? depth : cols, 5);
            dbuf<double> da(a.size()), db(b.size()), dc((size_t)rows * cols);
            da.up(a);
            db.up(b);
            linalg::multiplication<double, B>::apply(ta, tb, rows, cols, depth, da.p, ta ? rows : depth, db.p, tb ? depth : cols, dc.p, cols, nullptr, 0);
            cudaDeviceSynchronize();
            auto c = dc.down();
            for (int i = 0; i < rows; ++i)
                for (int j = 0; j < cols; ++j)
                {
                    double s = 0;
                    for (int k = 0; k < depth; ++k)
                        s += (ta ? a[k * rows + i] : a[i * depth + k]) * (tb ? b[j * depth + k] : b[k * cols + j]);
                    all_ok = all_ok && std::fabs(s - c[i * cols + j]) <= 1e-9;
                }
        }
    CHECK(all_ok, "multiplication all transpose combinations");
}

static void test_validation()
{
    int threw = 0;
    try { linalg::lu_decomposition<double, B>::apply(nullptr, 4, nullptr, nullptr, 0); } catch (const std::invalid_argument&) { ++threw; }
    try { linalg::linear_solver<double, B>::apply(nullptr, nullptr, 0, nullptr, linalg::linear_solver_type::LU_LINEAR_SOLVER, nullptr, 0); } catch (const std::invalid_argument&) { ++threw; }
    try { double* p = nullptr; linalg::multiplication<double, B>::apply(false, false, 0, 1, 1, 1.0, p, 1, p, 1, 0.0, p, 1, nullptr, 0); } catch (const std::invalid_argument&) { ++threw; }
    CHECK(threw == 3, "null or zero-size arguments throw invalid_argument");
}

static void test_singular_status()
{
    dbuf<double>     m(4);
    dbuf<linalg_int> piv(2);
    m.up(std::vector<double>(4, 0.0));
    const size_t        bytes = linalg::lu_decomposition<double, B>::workspace_size(2);
    dbuf<unsigned char> ws(bytes);
    int                 info = 0;
    const bool ok = linalg::lu_decomposition<double, B>::apply(m.p, 2, piv.p, ws.p, bytes, &info);
    CHECK(!ok && info == 1, "singular 2x2 zeros: false, info 1");
}

// Mirrors the reference's GPU inversion test (A * A^-1 == I on an SPD matrix
// of order 23, null pivot allowed in LU mode) and its 2x2 determinant case.
static void test_inversion_determinant()
{
    const int n = 23;
    auto      r = random_matrix(n, n, 11, -1, 1);
    std::vector<double> a((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
            double s = 0;
            for (int k = 0; k < n; ++k) s += r[i * n + k] * r[j * n + k];
            a[i * n + j] = s + (i == j ? n : 0.0);
        }
    const auto          type  = linalg::linear_solver_type::LU_LINEAR_SOLVER;
    const size_t        bytes = linalg::inversion<double, B>::workspace_size(n, type);
    dbuf<unsigned char> ws(bytes);
    dbuf<double>        dm(a.size());
    dm.up(a);
    linalg::inversion<double, B>::apply(dm.p, nullptr, n, type, ws.p, bytes);
    cudaDeviceSynchronize();
    auto   inv = dm.down();
    double err = 0;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
            double s = 0;
            for (int k = 0; k < n; ++k) s += inv[i * n + k] * a[k * n + j];
            err = std::fmax(err, std::fabs(s - (i == j ? 1.0 : 0.0)));
        }
    CHECK(err <= 1e-12 * n, "inversion LU mode, null pivot: A^-1 A == I");

    dm.up(a);
    const size_t        dbytes = linalg::determinant<double, B>::workspace_size(n, type);
    dbuf<unsigned char> dws(dbytes);
    const double        det = linalg::determinant<double, B>::apply(dm.p, nullptr, n, type, dws.p, dbytes);
    CHECK(det > 0.0, "determinant of an SPD matrix is positive");

    dm.up(a);
    const auto   ctype  = linalg::linear_solver_type::CHOLESKY_LINEAR_SOLVER;
    const size_t cbytes = linalg::determinant<double, B>::workspace_size(n, ctype);
    dbuf<unsigned char> cws(cbytes);
    const double cdet = linalg::determinant<double, B>::apply(dm.p, nullptr, n, ctype, cws.p, cbytes);
    CHECK(std::fabs(cdet - det) <= 1e-10 * std::fabs(det), "determinant CHOLESKY mode == LU mode on an SPD matrix");

    dbuf<double> d2(4);
    d2.up({4.0, 0.0, 0.0, 2.0});
    cudaStream_t s = nullptr;
    cudaStreamCreate(&s);
    const double det2 = linalg::determinant<double, B>::apply(d2.p, nullptr, 2, type, dws.p, dbytes, s);
    cudaStreamDestroy(s);
    CHECK(det2 == 8.0, "determinant [[4,0],[0,2]] == 8");

    dbuf<float> f2(4);
    f2.up(std::vector<float>{0.0f, 1.0f, 1.0f, 0.0f});
    const size_t        fbytes = linalg::determinant<float, B>::workspace_size(2, type);
    dbuf<unsigned char> fws(fbytes);
    const float fdet = linalg::determinant<float, B>::apply(f2.p, nullptr, 2, type, fws.p, fbytes);
    CHECK(fdet == -1.0f, "determinant of a row swap is -1 (pivot sign applied)");

    int threw = 0;
    try { linalg::inversion<double, B>::apply(nullptr, nullptr, n, type, ws.p, bytes); } catch (const std::invalid_argument&) { ++threw; }
    try { linalg::inversion<double, B>::apply(dm.p, nullptr, 0, type, ws.p, bytes); } catch (const std::invalid_argument&) { ++threw; }
    try { linalg::inversion<double, B>::apply(dm.p, nullptr, n, (linalg::linear_solver_type)5, ws.p, bytes); } catch (const std::invalid_argument&) { ++threw; }
    try { linalg::determinant<double, B>::apply(nullptr, nullptr, n, type, dws.p, dbytes); } catch (const std::invalid_argument&) { ++threw; }
    CHECK(threw == 4, "inversion / determinant argument checks throw");
}

// batched_matrix_multiplication: each entry the fma chain over k from zero
static void test_cholesky()
{
    const int n = 150;
    auto      r = random_matrix(n, n, 17, -1, 1);
    std::vector<double> a((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
        {
            double s = 0;
            for (int k = 0; k < n; ++k) s += r[i * n + k] * r[j * n + k];
            a[i * n + j] = s + (i == j ? n : 0.0);
        }
    using CD          = linalg::cholesky_decomposition<double, B>;
    const auto   low  = linalg::cholesky_decomposition_enum::LOWER_TRIANGULAR;
    const auto   up   = linalg::cholesky_decomposition_enum::UPPER_TRIANGULAR;
    const size_t bytes = CD::workspace_size(n, low);
    dbuf<unsigned char> ws(bytes);
    dbuf<double>        dm(a.size());
    for (auto type : {low, up})
    {
        dm.up(a);
        int        info = -1;
        const bool ok   = CD::apply(dm.p, n, type, ws.p, bytes, &info);
        auto       f    = dm.down();
        double     err = 0, other = 0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
            {
                double s = 0;  // (L L^T)_ij, or (U^T U)_ij
                for (int k = 0; k < n; ++k)
                    s += type == low ? f[i * n + k] * f[j * n + k] : f[k * n + i] * f[k * n + j];
                err = std::fmax(err, std::fabs(s - a[i * n + j]));
                if (type == low ? j > i : j < i) other = std::fmax(other, std::fabs(f[i * n + j]));
            }
        CHECK(ok && info == 0 && err <= 1e-11 * n && other == 0.0,
            type == low ? "cholesky_decomposition LOWER: L L^T == A" : "cholesky_decomposition UPPER: U^T U == A");
    }
    std::vector<double> bad = a;
    bad[40 * n + 40]        = -1.0;
    dm.up(bad);
    int info = 0;
    CHECK(!CD::apply(dm.p, n, low, ws.p, bytes, &info) && info == 41,
        "cholesky_decomposition: non-positive pivot -> false, info = row + 1");
    bool threw = false;
    try
    {
        CD::apply(dm.p, n, static_cast<linalg::cholesky_decomposition_enum>('X'), ws.p, bytes, &info);
    }
    catch (const std::invalid_argument&)
    {
        threw = true;
    }
    CHECK(threw, "cholesky_decomposition: unknown enum throws std::invalid_argument");
    dbuf<float> f2(4);
    f2.up(std::vector<float>{4.0f, 2.0f, 2.0f, 5.0f});
    dbuf<unsigned char> fws(linalg::cholesky_decomposition<float, B>::workspace_size(2, low));
    linalg::cholesky_decomposition<float, B>::apply(f2.p, 2, low, fws.p, fws.n, &info);
    const auto l = f2.down();
    CHECK(info == 0 && l[0] == 2.0f && l[1] == 0.0f && l[2] == 1.0f && l[3] == 2.0f,
        "cholesky_decomposition<float>: [[4,2],[2,5]] -> [[2,0],[1,2]]");
}

static void test_transpose()
{
    using TD = linalg::transpose<double, B>;
    for (auto shape : {std::pair<int, int>{130, 130}, std::pair<int, int>{70, 200}})
    {
        const int           rows = shape.first, cols = shape.second;
        std::vector<double> a((size_t)rows * cols);
        for (size_t e = 0; e < a.size(); ++e) a[e] = (double)e;
        dbuf<double>        dm(a.size());
        dm.up(a);
        const size_t        bytes = TD::workspace_size(rows, cols);
        dbuf<unsigned char> ws(bytes ? bytes : 1);
        TD::apply(rows, cols, dm.p, ws.p, bytes);
        cudaDeviceSynchronize();
        const auto t  = dm.down();
        bool       ok = (rows == cols) == (bytes == 0);
        for (int i = 0; i < rows; ++i)
            for (int j = 0; j < cols; ++j) ok = ok && t[(size_t)j * rows + i] == a[(size_t)i * cols + j];
        CHECK(ok, rows == cols ? "transpose square, in place, no workspace" : "transpose 70 x 200 through the workspace");
    }
    bool threw = false;
    try
    {
        TD::apply(0, 4, nullptr, nullptr, 0);
    }
    catch (const std::invalid_argument&)
    {
        threw = true;
    }
    CHECK(threw, "transpose: null matrix throws std::invalid_argument");
}

static void test_batched_multiplication()
{
    const int dim = 37, count = 4;
    auto      a = random_matrix(count * dim, dim, 21);
    auto      b = random_matrix(count * dim, dim, 22);
    dbuf<double> da(a.size()), db(b.size()), dc(a.size());
    da.up(a);
    db.up(b);
    linalg::batched_matrix_multiplication(dim, count, da.p, db.p, dc.p);
    cudaDeviceSynchronize();
    auto c  = dc.down();
    bool ok = true;
    for (int q = 0; q < count; ++q)
        for (int i = 0; i < dim; ++i)
            for (int j = 0; j < dim; ++j)
            {
                double s = 0;
                for (int k = 0; k < dim; ++k)
                    s = std::fma(a[(size_t)q * dim * dim + i * dim + k], b[(size_t)q * dim * dim + k * dim + j], s);
                ok = ok && s == c[(size_t)q * dim * dim + i * dim + j];
            }
    CHECK(ok, "batched_matrix_multiplication bit-identical to the fma chain");
    int threw = 0;
    try { linalg::batched_matrix_multiplication(0, count, da.p, db.p, dc.p); } catch (const std::invalid_argument&) { ++threw; }
    try { linalg::batched_matrix_multiplication(dim, count, static_cast<const double*>(nullptr), db.p, dc.p); } catch (const std::invalid_argument&) { ++threw; }
    CHECK(threw == 2, "batched_matrix_multiplication argument checks throw");
}

int main()
{
    test_lu();
    test_linear_solver();
    test_triangular();
    test_multiplication();
    test_validation();
    test_singular_status();
    test_inversion_determinant();
    test_cholesky();
    test_transpose();
    test_batched_multiplication();
    std::printf("%s (%d failures)\n", g_fail ? "FAILED" : "ALL PASSED", g_fail);
    return g_fail ? 1 : 0;
}
