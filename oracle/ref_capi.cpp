/*
 * extern "C" wrappers over the reference's own NATIVE specializations, so the
 * Python tests and the CPU baseline arm of bench.py can call the reference
 * implementation through ctypes.  Compiled together with the reference's
 * sources (src/matrix_operation/cpu/native/{lu_decomposition,linear_solver,
 * triangular_solver,multiplication,cholesky_decomposition,inversion}_native.cpp
 * and src/matrix_operation/cpu/determinant.cpp) by oracle/Makefile into
 * oracle/_ref/libref_native.so.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the B200 library links or calls this.
 *
 * Every wrapper allocates the workspace the reference asks for with
 * workspace_size() (the reference never allocates by itself), catches the
 * reference's exceptions and returns a status:
 *    0  success
 *    1  lu_decomposition reported a singular U (info written)
 *   -1  the reference threw (invalid argument)
 *   -2  allocation failure
 */
#include <cstdint>
#include <new>
#include <vector>

#include "include/matrix_operation/cholesky_decomposition.h"
#include "include/matrix_operation/determinant.h"
#include "include/matrix_operation/inversion.h"
#include "include/matrix_operation/linear_solver.h"
#include "include/matrix_operation/lu_decomposition.h"
#include "include/matrix_operation/multiplication.h"
#include "include/matrix_operation/transpose.h"
#include "include/matrix_operation/triangular_solver.h"

using linalg::linalg_backend;

namespace
{
template <typename T> int ref_getrf(T* m, int64_t n, int64_t* pivot, int* info)
{
    try
    {
        const size_t bytes = linalg::lu_decomposition<T, linalg_backend::NATIVE>::workspace_size(n);
        std::vector<unsigned char> ws(bytes ? bytes : 1);
        int local_info   = -1;
        const bool ok = linalg::lu_decomposition<T, linalg_backend::NATIVE>::apply(
            m, n, reinterpret_cast<linalg_int*>(pivot), ws.data(), bytes, &local_info);
        if (info)
        {
            *info = local_info;
        }
        return ok ? 0 : 1;
    }
    catch (const std::bad_alloc&)
    {
        return -2;
    }
    catch (...)
    {
        return -1;
    }
}

template <typename T>
int ref_gesv(T* m, int64_t* pivot, int64_t n, T* x, int type)
{
    try
    {
        const auto t     = static_cast<linalg::linear_solver_type>(type);
        const size_t bytes = linalg::linear_solver<T, linalg_backend::NATIVE>::workspace_size(n, t);
        std::vector<unsigned char> ws(bytes ? bytes : 1);
        linalg::linear_solver<T, linalg_backend::NATIVE>::apply(
            m, reinterpret_cast<linalg_int*>(pivot), n, x, t, ws.data(), bytes);
        return 0;
    }
    catch (const std::bad_alloc&)
    {
        return -2;
    }
    catch (...)
    {
        return -1;
    }
}

template <typename T>
int ref_trsm(int upper, int transpose, int unit, int64_t n, int64_t nrhs, const T* a,
    int64_t lda, const T* b, int64_t ldb, T* x, int64_t ldx)
{
    try
    {
        size_t bytes = 0;
        if (n > 0 && nrhs > 0)
        {
            bytes = linalg::triangular_solver<T, linalg_backend::NATIVE>::workspace_size(n, nrhs);
        }
        std::vector<unsigned char> ws(bytes ? bytes : 1);
        linalg::triangular_solver<T, linalg_backend::NATIVE>::apply(upper != 0, transpose != 0,
            unit != 0, n, nrhs, a, lda, b, ldb, x, ldx, ws.data(), bytes);
        return 0;
    }
    catch (const std::bad_alloc&)
    {
        return -2;
    }
    catch (...)
    {
        return -1;
    }
}

template <typename T>
int ref_gemm(int ta, int tb, int64_t rows, int64_t cols, int64_t depth, T alpha, const T* a,
    int64_t lda, const T* b, int64_t ldb, T beta, T* c, int64_t ldc)
{
    try
    {
        size_t bytes = 0;
        if (rows > 0 && cols > 0 && depth > 0)
        {
            bytes = linalg::multiplication<T, linalg_backend::NATIVE>::workspace_size(
                rows, cols, depth);
        }
        std::vector<unsigned char> ws(bytes ? bytes : 1);
        linalg::multiplication<T, linalg_backend::NATIVE>::apply(ta != 0, tb != 0, rows, cols,
            depth, alpha, a, lda, b, ldb, beta, c, ldc, ws.data(), bytes);
        return 0;
    }
    catch (const std::bad_alloc&)
    {
        return -2;
    }
    catch (...)
    {
        return -1;
    }
}
template <typename T> int ref_potrf(T* m, int64_t n, int upper, int* info)
{
    try
    {
        int        local = -1;
        const auto type  = upper ? linalg::cholesky_decomposition_enum::UPPER_TRIANGULAR
                                 : linalg::cholesky_decomposition_enum::LOWER_TRIANGULAR;
        const bool ok    = linalg::cholesky_decomposition<T, linalg_backend::NATIVE>::apply(m, n, type, nullptr, 0,
            &local);
        if (info)
        {
            *info = local;
        }
        return ok ? 0 : 1;
    }
    catch (...)
    {
        return -1;
    }
}

template <typename T> int ref_getri(T* m, int64_t* pivot, int64_t n, int type)
{
    try
    {
        const auto   t     = static_cast<linalg::linear_solver_type>(type);
        const size_t bytes = linalg::inversion<T, linalg_backend::NATIVE>::workspace_size(n, t);
        std::vector<unsigned char> ws(bytes ? bytes : 1);
        linalg::inversion<T, linalg_backend::NATIVE>::apply(
            m, reinterpret_cast<linalg_int*>(pivot), n, t, ws.data(), bytes);
        return 0;
    }
    catch (const std::bad_alloc&)
    {
        return -2;
    }
    catch (...)
    {
        return -1;
    }
}

template <typename T> int ref_det(T* m, int64_t* pivot, int64_t n, int type, T* out)
{
    try
    {
        const auto   t     = static_cast<linalg::linear_solver_type>(type);
        const size_t bytes = linalg::determinant<T, linalg_backend::NATIVE>::workspace_size(n, t);
        std::vector<unsigned char> ws(bytes ? bytes : 1);
        *out = linalg::determinant<T, linalg_backend::NATIVE>::apply(
            m, reinterpret_cast<linalg_int*>(pivot), n, t, ws.data(), bytes);
        return 0;
    }
    catch (const std::bad_alloc&)
    {
        return -2;
    }
    catch (...)
    {
        return -1;
    }
}
template <typename T> int ref_transpose(int64_t rows, int64_t cols, T* m)
{
    try
    {
        const size_t bytes = linalg::transpose<T, linalg_backend::NATIVE>::workspace_size(rows, cols);
        std::vector<unsigned char> ws(bytes ? bytes : 1);
        linalg::transpose<T, linalg_backend::NATIVE>::apply(rows, cols, m, ws.data(), bytes);
        return 0;
    }
    catch (const std::bad_alloc&)
    {
        return -2;
    }
    catch (...)
    {
        return -1;
    }
}
}  // namespace

extern "C" {
int ref_dgetrf(double* m, int64_t n, int64_t* pivot, int* info)
{
    return ref_getrf(m, n, pivot, info);
}
int ref_sgetrf(float* m, int64_t n, int64_t* pivot, int* info)
{
    return ref_getrf(m, n, pivot, info);
}
int ref_dgesv(double* m, int64_t* pivot, int64_t n, double* x, int type)
{
    return ref_gesv(m, pivot, n, x, type);
}
int ref_sgesv(float* m, int64_t* pivot, int64_t n, float* x, int type)
{
    return ref_gesv(m, pivot, n, x, type);
}
int ref_dtrsm(int upper, int transpose, int unit, int64_t n, int64_t nrhs, const double* a,
    int64_t lda, const double* b, int64_t ldb, double* x, int64_t ldx)
{
    return ref_trsm(upper, transpose, unit, n, nrhs, a, lda, b, ldb, x, ldx);
}
int ref_strsm(int upper, int transpose, int unit, int64_t n, int64_t nrhs, const float* a,
    int64_t lda, const float* b, int64_t ldb, float* x, int64_t ldx)
{
    return ref_trsm(upper, transpose, unit, n, nrhs, a, lda, b, ldb, x, ldx);
}
int ref_dgemm(int ta, int tb, int64_t rows, int64_t cols, int64_t depth, double alpha,
    const double* a, int64_t lda, const double* b, int64_t ldb, double beta, double* c,
    int64_t ldc)
{
    return ref_gemm(ta, tb, rows, cols, depth, alpha, a, lda, b, ldb, beta, c, ldc);
}
int ref_sgemm(int ta, int tb, int64_t rows, int64_t cols, int64_t depth, float alpha,
    const float* a, int64_t lda, const float* b, int64_t ldb, float beta, float* c, int64_t ldc)
{
    return ref_gemm(ta, tb, rows, cols, depth, alpha, a, lda, b, ldb, beta, c, ldc);
}
int ref_dpotrf(double* m, int64_t n, int upper, int* info)
{
    return ref_potrf(m, n, upper, info);
}
int ref_spotrf(float* m, int64_t n, int upper, int* info)
{
    return ref_potrf(m, n, upper, info);
}
int ref_dgetri(double* m, int64_t* pivot, int64_t n, int type)
{
    return ref_getri(m, pivot, n, type);
}
int ref_sgetri(float* m, int64_t* pivot, int64_t n, int type)
{
    return ref_getri(m, pivot, n, type);
}
int ref_ddet(double* m, int64_t* pivot, int64_t n, int type, double* out)
{
    return ref_det(m, pivot, n, type, out);
}
int ref_sdet(float* m, int64_t* pivot, int64_t n, int type, float* out)
{
    return ref_det(m, pivot, n, type, out);
}
int ref_dtranspose(int64_t rows, int64_t cols, double* m)
{
    return ref_transpose(rows, cols, m);
}
int ref_stranspose(int64_t rows, int64_t cols, float* m)
{
    return ref_transpose(rows, cols, m);
}
size_t ref_dgetrf_workspace_size(int64_t n)
{
    return linalg::lu_decomposition<double, linalg_backend::NATIVE>::workspace_size(n);
}
}
