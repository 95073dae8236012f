/*
 * extern "C" wrappers over the reference's own CUDA_BLAS (cuSOLVER) LU solve,
 * linear_solver<double, linalg_backend::CUDA_BLAS> in LU and Cholesky modes, and its
 * CUDA_BLAS inversion and determinant in LU mode, so bench.py can time the
 * reference's GPU backend beside this library.  Compiled together with the
 * reference's sources (src/matrix_operation/gpu/cublas/{linear_solver,
 * lu_decomposition,transpose,cholesky_decomposition}_cublas.cpp,
 * inversion_cublas.cu and multiplication_batched_cublas.cu) by
 * baseline/Makefile into
 * baseline/_ref/libref_cublas.so.
 *
 * Timing-comparison code only.  Nothing in the B200 library links or calls
 * this; it runs NVIDIA's cuSOLVER and cuBLAS exactly as the reference does.
 *
 * All pointers are device pointers (the reference's GPU contract); the
 * caller passes a workspace of ref_cublas_dgesv_workspace_size(n) bytes.
 * Returns 0, or -1 if the reference threw (message in ref_cublas_last_error).
 */
#include <cstdint>
#include <cstring>
#include <exception>
#include <string>

#include "include/matrix_operation/determinant.h"
#include "include/matrix_operation/inversion.h"
#include "include/matrix_operation/linear_solver.h"
#include "include/matrix_operation/multiplication_batched.h"
#include "include/matrix_operation/transpose.h"

using linalg::linalg_backend;
using linalg::linear_solver_type;

namespace
{
thread_local std::string g_err;
}

extern "C" {

const char* ref_cublas_last_error(void) { return g_err.c_str(); }

size_t ref_cublas_dgesv_workspace_size(int64_t n)
{
    try
    {
        return linalg::linear_solver<double, linalg_backend::CUDA_BLAS>::workspace_size(
            n, linear_solver_type::LU_LINEAR_SOLVER);
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return 0;
    }
}

int ref_cublas_dgesv(double* m, int64_t* pivot, int64_t n, double* x, void* ws, size_t ws_bytes, void* stream)
{
    try
    {
        linalg::linear_solver<double, linalg_backend::CUDA_BLAS>::apply(m, reinterpret_cast<linalg_int*>(pivot), n,
            x, linear_solver_type::LU_LINEAR_SOLVER, ws, ws_bytes, stream);
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return -1;
    }
}

/* linear_solver<double, CUDA_BLAS> in CHOLESKY_LINEAR_SOLVER mode (cuSOLVER
 * potrf + potrs); pivot is unused by that mode. */
size_t ref_cublas_dcholesky_solve_workspace_size(int64_t n)
{
    try
    {
        return linalg::linear_solver<double, linalg_backend::CUDA_BLAS>::workspace_size(
            n, linear_solver_type::CHOLESKY_LINEAR_SOLVER);
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return 0;
    }
}

int ref_cublas_dcholesky_solve(double* m, int64_t n, double* x, void* ws, size_t ws_bytes, void* stream)
{
    try
    {
        linalg::linear_solver<double, linalg_backend::CUDA_BLAS>::apply(m, nullptr, n, x,
            linear_solver_type::CHOLESKY_LINEAR_SOLVER, ws, ws_bytes, stream);
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return -1;
    }
}

/* transpose<double, CUDA_BLAS> in place (cuBLAS geam into scratch, then a
 * device-to-device copy back). */
size_t ref_cublas_dtranspose_workspace_size(int64_t rows, int64_t cols)
{
    try
    {
        return linalg::transpose<double, linalg_backend::CUDA_BLAS>::workspace_size(rows, cols);
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return 0;
    }
}

int ref_cublas_dtranspose(int64_t rows, int64_t cols, double* m, void* ws, size_t ws_bytes, void* stream)
{
    try
    {
        linalg::transpose<double, linalg_backend::CUDA_BLAS>::apply(rows, cols, m, ws, ws_bytes, stream);
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return -1;
    }
}

size_t ref_cublas_dinverse_workspace_size(int64_t n)
{
    try
    {
        return linalg::inversion<double, linalg_backend::CUDA_BLAS>::workspace_size(
            n, linear_solver_type::LU_LINEAR_SOLVER);
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return 0;
    }
}

int ref_cublas_dinverse(double* m, int64_t n, void* ws, size_t ws_bytes, void* stream)
{
    try
    {
        linalg::inversion<double, linalg_backend::CUDA_BLAS>::apply(
            m, nullptr, n, linear_solver_type::LU_LINEAR_SOLVER, ws, ws_bytes, stream);
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return -1;
    }
}

size_t ref_cublas_ddeterminant_workspace_size(int64_t n)
{
    try
    {
        return linalg::determinant<double, linalg_backend::CUDA_BLAS>::workspace_size(
            n, linear_solver_type::LU_LINEAR_SOLVER);
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return 0;
    }
}

int ref_cublas_ddeterminant(double* m, int64_t n, double* out, void* ws, size_t ws_bytes, void* stream)
{
    try
    {
        *out = linalg::determinant<double, linalg_backend::CUDA_BLAS>::apply(
            m, nullptr, n, linear_solver_type::LU_LINEAR_SOLVER, ws, ws_bytes, stream);
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return -1;
    }
}

int ref_cublas_dgemm_batched(int64_t dim, int64_t count, const double* a, const double* b, double* c, void* stream)
{
    try
    {
        linalg::batched_matrix_multiplication(dim, count, a, b, c, stream);
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return -1;
    }
}

int ref_cublas_sgemm_batched(int64_t dim, int64_t count, const float* a, const float* b, float* c, void* stream)
{
    try
    {
        linalg::batched_matrix_multiplication(dim, count, a, b, c, stream);
        return 0;
    }
    catch (const std::exception& e)
    {
        g_err = e.what();
        return -1;
    }
}
}
