/*
 * The reference's public operator interface for the LU-solve path, restated
 * so the B200 specializations compile without the reference tree:
 *   include/common/backend.h:21-29            linalg_backend (+ B200 appended)
 *   include/common/types.h:26-27              linalg_int
 *   include/matrix_operation/lu_decomposition.h:15-54
 *   include/matrix_operation/linear_solver.h:15-65
 *   include/matrix_operation/triangular_solver.h:20-38
 *   include/matrix_operation/multiplication.h:15-114
 *   include/matrix_operation/inversion.h:15-53
 *   include/matrix_operation/determinant.h
 *   include/matrix_operation/multiplication_batched.h
 *   include/matrix_operation/cholesky_decomposition.h:15-94
 *   include/matrix_operation/transpose.h
 * Names, argument order, default arguments and meaning are the reference's;
 * that is what makes the backend a drop-in.  Inside the reference tree define
 * LINALG_B200_USE_REFERENCE_HEADERS and add B200 as the last enumerator of
 * linalg_backend instead (INTEGRATION.md shows the one-line patch).
 */
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(LINALG_B200_USE_REFERENCE_HEADERS)
#include "include/common/backend.h"
#include "include/common/types.h"
#include "include/matrix_operation/cholesky_decomposition.h"
#include "include/matrix_operation/determinant.h"
#include "include/matrix_operation/inversion.h"
#include "include/matrix_operation/linear_solver.h"
#include "include/matrix_operation/lu_decomposition.h"
#include "include/matrix_operation/multiplication.h"
#include "include/matrix_operation/multiplication_batched.h"
#include "include/matrix_operation/transpose.h"
#include "include/matrix_operation/triangular_solver.h"
#else

#if !defined(linalg_int)
#define linalg_int long long int
#define linalg_long unsigned long long int
#endif

#if !defined(LINALG_API)
#if defined(__GNUC__)
#define LINALG_API __attribute__((visibility("default")))
#else
#define LINALG_API
#endif
#endif

namespace linalg
{
enum class linalg_backend : std::uint8_t
{
    NATIVE,
    BLAS_LAPACKE,
    MKL,
    CUDA_BLAS,
    ROCM_BLAS,
    METAL_BLAS,
    B200
};

enum class linear_solver_type : std::uint8_t
{
    LU_LINEAR_SOLVER               = 1,
    LU_UPFRONT_LINEAR_SOLVER       = 2,
    CHOLESKY_LINEAR_SOLVER         = 3,
    CHOLESKY_UPFRONT_LINEAR_SOLVER = 4,
};

enum class cholesky_decomposition_enum : char
{
    LOWER_TRIANGULAR = 'L',
    UPPER_TRIANGULAR = 'U'
};

template <typename T, linalg_backend Backend> struct cholesky_decomposition
{
    LINALG_API static bool apply(T* C, linalg_int lda, cholesky_decomposition_enum type, void* workspace,
        size_t workspace_size, int* info = nullptr, void* stream = nullptr);
    LINALG_API static bool apply_aad(T* L_aad, const T* L, linalg_int lda, cholesky_decomposition_enum type,
        T* A_aad);
    LINALG_API static size_t workspace_size(linalg_int lda, cholesky_decomposition_enum type);
};

template <typename T, linalg_backend Backend> struct lu_decomposition
{
    LINALG_API static bool apply(T* m, linalg_int lda, linalg_int* pivot, void* workspace,
        size_t workspace_size, int* info = nullptr, void* stream = nullptr);
    LINALG_API static size_t workspace_size(linalg_int lda);
};

template <typename T, linalg_backend Backend> struct linear_solver
{
    LINALG_API static void apply(T* m, linalg_int* pivot, linalg_int lda, T* x,
        linear_solver_type type, void* workspace, size_t workspace_size, void* stream = nullptr);
    LINALG_API static size_t workspace_size(linalg_int lda, linear_solver_type type);
};

template <typename T, linalg_backend Backend> struct triangular_solver
{
    LINALG_API static void apply(bool upper, bool transpose, bool unit_diagonal, linalg_int n,
        linalg_int nrhs, const T* a, linalg_int lda, const T* b, linalg_int ldb, T* x,
        linalg_int ldx, void* workspace, size_t workspace_size, void* stream = nullptr);
    LINALG_API static size_t workspace_size(linalg_int n, linalg_int nrhs);
};

template <typename T, linalg_backend Backend> struct multiplication
{
    LINALG_API static void apply(bool transpose_a, bool transpose_b, linalg_int rows,
        linalg_int columns, linalg_int depth, T alpha, const T* a, linalg_int lda, const T* b,
        linalg_int ldb, T beta, T* c, linalg_int ldc, void* workspace, size_t workspace_size,
        void* stream = nullptr);

    static void apply(bool transpose_a, bool transpose_b, linalg_int rows, linalg_int columns,
        linalg_int depth, const T* a, linalg_int lda, const T* b, linalg_int ldb, T* c,
        linalg_int ldc, void* workspace, size_t workspace_size, void* stream = nullptr)
    {
        apply(transpose_a, transpose_b, rows, columns, depth, T(1), a, lda, b, ldb, T(0), c, ldc,
            workspace, workspace_size, stream);
    }

    LINALG_API static size_t workspace_size(linalg_int rows, linalg_int columns, linalg_int depth);
};

template <typename T, linalg_backend Backend> struct inversion
{
    LINALG_API static void apply(T* m, linalg_int* pivot, linalg_int lda, linear_solver_type type,
        void* workspace, size_t workspace_size, void* stream = nullptr);
    LINALG_API static size_t workspace_size(linalg_int lda, linear_solver_type type);
};

LINALG_API void batched_matrix_multiplication(linalg_int dim, linalg_int count, const float* a, const float* b,
    float* c, void* stream = nullptr);
LINALG_API void batched_matrix_multiplication(linalg_int dim, linalg_int count, const double* a,
    const double* b, double* c, void* stream = nullptr);

template <typename T, linalg_backend Backend> struct determinant
{
    LINALG_API static T apply(T* m, linalg_int* pivot, linalg_int lda, linear_solver_type type,
        void* workspace, size_t workspace_size, void* stream = nullptr);
    LINALG_API static size_t workspace_size(linalg_int lda, linear_solver_type type);
};

template <typename T, linalg_backend Backend> struct transpose
{
    LINALG_API static void apply(linalg_long rows, linalg_long columns, T* m, void* workspace,
        size_t workspace_size, void* stream = nullptr);
    LINALG_API static size_t workspace_size(linalg_long rows, linalg_long columns);
};
}  // namespace linalg
#endif
