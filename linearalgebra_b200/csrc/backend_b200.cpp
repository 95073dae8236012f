// linalg_backend::B200 specializations of the reference's operator templates
// (include/linalg_b200/backend_b200.h), each a thin shim over the C ABI.
#include "../../include/linalg_b200/backend_b200.h"

#include <stdexcept>
#include <string>

#include "../../include/b200la.h"

namespace linalg
{
namespace
{
// Turn a negative C-ABI status into the exception the reference's checks
// would raise; pass non-negative statuses through.
int check_status(int st)
{
    if (st >= 0)
    {
        return st;
    }
    const std::string msg = b200la_last_error();
    if (st == B200LA_INVALID_ARGUMENT || st == B200LA_WORKSPACE_TOO_SMALL ||
        st == B200LA_NOT_SUPPORTED)
    {
        throw std::invalid_argument(msg);
    }
    throw std::runtime_error(msg);
}

int64_t* pv(linalg_int* p) { return reinterpret_cast<int64_t*>(p); }

// 0 lower, 1 upper; any other enum value reaches the C ABI as 2, which
// rejects it ("Unsupported enum type!", as cholesky_decomposition_native.cpp)
int triangle(cholesky_decomposition_enum type)
{
    return type == cholesky_decomposition_enum::LOWER_TRIANGULAR   ? 0
           : type == cholesky_decomposition_enum::UPPER_TRIANGULAR ? 1
                                                                   : 2;
}
}  // namespace

// ---- cholesky_decomposition -------------------------------------------------
template <>
bool cholesky_decomposition<double, linalg_backend::B200>::apply(double* C, linalg_int lda,
    cholesky_decomposition_enum type, void* workspace, size_t workspace_size, int* info, void* stream)
{
    return check_status(b200la_dpotrf(C, lda, triangle(type), workspace, workspace_size, info, stream)) ==
           B200LA_SUCCESS;
}
template <>
bool cholesky_decomposition<float, linalg_backend::B200>::apply(float* C, linalg_int lda,
    cholesky_decomposition_enum type, void* workspace, size_t workspace_size, int* info, void* stream)
{
    return check_status(b200la_spotrf(C, lda, triangle(type), workspace, workspace_size, info, stream)) ==
           B200LA_SUCCESS;
}
template <>
bool cholesky_decomposition<double, linalg_backend::B200>::apply_aad(double*, const double*, linalg_int,
    cholesky_decomposition_enum, double*)
{
    throw std::invalid_argument("cholesky_decomposition<double, B200>::apply_aad: not provided by this backend");
}
template <>
bool cholesky_decomposition<float, linalg_backend::B200>::apply_aad(float*, const float*, linalg_int,
    cholesky_decomposition_enum, float*)
{
    throw std::invalid_argument("cholesky_decomposition<float, B200>::apply_aad: not provided by this backend");
}
template <>
size_t cholesky_decomposition<double, linalg_backend::B200>::workspace_size(linalg_int lda,
    cholesky_decomposition_enum)
{
    return b200la_dgetrf_workspace_size(lda);
}
template <>
size_t cholesky_decomposition<float, linalg_backend::B200>::workspace_size(linalg_int lda,
    cholesky_decomposition_enum)
{
    return b200la_sgetrf_workspace_size(lda);
}

// ---- lu_decomposition -------------------------------------------------------
template <>
bool lu_decomposition<double, linalg_backend::B200>::apply(double* m, linalg_int lda,
    linalg_int* pivot, void* workspace, size_t workspace_size, int* info, void* stream)
{
    return check_status(b200la_dgetrf(m, lda, pv(pivot), workspace, workspace_size, info, stream)) ==
           B200LA_SUCCESS;
}
template <>
bool lu_decomposition<float, linalg_backend::B200>::apply(float* m, linalg_int lda,
    linalg_int* pivot, void* workspace, size_t workspace_size, int* info, void* stream)
{
    return check_status(b200la_sgetrf(m, lda, pv(pivot), workspace, workspace_size, info, stream)) ==
           B200LA_SUCCESS;
}
template <> size_t lu_decomposition<double, linalg_backend::B200>::workspace_size(linalg_int lda)
{
    return b200la_dgetrf_workspace_size(lda);
}
template <> size_t lu_decomposition<float, linalg_backend::B200>::workspace_size(linalg_int lda)
{
    return b200la_sgetrf_workspace_size(lda);
}

// ---- linear_solver ----------------------------------------------------------
template <>
void linear_solver<double, linalg_backend::B200>::apply(double* m, linalg_int* pivot,
    linalg_int lda, double* x, linear_solver_type type, void* workspace, size_t workspace_size,
    void* stream)
{
    check_status(b200la_dgesv(m, pv(pivot), lda, x, static_cast<int>(type), workspace,
        workspace_size, stream));
}
template <>
void linear_solver<float, linalg_backend::B200>::apply(float* m, linalg_int* pivot, linalg_int lda,
    float* x, linear_solver_type type, void* workspace, size_t workspace_size, void* stream)
{
    check_status(b200la_sgesv(m, pv(pivot), lda, x, static_cast<int>(type), workspace,
        workspace_size, stream));
}
template <>
size_t linear_solver<double, linalg_backend::B200>::workspace_size(
    linalg_int lda, linear_solver_type type)
{
    return b200la_dgesv_workspace_size(lda, static_cast<int>(type));
}
template <>
size_t linear_solver<float, linalg_backend::B200>::workspace_size(
    linalg_int lda, linear_solver_type type)
{
    return b200la_sgesv_workspace_size(lda, static_cast<int>(type));
}

// ---- triangular_solver ------------------------------------------------------
template <>
void triangular_solver<double, linalg_backend::B200>::apply(bool upper, bool transpose,
    bool unit_diagonal, linalg_int n, linalg_int nrhs, const double* a, linalg_int lda,
    const double* b, linalg_int ldb, double* x, linalg_int ldx, void* workspace,
    size_t workspace_size, void* stream)
{
    check_status(b200la_dtrsm(upper, transpose, unit_diagonal, n, nrhs, a, lda, b, ldb, x, ldx,
        workspace, workspace_size, stream));
}
template <>
void triangular_solver<float, linalg_backend::B200>::apply(bool upper, bool transpose,
    bool unit_diagonal, linalg_int n, linalg_int nrhs, const float* a, linalg_int lda,
    const float* b, linalg_int ldb, float* x, linalg_int ldx, void* workspace,
    size_t workspace_size, void* stream)
{
    check_status(b200la_strsm(upper, transpose, unit_diagonal, n, nrhs, a, lda, b, ldb, x, ldx,
        workspace, workspace_size, stream));
}
template <>
size_t triangular_solver<double, linalg_backend::B200>::workspace_size(linalg_int n, linalg_int nrhs)
{
    return b200la_dtrsm_workspace_size(n, nrhs);
}
template <>
size_t triangular_solver<float, linalg_backend::B200>::workspace_size(linalg_int n, linalg_int nrhs)
{
    return b200la_strsm_workspace_size(n, nrhs);
}

// ---- multiplication ---------------------------------------------------------
template <>
void multiplication<double, linalg_backend::B200>::apply(bool transpose_a, bool transpose_b,
    linalg_int rows, linalg_int columns, linalg_int depth, double alpha, const double* a,
    linalg_int lda, const double* b, linalg_int ldb, double beta, double* c, linalg_int ldc,
    void* workspace, size_t workspace_size, void* stream)
{
    check_status(b200la_dgemm(transpose_a, transpose_b, rows, columns, depth, alpha, a, lda, b, ldb,
        beta, c, ldc, workspace, workspace_size, stream));
}
template <>
void multiplication<float, linalg_backend::B200>::apply(bool transpose_a, bool transpose_b,
    linalg_int rows, linalg_int columns, linalg_int depth, float alpha, const float* a,
    linalg_int lda, const float* b, linalg_int ldb, float beta, float* c, linalg_int ldc,
    void* workspace, size_t workspace_size, void* stream)
{
    check_status(b200la_sgemm(transpose_a, transpose_b, rows, columns, depth, alpha, a, lda, b, ldb,
        beta, c, ldc, workspace, workspace_size, stream));
}
template <>
size_t multiplication<double, linalg_backend::B200>::workspace_size(
    linalg_int rows, linalg_int columns, linalg_int depth)
{
    return b200la_dgemm_workspace_size(rows, columns, depth);
}
template <>
size_t multiplication<float, linalg_backend::B200>::workspace_size(
    linalg_int rows, linalg_int columns, linalg_int depth)
{
    return b200la_sgemm_workspace_size(rows, columns, depth);
}

// ---- transpose --------------------------------------------------------------
namespace
{
// rows / columns above INT64_MAX cannot describe a device matrix; they reach
// the C ABI as negative values, which it rejects like zero
int64_t extent(linalg_long v) { return static_cast<int64_t>(v); }
}  // namespace
template <>
void transpose<double, linalg_backend::B200>::apply(linalg_long rows, linalg_long columns, double* m,
    void* workspace, size_t workspace_size, void* stream)
{
    check_status(b200la_dtranspose(extent(rows), extent(columns), m, workspace, workspace_size, stream));
}
template <>
void transpose<float, linalg_backend::B200>::apply(linalg_long rows, linalg_long columns, float* m,
    void* workspace, size_t workspace_size, void* stream)
{
    check_status(b200la_stranspose(extent(rows), extent(columns), m, workspace, workspace_size, stream));
}
template <> size_t transpose<double, linalg_backend::B200>::workspace_size(linalg_long rows, linalg_long columns)
{
    return b200la_dtranspose_workspace_size(extent(rows), extent(columns));
}
template <> size_t transpose<float, linalg_backend::B200>::workspace_size(linalg_long rows, linalg_long columns)
{
    return b200la_stranspose_workspace_size(extent(rows), extent(columns));
}

// ---- inversion --------------------------------------------------------------
template <>
void inversion<double, linalg_backend::B200>::apply(double* m, linalg_int* pivot, linalg_int lda,
    linear_solver_type type, void* workspace, size_t workspace_size, void* stream)
{
    check_status(b200la_dinverse(m, pv(pivot), lda, static_cast<int>(type), workspace,
        workspace_size, stream));
}
template <>
void inversion<float, linalg_backend::B200>::apply(float* m, linalg_int* pivot, linalg_int lda,
    linear_solver_type type, void* workspace, size_t workspace_size, void* stream)
{
    check_status(b200la_sinverse(m, pv(pivot), lda, static_cast<int>(type), workspace,
        workspace_size, stream));
}
template <>
size_t inversion<double, linalg_backend::B200>::workspace_size(linalg_int lda, linear_solver_type type)
{
    return b200la_dinverse_workspace_size(lda, static_cast<int>(type));
}
template <>
size_t inversion<float, linalg_backend::B200>::workspace_size(linalg_int lda, linear_solver_type type)
{
    return b200la_sinverse_workspace_size(lda, static_cast<int>(type));
}

// ---- determinant ------------------------------------------------------------
// det(A) = sign * product; an exactly singular factorization gives +0.
template <>
double determinant<double, linalg_backend::B200>::apply(double* m, linalg_int* pivot,
    linalg_int lda, linear_solver_type type, void* workspace, size_t workspace_size, void* stream)
{
    double product = 0.0;
    int    sign    = 1;
    check_status(b200la_ddeterminant(m, pv(pivot), lda, static_cast<int>(type), &product, &sign,
        nullptr, workspace, workspace_size, stream));
    if (type == linear_solver_type::CHOLESKY_LINEAR_SOLVER ||
        type == linear_solver_type::CHOLESKY_UPFRONT_LINEAR_SOLVER)
    {
        return product * product;  // det(A) = (prod l_ii)^2, as CUDA_BLAS returns it
    }
    return product == 0.0 ? 0.0 : (sign < 0 ? -product : product);
}
template <>
float determinant<float, linalg_backend::B200>::apply(float* m, linalg_int* pivot, linalg_int lda,
    linear_solver_type type, void* workspace, size_t workspace_size, void* stream)
{
    float product = 0.0f;
    int   sign    = 1;
    check_status(b200la_sdeterminant(m, pv(pivot), lda, static_cast<int>(type), &product, &sign,
        nullptr, workspace, workspace_size, stream));
    if (type == linear_solver_type::CHOLESKY_LINEAR_SOLVER ||
        type == linear_solver_type::CHOLESKY_UPFRONT_LINEAR_SOLVER)
    {
        return product * product;  // det(A) = (prod l_ii)^2, as CUDA_BLAS returns it
    }
    return product == 0.0f ? 0.0f : (sign < 0 ? -product : product);
}
template <>
size_t determinant<double, linalg_backend::B200>::workspace_size(linalg_int lda, linear_solver_type type)
{
    return b200la_ddeterminant_workspace_size(lda, static_cast<int>(type));
}
template <>
size_t determinant<float, linalg_backend::B200>::workspace_size(linalg_int lda, linear_solver_type type)
{
    return b200la_sdeterminant_workspace_size(lda, static_cast<int>(type));
}

// ---- batched multiplication ---------------------------------------------------
#if !defined(LINALG_HAS_CUBLAS) || !LINALG_HAS_CUBLAS
void batched_matrix_multiplication(linalg_int dim, linalg_int count, const float* a, const float* b, float* c,
    void* stream)
{
    check_status(b200la_sgemm_batched(dim, count, a, b, c, stream));
}
void batched_matrix_multiplication(linalg_int dim, linalg_int count, const double* a, const double* b, double* c,
    void* stream)
{
    check_status(b200la_dgemm_batched(dim, count, a, b, c, stream));
}
#endif
}  // namespace linalg
