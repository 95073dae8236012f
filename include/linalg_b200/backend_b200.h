/*
 * linalg_backend::B200 specializations of the reference's LU-solve operators
 * (see reference_api.h for the interface they implement).  Each is a thin
 * C++ shim over the C ABI in b200la.h: device pointers only, row-major,
 * 1-based int64 LAPACK pivots, caller-owned device workspace.  Errors throw
 * like the reference's LINALG_CHECK: std::invalid_argument for invalid
 * arguments (null pointers, bad sizes or strides, aliasing, short workspace),
 * std::runtime_error for CUDA or device-side failures.
 *
 * Semantics follow the reference's NATIVE backend (not CUDA_BLAS):
 *  - lu_decomposition synchronizes `stream` and writes the host `info`;
 *  - linear_solver honours the caller's pivots in LU_UPFRONT mode and, in
 *    LU mode, leaves x unchanged when U is exactly singular;
 *  - cholesky_decomposition (lower and upper) and the Cholesky modes of
 *    linear_solver are provided (factors bit-identical to NATIVE);
 *    cholesky_decomposition::apply synchronizes its stream and writes info
 *    to host memory before it returns (the host backends' contract), and
 *    returns false when the matrix is not positive definite; determinant's
 *    Cholesky modes return det(A) = (prod l_ii)^2 (CUDA_BLAS's value; NATIVE
 *    returns prod l_ii, which b200la_ddeterminant reports as `product`);
 *    the Cholesky modes of inversion and apply_aad are not provided
 *    (std::invalid_argument);
 *  - inversion and determinant honour LU_UPFRONT (m and pivot are the
 *    caller's factors) and, in LU mode, accept a null pivot (CUDA_BLAS's
 *    contract) by keeping the pivots in the workspace; inversion is
 *    asynchronous like CUDA_BLAS's, determinant synchronizes and returns;
 *  - determinant returns det(A) with the pivot sign applied, as CUDA_BLAS
 *    does; the NATIVE reduction omits that sign (include/matrix_operation/
 *    determinant.h), its magnitude is the same bits (b200la_ddeterminant
 *    returns both parts);
 *  - batched_matrix_multiplication (a free function in the reference, one
 *    definition per build) is defined by this library unless the build
 *    also compiles the CUDA_BLAS one (LINALG_HAS_CUBLAS), which it replaces.
 */
#pragma once

#include "reference_api.h"

namespace linalg
{
template <> bool cholesky_decomposition<double, linalg_backend::B200>::apply(double*, linalg_int,
    cholesky_decomposition_enum, void*, size_t, int*, void*);
template <> bool cholesky_decomposition<float, linalg_backend::B200>::apply(float*, linalg_int,
    cholesky_decomposition_enum, void*, size_t, int*, void*);
template <> bool cholesky_decomposition<double, linalg_backend::B200>::apply_aad(double*, const double*,
    linalg_int, cholesky_decomposition_enum, double*);
template <> bool cholesky_decomposition<float, linalg_backend::B200>::apply_aad(float*, const float*,
    linalg_int, cholesky_decomposition_enum, float*);
template <> size_t cholesky_decomposition<double, linalg_backend::B200>::workspace_size(linalg_int,
    cholesky_decomposition_enum);
template <> size_t cholesky_decomposition<float, linalg_backend::B200>::workspace_size(linalg_int,
    cholesky_decomposition_enum);

template <> bool lu_decomposition<double, linalg_backend::B200>::apply(double*, linalg_int,
    linalg_int*, void*, size_t, int*, void*);
template <> bool lu_decomposition<float, linalg_backend::B200>::apply(float*, linalg_int,
    linalg_int*, void*, size_t, int*, void*);
template <> size_t lu_decomposition<double, linalg_backend::B200>::workspace_size(linalg_int);
template <> size_t lu_decomposition<float, linalg_backend::B200>::workspace_size(linalg_int);

template <> void linear_solver<double, linalg_backend::B200>::apply(double*, linalg_int*,
    linalg_int, double*, linear_solver_type, void*, size_t, void*);
template <> void linear_solver<float, linalg_backend::B200>::apply(float*, linalg_int*, linalg_int,
    float*, linear_solver_type, void*, size_t, void*);
template <> size_t linear_solver<double, linalg_backend::B200>::workspace_size(linalg_int,
    linear_solver_type);
template <> size_t linear_solver<float, linalg_backend::B200>::workspace_size(linalg_int,
    linear_solver_type);

template <> void triangular_solver<double, linalg_backend::B200>::apply(bool, bool, bool,
    linalg_int, linalg_int, const double*, linalg_int, const double*, linalg_int, double*,
    linalg_int, void*, size_t, void*);
template <> void triangular_solver<float, linalg_backend::B200>::apply(bool, bool, bool, linalg_int,
    linalg_int, const float*, linalg_int, const float*, linalg_int, float*, linalg_int, void*,
    size_t, void*);
template <> size_t triangular_solver<double, linalg_backend::B200>::workspace_size(linalg_int,
    linalg_int);
template <> size_t triangular_solver<float, linalg_backend::B200>::workspace_size(linalg_int,
    linalg_int);

template <> void multiplication<double, linalg_backend::B200>::apply(bool, bool, linalg_int,
    linalg_int, linalg_int, double, const double*, linalg_int, const double*, linalg_int, double,
    double*, linalg_int, void*, size_t, void*);
template <> void multiplication<float, linalg_backend::B200>::apply(bool, bool, linalg_int,
    linalg_int, linalg_int, float, const float*, linalg_int, const float*, linalg_int, float,
    float*, linalg_int, void*, size_t, void*);
template <> size_t multiplication<double, linalg_backend::B200>::workspace_size(linalg_int,
    linalg_int, linalg_int);
template <> size_t multiplication<float, linalg_backend::B200>::workspace_size(linalg_int,
    linalg_int, linalg_int);

template <> void inversion<double, linalg_backend::B200>::apply(double*, linalg_int*, linalg_int,
    linear_solver_type, void*, size_t, void*);
template <> void inversion<float, linalg_backend::B200>::apply(float*, linalg_int*, linalg_int,
    linear_solver_type, void*, size_t, void*);
template <> size_t inversion<double, linalg_backend::B200>::workspace_size(linalg_int,
    linear_solver_type);
template <> size_t inversion<float, linalg_backend::B200>::workspace_size(linalg_int,
    linear_solver_type);

template <> double determinant<double, linalg_backend::B200>::apply(double*, linalg_int*,
    linalg_int, linear_solver_type, void*, size_t, void*);
template <> float determinant<float, linalg_backend::B200>::apply(float*, linalg_int*, linalg_int,
    linear_solver_type, void*, size_t, void*);
template <> size_t determinant<double, linalg_backend::B200>::workspace_size(linalg_int,
    linear_solver_type);
template <> size_t determinant<float, linalg_backend::B200>::workspace_size(linalg_int,
    linear_solver_type);

template <> void transpose<double, linalg_backend::B200>::apply(linalg_long, linalg_long, double*, void*,
    size_t, void*);
template <> void transpose<float, linalg_backend::B200>::apply(linalg_long, linalg_long, float*, void*,
    size_t, void*);
template <> size_t transpose<double, linalg_backend::B200>::workspace_size(linalg_long, linalg_long);
template <> size_t transpose<float, linalg_backend::B200>::workspace_size(linalg_long, linalg_long);
}  // namespace linalg
