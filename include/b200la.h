/*
 * b200la.h -- C ABI of the B200 (sm_100a) backend for LinearAlgebra's
 * LU-solve path.
 *
 * Every entry point takes plain pointers and sizes.  Matrix, pivot, right-hand
 * side and workspace pointers are DEVICE pointers (the reference's GPU
 * contract, docs/gpu_backend_design.md:22-36); `stream` is a cudaStream_t
 * passed as void* (NULL = the legacy default stream).  Matrices are row-major.
 * Pivots are int64, 1-based, LAPACK style: pivot[i] is the row swapped with row
 * i at step i, applied in increasing i (include/matrix_operation/
 * lu_decomposition.h:25-26).  The library never allocates: callers query
 * *_workspace_size() and pass that many bytes of device memory.
 *
 * Return value: a b200la_status.  Negative values are errors (the C++ shim in
 * include/linalg_b200/backend_b200.h turns them into exceptions, like the
 * reference's LINALG_CHECK); b200la_last_error() gives a message for the
 * calling thread's most recent error.
 */
#ifndef B200LA_H
#define B200LA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define B200LA_API __attribute__((visibility("default")))
#else
#define B200LA_API
#endif

typedef enum b200la_status
{
    B200LA_SUCCESS              = 0,
    B200LA_SINGULAR             = 1,  /* exact zero pivot: factors complete, U singular */
    B200LA_NOT_CONVERGED        = 2,  /* refinement did not reach the requested accuracy */
    B200LA_INVALID_ARGUMENT     = -1, /* null pointer, bad size/stride, aliasing */
    B200LA_WORKSPACE_TOO_SMALL  = -2,
    B200LA_CUDA_ERROR           = -3, /* a CUDA runtime call or launch failed */
    B200LA_DEVICE_TIMEOUT       = -4, /* a bounded device-side wait gave up */
    B200LA_NOT_SUPPORTED        = -5  /* no sm_100 device, or an unsupported size */
} b200la_status;

/* linear_solver modes, same values as the reference's linear_solver_type
 * (include/matrix_operation/linear_solver.h:15-21). */
#define B200LA_LU_LINEAR_SOLVER 1
#define B200LA_LU_UPFRONT_LINEAR_SOLVER 2
#define B200LA_CHOLESKY_LINEAR_SOLVER 3
#define B200LA_CHOLESKY_UPFRONT_LINEAR_SOLVER 4

B200LA_API const char* b200la_last_error(void);
B200LA_API const char* b200la_status_string(int status);
B200LA_API int         b200la_version(void);

/* Number of kernel launches the library has issued in this process. */
B200LA_API int64_t b200la_launch_count(void);

/* Launch recorder for measurement: while started, every launch of a kernel
 * class in `class_mask` (bit 0 panel, 1 row interchange + U12 solve,
 * 2 trailing update, 3 triangular solves, 4 general GEMM, 5 mixed-precision
 * factorization GEMM, 6 FP64 residual, 7 batched solver, 8 mixed-precision
 * operand preparation and outer U12 solve, 9 precision selector: network
 * and matrix statistics, 10 inversion GEMM updates, 11 inversion and
 * determinant helpers: identity, column gather, diagonal product,
 * 12 Cholesky trailing updates, 13 Cholesky diagonal blocks, panel solves,
 * zeroing and transposition, 14 transpose) is
 * bracketed by a
 * pair of CUDA events on its stream.  b200la_profile_stop synchronizes those
 * events and returns the summed device time (ms) and launch count of one
 * class; it also stops recording. */
B200LA_API void b200la_profile_start(int class_mask);
B200LA_API int  b200la_profile_stop(int kernel_class, double* total_ms, int64_t* launches);

/* ---- lu_decomposition ---------------------------------------------------
 * Replaces lu_decomposition<T, Backend>::apply / ::workspace_size
 * (include/matrix_operation/lu_decomposition.h:38-53; CUDA_BLAS sibling
 * src/matrix_operation/gpu/cublas/lu_decomposition_cublas.cpp:172-203).
 * m: n x n row-major, lda == n (the reference's lda is the order and the
 * stride).  pivot: n device int64.  info: HOST int, may be NULL; 0 or the
 * 1-based index of the first exactly-zero U diagonal entry.  Synchronizes
 * `stream` before returning (the reference's contract for this op).
 * Returns B200LA_SUCCESS, B200LA_SINGULAR or an error. */
B200LA_API size_t b200la_dgetrf_workspace_size(int64_t n);
B200LA_API size_t b200la_sgetrf_workspace_size(int64_t n);
B200LA_API int    b200la_dgetrf(double* m, int64_t n, int64_t* pivot, void* workspace,
       size_t workspace_bytes, int* info, void* stream);
B200LA_API int    b200la_sgetrf(float* m, int64_t n, int64_t* pivot, void* workspace,
       size_t workspace_bytes, int* info, void* stream);

/* Asynchronous factorization (no host synchronization): the status lands in
 * the workspace's device status block; read it with b200la_workspace_status.
 * Extension beyond the reference API (needed for graph capture and
 * pipelines). */
B200LA_API int b200la_dgetrf_async(double* m, int64_t n, int64_t* pivot, void* workspace,
    size_t workspace_bytes, void* stream);
B200LA_API int b200la_sgetrf_async(float* m, int64_t n, int64_t* pivot, void* workspace,
    size_t workspace_bytes, void* stream);

/* Copies the device status block at the start of `workspace` to the host
 * (synchronizing `stream`): *info = LAPACK info of the last factorization,
 * returns B200LA_SUCCESS / B200LA_SINGULAR / B200LA_DEVICE_TIMEOUT. */
B200LA_API int b200la_workspace_status(const void* workspace, int* info, void* stream);

/* Failure-detection check of the bounded device-side waits.  No counterpart
 * in the reference (its CPU path has no inter-thread waits; its numerical
 * status is lu_decomposition_native.cpp:147-157,424-428).  Runs the forward
 * triangular solve of b200la_dgesv's solve step on the factors `lu` (n x n,
 * n >= 128) with its first 64-row block never claimed, so every other block
 * waits, at most wait_ns (100 us .. 2 s), for a publication that never
 * comes, records DEV_WAIT_TIMEOUT in the workspace's status block and
 * returns.  x is left unchanged.  Synchronizes `stream`; returns
 * B200LA_DEVICE_TIMEOUT when the waits ran out.  Workspace: the size
 * b200la_dgesv_workspace_size(n, B200LA_LU_LINEAR_SOLVER) reports. */
/* Latency floor of the cluster panel's per-column pivot exchange, for the
 * panel's latency roofline.  No counterpart in the reference (its panel,
 * lu_decomposition_native.cpp:158-232, is sequential).  Runs only the
 * exchange of the cluster panel kernel (a key posted by every CTA, cluster
 * barrier, the keys and one pivot row read through distributed shared
 * memory by one warp, two block barriers) for `columns` columns of FP64
 * (elem_bytes 8) or FP32 (4) rows of a width-32 or -64 panel, and writes the
 * device-timed nanoseconds per column.  Synchronizes `stream`.
 * Workspace: 256 bytes. */
B200LA_API int b200la_panel_exchange_floor(int elem_bytes, int width, int columns, double* ns_per_column,
    void* workspace, size_t workspace_bytes, void* stream);

B200LA_API int b200la_test_wait_expiry(const double* lu, int64_t n, double* x, uint64_t wait_ns,
    void* workspace, size_t workspace_bytes, void* stream);

/* ---- cholesky_decomposition ------------------------------------------------
 * Replaces cholesky_decomposition<T, Backend>::apply / ::workspace_size
 * (include/matrix_operation/cholesky_decomposition.h; NATIVE
 * src/matrix_operation/cpu/native/cholesky_decomposition_native.cpp): m
 * (n x n row-major, symmetric positive definite; the lower triangle is read)
 * becomes L (upper == 0, zeros above) or U = L^T (upper != 0, zeros below),
 * bit-identical to the reference.  info: HOST int, may be NULL; 0 or the
 * 1-based index of the first non-positive pivot (the matrix is then left as
 * the reference leaves it).  Workspace: b200la_dgetrf_workspace_size(n).
 * Synchronizes `stream`.  Returns B200LA_SUCCESS, B200LA_SINGULAR (not
 * positive definite) or an error. */
B200LA_API int b200la_dpotrf(double* m, int64_t n, int upper, void* workspace, size_t workspace_bytes,
    int* info, void* stream);
B200LA_API int b200la_spotrf(float* m, int64_t n, int upper, void* workspace, size_t workspace_bytes,
    int* info, void* stream);

/* ---- linear_solver ---------------------------------------------------------
 * Replaces linear_solver<T, Backend>::apply / ::workspace_size
 * (include/matrix_operation/linear_solver.h:46-64; NATIVE semantics of
 * src/matrix_operation/cpu/native/linear_solver_native.cpp:149-191).
 * mode B200LA_LU_LINEAR_SOLVER factors m in place (pivot written) and then
 * solves, unless the factorization found an exact zero pivot, in which case x
 * is left unchanged; B200LA_LU_UPFRONT_LINEAR_SOLVER reuses m and pivot as
 * given.  B200LA_CHOLESKY_LINEAR_SOLVER factors m in place (lower, as
 * b200la_dpotrf) and solves unless it is not positive definite;
 * B200LA_CHOLESKY_UPFRONT_LINEAR_SOLVER solves with the lower factor in m
 * (pivot unused).  x: n device values, overwritten with the solution.
 * Asynchronous on `stream`. */
B200LA_API size_t b200la_dgesv_workspace_size(int64_t n, int mode);
B200LA_API size_t b200la_sgesv_workspace_size(int64_t n, int mode);
B200LA_API int    b200la_dgesv(double* m, int64_t* pivot, int64_t n, double* x, int mode,
       void* workspace, size_t workspace_bytes, void* stream);
B200LA_API int    b200la_sgesv(float* m, int64_t* pivot, int64_t n, float* x, int mode,
       void* workspace, size_t workspace_bytes, void* stream);

/* Multi-right-hand-side solve with existing factors and pivots: x is
 * n x nrhs row-major with row stride ldx >= nrhs.  Extension (the reference
 * linear_solver is single-RHS). */
B200LA_API size_t b200la_dgetrs_workspace_size(int64_t n, int64_t nrhs);
B200LA_API int    b200la_dgetrs(const double* lu, const int64_t* pivot, int64_t n, int64_t nrhs,
       double* x, int64_t ldx, void* workspace, size_t workspace_bytes, void* stream);

/* Allocation-free variant of b200la_dgesv, for callers that cannot allocate
 * device memory (for example a host-language binding or a plugin host that is
 * handed only the matrix, pivot and right-hand-side pointers, or a service
 * that forbids allocation after start-up).  No counterpart in the reference.
 * Same arguments and semantics as b200la_dgesv minus the workspace (all four
 * modes; pivot may be NULL in the Cholesky modes): the scratch is one fixed
 * 1 MiB device array inside this library, which every GPU that loads the
 * library holds until the process exits.  Limit: n <= 16384 (larger orders
 * return B200LA_INVALID_ARGUMENT).  It allocates no device memory; it does
 * use other driver resources:
 *   - the first call in a CUDA context looks up the array's device address
 *     (cudaGetSymbolAddress, with the device current) and caches it under
 *     that context's id;
 *   - the first LU-mode call with n > 128 on a device creates the library's
 *     process-wide side stream for the factorization's look-ahead;
 *   - every LU-mode call with n > 128 creates and destroys two CUDA events.
 * Make the first call on each device (with n > 128) before any stream
 * capture.  Every call shares the one array, so calls whose GPU work overlaps
 * (other streams, other host threads) race and must be serialized by the
 * caller. */
B200LA_API int b200la_dgesv_noalloc(double* m, int64_t* pivot, int64_t n, double* x, int mode,
    void* stream);

/* ---- triangular_solver ----------------------------------------------------
 * Replaces triangular_solver<T, Backend>::apply / ::workspace_size
 * (include/matrix_operation/triangular_solver.h:22-37; argument checks of
 * src/common/triangular_solver_checks.h:11-35).  Solves op(A) X = B; A n x n
 * (row stride lda >= n), B and X n x nrhs (ldb, ldx >= nrhs).  Only the
 * selected triangle is read; the diagonal is not read when unit != 0.  A and
 * B are preserved; A, B, X must be distinct buffers.  Asynchronous. */
B200LA_API size_t b200la_dtrsm_workspace_size(int64_t n, int64_t nrhs);
B200LA_API size_t b200la_strsm_workspace_size(int64_t n, int64_t nrhs);
B200LA_API int    b200la_dtrsm(int upper, int transpose, int unit, int64_t n, int64_t nrhs,
       const double* a, int64_t lda, const double* b, int64_t ldb, double* x, int64_t ldx,
       void* workspace, size_t workspace_bytes, void* stream);
B200LA_API int    b200la_strsm(int upper, int transpose, int unit, int64_t n, int64_t nrhs,
       const float* a, int64_t lda, const float* b, int64_t ldb, float* x, int64_t ldx,
       void* workspace, size_t workspace_bytes, void* stream);

/* ---- inversion (LU and Cholesky modes) ----------------------------------------
 * Replaces inversion<T, Backend>::apply / ::workspace_size
 * (include/matrix_operation/inversion.h:15-53; NATIVE semantics of
 * src/matrix_operation/cpu/native/inversion_native.cpp:412-452).  m: n x n
 * row-major (lda == n), overwritten with the inverse.  Mode
 * B200LA_LU_LINEAR_SOLVER factors m first (pivots written to `pivot`, or kept
 * in the workspace when pivot is NULL, as the CUDA_BLAS backend allows) and
 * leaves the factors in m when the factorization met an exact zero pivot;
 * B200LA_LU_UPFRONT_LINEAR_SOLVER inverts the factors and pivots given in m
 * and pivot.  B200LA_CHOLESKY_LINEAR_SOLVER factors m (lower Cholesky) and
 * leaves the partial factor in m at a non-positive pivot;
 * B200LA_CHOLESKY_UPFRONT_LINEAR_SOLVER inverts the lower factor given in m
 * (its upper triangle is not read); both return an exactly symmetric
 * inverse and ignore `pivot`.  Asynchronous on `stream`; the
 * factorization's status (info = the 1-based row of the first zero or
 * non-positive pivot) lands in the workspace (b200la_workspace_status).
 * Workspace: one n x n scratch plus O(n), the same in every mode; the
 * inverse agrees with the reference's to rounding, not bit for bit (its
 * entries come from GEMM-blocked substitutions). */
B200LA_API size_t b200la_dinverse_workspace_size(int64_t n, int mode);
B200LA_API size_t b200la_sinverse_workspace_size(int64_t n, int mode);
B200LA_API int    b200la_dinverse(double* m, int64_t* pivot, int64_t n, int mode, void* workspace,
       size_t workspace_bytes, void* stream);
B200LA_API int    b200la_sinverse(float* m, int64_t* pivot, int64_t n, int mode, void* workspace,
       size_t workspace_bytes, void* stream);

/* ---- determinant (LU and Cholesky modes) -------------------------------------
 * Replaces determinant<T, Backend>::apply / ::workspace_size
 * (include/matrix_operation/determinant.h; src/matrix_operation/cpu/
 * determinant.cpp:18-27,56-80).  Mode B200LA_LU_LINEAR_SOLVER factors m in
 * place (pivot as for inversion, NULL allowed); LU_UPFRONT reads the given
 * factors and pivots.  Outputs (host): *product = the product of U's
 * diagonal in index order, one multiply at a time in the input type (the
 * reference's NATIVE value, bit for bit; 0 when LU mode met an exact zero
 * pivot, then the return is B200LA_SINGULAR); *sign = (-1)^(number of i with
 * pivot[i] != i+1), may be NULL, so that det(A) = sign * product (the
 * reference's NATIVE reduction omits this sign, its CUDA_BLAS one applies
 * it); *log_abs = sum of log|u_ii|, may be NULL, finite where the product
 * over- or underflows.  Cholesky modes (determinant.cpp:28-37,80-90):
 * B200LA_CHOLESKY_LINEAR_SOLVER factors m (lower, bit-identical to NATIVE)
 * and B200LA_CHOLESKY_UPFRONT_LINEAR_SOLVER reads the given lower factor;
 * *product = the product of the factor's diagonal in index order (NATIVE's
 * value, which is sqrt(det A); 0 and B200LA_SINGULAR when m is not positive
 * definite), *sign = 1, *log_abs = log det(A) = 2 sum log l_ii; pivot is
 * unused.  Synchronous (the reference returns the value). */
B200LA_API size_t b200la_ddeterminant_workspace_size(int64_t n, int mode);
B200LA_API size_t b200la_sdeterminant_workspace_size(int64_t n, int mode);
B200LA_API int    b200la_ddeterminant(double* m, int64_t* pivot, int64_t n, int mode, double* product,
       int* sign, double* log_abs, void* workspace, size_t workspace_bytes, void* stream);
B200LA_API int    b200la_sdeterminant(float* m, int64_t* pivot, int64_t n, int mode, float* product,
       int* sign, double* log_abs, void* workspace, size_t workspace_bytes, void* stream);

/* ---- multiplication --------------------------------------------------------
 * Replaces multiplication<T, Backend>::apply (16-argument form) /
 * ::workspace_size (include/matrix_operation/multiplication.h:47-62,107-114):
 * c = alpha op(a) op(b) + beta c, row-major, BLAS contract (beta == 0: c is
 * write-only; alpha == 0: a and b are not read).  FP64 with op(b) = b runs
 * on the FP64 tensor cores and gives the reference NATIVE loop's bits
 * (beta c, then fma(alpha a_ik, b_kj, c) in k order).  Asynchronous. */
B200LA_API size_t b200la_dgemm_workspace_size(int64_t rows, int64_t cols, int64_t depth);
B200LA_API size_t b200la_sgemm_workspace_size(int64_t rows, int64_t cols, int64_t depth);
B200LA_API int    b200la_dgemm(int transpose_a, int transpose_b, int64_t rows, int64_t cols,
       int64_t depth, double alpha, const double* a, int64_t lda, const double* b, int64_t ldb,
       double beta, double* c, int64_t ldc, void* workspace, size_t workspace_bytes,
       void* stream);
B200LA_API int    b200la_sgemm(int transpose_a, int transpose_b, int64_t rows, int64_t cols,
       int64_t depth, float alpha, const float* a, int64_t lda, const float* b, int64_t ldb,
       float beta, float* c, int64_t ldc, void* workspace, size_t workspace_bytes, void* stream);

/* ---- batched multiplication ------------------------------------------------
 * Replaces batched_matrix_multiplication (include/matrix_operation/
 * multiplication_batched.h; CUDA_BLAS kernel src/matrix_operation/gpu/cublas/
 * multiplication_batched_cublas.cu:15-40): c_i = a_i b_i for i < count,
 * each a dim x dim row-major matrix, packed back to back (element offset
 * i*dim*dim).  Each entry is the sum of the products from zero in k order
 * with fused multiply-adds, like the reference's kernel (FP64 on the FP64
 * tensor cores, FP32 on the SIMT FMA pipe).  Asynchronous. */
B200LA_API int b200la_dgemm_batched(int64_t dim, int64_t count, const double* a, const double* b, double* c,
    void* stream);
B200LA_API int b200la_sgemm_batched(int64_t dim, int64_t count, const float* a, const float* b, float* c,
    void* stream);

/* ---- transpose and row-major <-> column-major interop -----------------------
 * Replaces transpose<T, Backend>::apply / ::workspace_size
 * (include/matrix_operation/transpose.h; CUDA_BLAS src/matrix_operation/gpu/
 * cublas/transpose_cublas.cpp:25-57, NATIVE src/matrix_operation/cpu/native/
 * transpose_native.cpp): the row-major rows x columns matrix m becomes its
 * row-major columns x rows transpose, in place.  A square matrix needs no
 * workspace (workspace_size returns 0); otherwise the workspace holds
 * rows*columns elements.  rows and columns must be positive.  Asynchronous.
 * b200la_?transpose_out writes the transpose of src into dst (no overlap),
 * which is also the column-major copy of a row-major matrix and back:
 * the interop between this backend's row-major buffers and column-major
 * BLAS buffers.  Extension, no reference counterpart. */
B200LA_API size_t b200la_dtranspose_workspace_size(int64_t rows, int64_t columns);
B200LA_API size_t b200la_stranspose_workspace_size(int64_t rows, int64_t columns);
B200LA_API int b200la_dtranspose(int64_t rows, int64_t columns, double* m, void* workspace, size_t workspace_bytes,
    void* stream);
B200LA_API int b200la_stranspose(int64_t rows, int64_t columns, float* m, void* workspace, size_t workspace_bytes,
    void* stream);
B200LA_API int b200la_dtranspose_out(int64_t rows, int64_t columns, const double* src, double* dst, void* stream);
B200LA_API int b200la_stranspose_out(int64_t rows, int64_t columns, const float* src, float* dst, void* stream);

/* ---- mixed-precision LU solve with FP64 iterative refinement --------------
 * Solves A X = B (A n x n FP64, row stride n, left unchanged; B, X n x nrhs,
 * row strides ldb, ldx >= nrhs, nrhs <= 64) to a normwise backward error
 * max_j ||b_j - A x_j|| / (||A|| ||x_j|| + ||b_j||) (inf norms) <= tolerance:
 * LU with partial pivoting of an FP32 copy of A whose trailing updates run on
 * the tcgen05 tensor cores in the chosen precision with FP32 accumulation,
 * then FP64 refinement (residual, update and test in FP64), switching to
 * GMRES-IR preconditioned by the low-precision factors when plain
 * refinement stalls, and escalating to the next precision (FP8 -> BF16;
 * BF16, FP16, TF32 -> FP32; FP32 -> plain FP64 LU) when that fails too.  Synchronous (reads the residual norms).
 * Extension: the reference has no mixed-precision solver. */
#define B200LA_PREC_FP64 0 /* plain FP64 LU (the reference's algorithm) + refinement */
#define B200LA_PREC_FP32 1 /* FP32 factors, three-term TF32 tensor-core updates */
#define B200LA_PREC_TF32 2 /* FP32 factors, TF32 tensor-core updates */
#define B200LA_PREC_BF16 3 /* FP32 factors, BF16 tensor-core updates */
#define B200LA_PREC_FP16 4 /* FP32 factors, FP16 tensor-core updates */
#define B200LA_PREC_FP8  5 /* FP32 factors, FP8-E4M3 tensor-core updates with
                              power-of-two scales per row of L21 / column of U12;
                              escalates to BF16 */

typedef struct b200la_refine_options
{
    int    precision;      /* B200LA_PREC_* of the factorization */
    int    max_iterations; /* refinement iterations (default 50) */
    double tolerance;      /* target normwise backward error (default 1e-14) */
    int    gmres_restart;  /* GMRES-IR restart length, 0 disables (nrhs == 1 only) */
    int    escalate;       /* on failure, retry at the next precision up to FP64 */
} b200la_refine_options;

typedef struct b200la_refine_result
{
    int    precision_used;   /* B200LA_PREC_* of the factorization that finished */
    int    info;             /* LAPACK info of that factorization */
    int    converged;        /* backward error <= tolerance */
    int    iterations;       /* refinement corrections applied */
    int    gmres_iterations; /* inner GMRES iterations */
    int    escalations;      /* precision escalations */
    double backward_error;   /* final max_j eta_j */
    double factor_ms;        /* device time of the factorization(s) */
    double refine_ms;        /* device time of the solves and refinement */
} b200la_refine_result;

B200LA_API void   b200la_refine_default_options(b200la_refine_options* options);
B200LA_API size_t b200la_dsolve_mixed_workspace_size(int64_t n, int64_t nrhs,
       const b200la_refine_options* options);
B200LA_API int    b200la_dsolve_mixed(const double* a, int64_t n, int64_t nrhs, const double* b,
       int64_t ldb, double* x, int64_t ldx, const b200la_refine_options* options,
       b200la_refine_result* result, void* workspace, size_t workspace_bytes, void* stream);

/* Mixed-precision Cholesky-IR for a symmetric positive definite A (both
 * triangles given; the factorization reads the lower one): the Cholesky
 * factor of an FP32 copy of A (the blocked Cholesky of the CHOLESKY modes, in
 * FP32), used in LU form (L D^-1 and D L^T, D = diag(l_ii), identity
 * permutation) by the same FP64 refinement, GMRES-IR and escalation as
 * b200la_dsolve_mixed.  A non-positive pivot in FP32 ends that attempt
 * (info = its row) and escalates to the plain FP64 LU.  options->precision is
 * B200LA_PREC_FP32 or B200LA_PREC_FP64; same arguments, workspace
 * (b200la_dsolve_mixed_workspace_size), result and return codes as
 * b200la_dsolve_mixed.  Synchronous.  Extension: the reference's Cholesky
 * solve (linear_solver_native.cpp:177-189) has no mixed-precision form. */
B200LA_API int    b200la_dsolve_mixed_spd(const double* a, int64_t n, int64_t nrhs, const double* b,
       int64_t ldb, double* x, int64_t ldx, const b200la_refine_options* options,
       b200la_refine_result* result, void* workspace, size_t workspace_bytes, void* stream);

/* ---- learned precision selector --------------------------------------------
 * Extension: the reference has no precision selection.
 *
 * Network: 12 -> 64 -> 64 -> 4 MLP, ReLU, softmax over the classes
 * {FP8, BF16, FP32, FP64}, FP32.  params: b200la_mlp_param_count() = 5252
 * floats, W1[12][64] b1[64] W2[64][64] b2[64] W3[64][4] b3[4] (row-major,
 * y = x W + b), device memory.  x: batch x 12 standardized features.
 *   mlp_forward:  probs[batch][4] = softmax(net(x)).
 *   mlp_gradient: grads[5252] += d/dparams of the summed cross-entropy
 *                 against labels[batch] (0..3); *loss_sum += summed loss
 *                 (device float).  Forward and backward in one kernel.
 *   mlp_adam:     one Adam step on grads / batch (+ weight_decay * params),
 *                 step counted from 1; clears grads.
 * All asynchronous on `stream`. */
B200LA_API int b200la_mlp_param_count(void);
B200LA_API int b200la_mlp_forward(const float* params, const float* x, int64_t batch, float* probs,
       void* stream);
B200LA_API int b200la_mlp_gradient(const float* params, const float* x, const int32_t* labels,
       int64_t batch, float* grads, float* loss_sum, void* stream);
B200LA_API int b200la_mlp_adam(float* params, float* grads, float* m1, float* m2, int64_t batch,
       float lr, float beta1, float beta2, float eps, int step, float weight_decay, void* stream);

/* Matrix statistics behind the features: sixteen 64-bit words at `out`
 * (device), reset and gathered from A (n x n FP64, row-major, lda = n):
 * [0] ||A||_inf, [1] max|a_ij|, [2] sum a_ij^2, [3] max_i 1/(1+r_i) with
 * r_i = |a_ii| / sum_{j!=i}|a_ij|, [4] number of rows with r_i >= 1
 * (integer), [5] ||A||_1, [6] min row sum of |a|, [7] min|a_ii|,
 * [8] max|a_ii|, [9] sum|a_ij|, [10] min column sum, [11] sum|a_ii| (doubles
 * as bit patterns).  Asynchronous. */
B200LA_API int b200la_matrix_stats(const double* a, int64_t n, unsigned long long* out, void* stream);

/* The 12 selector features of A (host floats), all from the O(n^2)
 * statistics above: log2(n)/12; log10 of ||A||_inf/max|a|, ||A||_1/max|a|,
 * ||A||_F/(n max|a|), mean|a|/max|a|; log10(min_i r_i)/4; the fraction of
 * diagonally dominant rows; log10(min|a_ii|/max|a|)/4;
 * log10(max|a_ii|/max|a|); log10(min row sum/||A||_inf)/4;
 * log10(min column sum/||A||_1)/4; log10(mean|a_ii|/max|a|).  Workspace:
 * 128 bytes of device memory, 8-byte aligned.  Synchronous. */
B200LA_API int b200la_selector_features(const double* a, int64_t n, float* features, void* workspace,
       size_t workspace_bytes, void* stream);

/* 1-norm condition estimate kappa1 = ||A||_1 est(||A^-1||_1) from one FP32
 * LU of A (three-term TF32 updates): Hager's estimator (SIAM J. Sci. Stat.
 * Comput. 5, 1984) with Higham's stopping rules and alternating test vector
 * (ACM TOMS 14, 1988), the solves with A and A^T applied in FP64 with the
 * FP32 factors.  A lower bound of kappa1, usually within a small factor
 * while kappa1 * 2^-24 < 1.  Workspace: b200la_dsolve_mixed_workspace_size(n,
 * 1, NULL).  Returns B200LA_SINGULAR (kappa1 = inf) for an exactly singular
 * FP32 factor.  Synchronous.  Extension: no reference counterpart. */
B200LA_API int b200la_dcondition_estimate(const double* a, int64_t n, double* kappa1, int* info,
       void* workspace, size_t workspace_bytes, void* stream);

/* Solve A x = b (one right-hand side) with the precision the network picks
 * from the features above: `params` (device) holds the 5252 weights followed
 * by 24 floats, the features' mean[12] and inverse standard deviation[12].
 * The predicted precision is tried first (FP64: plain FP64 LU and
 * refinement); refinement failure escalates up to FP64 as in
 * b200la_dsolve_mixed, so the accuracy never depends on the prediction.
 * options->precision and ->escalate are ignored.  *predicted: B200LA_PREC_*
 * of the network's class; features: the 12 features (host, may be NULL).
 * Workspace as b200la_dsolve_mixed with nrhs = 1.  Synchronous. */
B200LA_API int b200la_dsolve_selected(const double* a, int64_t n, const double* b, double* x,
       const float* params, const b200la_refine_options* options, b200la_refine_result* result,
       int* predicted, float* features, void* workspace, size_t workspace_bytes, void* stream);

/* ---- batched solver for many small systems of uneven order ----------------
 * Solves `count` independent systems A_i x_i = b_i, 1 <= n_i <= 512, in ONE
 * persistent kernel launch (one CTA per system at a time, taken from an
 * atomic queue in the order given by `order`, NULL = index order; pass the
 * largest systems first).  Device arrays: sizes[count] (n_i), offsets_a
 * [count] (element offset of the row-major n_i x n_i matrix in a),
 * offsets_v[count] (element offset of b_i / x_i), status[count] (refinement
 * corrections used; 1000 + corrections for a system finished with FP64
 * factors after its FP32 refinement stalled; -(info) for an exactly singular
 * U; -1000000 if not converged), backward_error[count].  total_a / total_v: element sizes of a and b.  precision
 * B200LA_PREC_FP32 (FP32 factors, FP64 refinement to `tolerance`; systems
 * whose refinement stalls are refactored in FP64 by a second persistent
 * launch that skips all others) or B200LA_PREC_FP64 (FP64 LU + refinement).
 * nb_table[8]: per order bucket of 64 (the autotuner's choice), bits 0-7 the
 * panel width (16 or 32 for FP32 factors, 8 or 16 for FP64; another width
 * falls back to the largest) and bits 8-15 the threads that solve one
 * system / 32 (2 or 4; 0 = a whole CTA of 256): a CTA solves 256 / that many
 * systems at once.  b200la_batched_table_valid says whether every width is
 * one of those and every bucket's largest order fits its group's shared
 * memory and factor scratch.  The workspace holds one 2 MiB factor scratch
 * slot per CTA, min(total_v, 192) slots (a batch has at most total_v
 * systems); the systems are factored there, A is only read.
 * Asynchronous.  Extension: the reference has no batched solver. */
B200LA_API size_t b200la_dgesv_batched_workspace_size(int64_t total_a, int64_t total_v, int precision);
/* 1 if the host array table[8] is a valid nb_table for `precision`, else 0. */
B200LA_API int    b200la_batched_table_valid(int precision, const int32_t* table);
B200LA_API int    b200la_dgesv_batched(int64_t count, const int32_t* sizes, const int64_t* offsets_a,
       const int64_t* offsets_v, const int32_t* order, const double* a, const double* b, double* x,
       int64_t total_a, int64_t total_v, int precision, const int32_t* nb_table, int max_iterations,
       double tolerance, int32_t* status, double* backward_error, void* workspace,
       size_t workspace_bytes, void* stream);

/* ---- tensor-core update (mixed-precision LU building block) ---------------
 * c[m x n] (fp32, row stride ldc) -= a[m x k] * b[n x k]^T on the tcgen05
 * tensor cores with FP32 accumulation.  a and b are K-major (row stride k
 * elements), 16-byte aligned, k a multiple of 32 (TF32) or 64 (BF16/FP16).
 * kind: 0 = TF32 (fp32 containers), 1 = BF16, 2 = FP16.  split3 (TF32 only):
 * a = a + a_small, b = b + b_small split operands, product
 * a*b + a*b_small + a_small*b.  workspace: b200la_tc_update_workspace_size()
 * bytes of device memory (status block).  The trailing update of
 * lu_decomposition_native.cpp:400-422 done in low precision; no direct
 * reference counterpart. */
B200LA_API size_t b200la_tc_update_workspace_size(void);
B200LA_API int    b200la_sgemm_tc_update(int kind, int split3, float* c, int64_t ldc, int64_t m, int64_t n,
       int64_t k, const void* a, const void* b, const void* a_small, const void* b_small,
       void* workspace, size_t workspace_bytes, void* stream);
/* FP8-E4M3 form: c[i][j] -= a_inv_scale[i] * b_inv_scale[j] * sum_k a[i][k] b[j][k]
 * (tcgen05 kind::f8f6f4, FP32 accumulation); a, b are E4M3 bytes, K-major,
 * k a multiple of 128. */
B200LA_API int    b200la_sgemm_tc_update_fp8(float* c, int64_t ldc, int64_t m, int64_t n, int64_t k,
       const void* a, const void* b, const float* a_inv_scale, const float* b_inv_scale,
       void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* B200LA_H */
