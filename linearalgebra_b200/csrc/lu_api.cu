// Host drivers and extern "C" entry points for lu_decomposition,
// linear_solver (LU modes), the multi-RHS getrs extension,
// triangular_solver and multiplication.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <cstdlib>
#include <mutex>

#include "lu_driver.cuh"



using namespace b200la;

extern "C" {

B200LA_API size_t b200la_dgetrf_workspace_size(int64_t n) { return getrf_ws_size<double>(n); }
B200LA_API size_t b200la_sgetrf_workspace_size(int64_t n) { return getrf_ws_size<float>(n); }

B200LA_API int b200la_dgetrf(double* m, int64_t n, int64_t* pivot, void* ws, size_t bytes, int* info,
    void* stream)
{
    return getrf_sync<double>(m, n, pivot, ws, bytes, info, stream);
}
B200LA_API int b200la_sgetrf(float* m, int64_t n, int64_t* pivot, void* ws, size_t bytes, int* info,
    void* stream)
{
    return getrf_sync<float>(m, n, pivot, ws, bytes, info, stream);
}
B200LA_API int b200la_dgetrf_async(double* m, int64_t n, int64_t* pivot, void* ws, size_t bytes,
    void* stream)
{
    return getrf_async<double>(m, n, pivot, ws, bytes, stream);
}
B200LA_API int b200la_sgetrf_async(float* m, int64_t n, int64_t* pivot, void* ws, size_t bytes,
    void* stream)
{
    return getrf_async<float>(m, n, pivot, ws, bytes, stream);
}

B200LA_API int b200la_workspace_status(const void* ws, int* info, void* stream)
{
    if (ws == nullptr)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "workspace_status: null workspace");
    }
    return read_status(static_cast<const DeviceStatus*>(ws), info, as_stream(stream));
}

B200LA_API size_t b200la_dgesv_workspace_size(int64_t n, int mode) { return gesv_ws_size<double>(n, mode); }
B200LA_API size_t b200la_sgesv_workspace_size(int64_t n, int mode) { return gesv_ws_size<float>(n, mode); }
B200LA_API int b200la_dgesv(double* m, int64_t* pivot, int64_t n, double* x, int mode, void* ws,
    size_t bytes, void* stream)
{
    return gesv<double>(m, pivot, n, x, mode, ws, bytes, stream);
}
B200LA_API int b200la_sgesv(float* m, int64_t* pivot, int64_t n, float* x, int mode, void* ws,
    size_t bytes, void* stream)
{
    return gesv<float>(m, pivot, n, x, mode, ws, bytes, stream);
}

B200LA_API int b200la_dpotrf(double* m, int64_t n, int upper, void* ws, size_t bytes, int* info, void* stream)
{
    return potrf<double>(m, n, upper, ws, bytes, info, stream);
}
B200LA_API int b200la_spotrf(float* m, int64_t n, int upper, void* ws, size_t bytes, int* info, void* stream)
{
    return potrf<float>(m, n, upper, ws, bytes, info, stream);
}
B200LA_API int b200la_dgemm_batched(int64_t dim, int64_t count, const double* a, const double* b, double* c,
    void* stream)
{
    return gemm_batched<double>(dim, count, a, b, c, stream);
}
B200LA_API int b200la_sgemm_batched(int64_t dim, int64_t count, const float* a, const float* b, float* c,
    void* stream)
{
    return gemm_batched<float>(dim, count, a, b, c, stream);
}
B200LA_API size_t b200la_dgetrs_workspace_size(int64_t n, int64_t nrhs) { return getrs_ws_size<double>(n, nrhs); }
B200LA_API int b200la_dgetrs(const double* lu, const int64_t* pivot, int64_t n, int64_t nrhs, double* x,
    int64_t ldx, void* ws, size_t bytes, void* stream)
{
    return getrs<double>(lu, pivot, n, nrhs, x, ldx, ws, bytes, stream);
}

B200LA_API size_t b200la_dtrsm_workspace_size(int64_t, int64_t) { return 0; }
B200LA_API size_t b200la_strsm_workspace_size(int64_t, int64_t) { return 0; }
B200LA_API int b200la_dtrsm(int upper, int transpose, int unit, int64_t n, int64_t nrhs, const double* a,
    int64_t lda, const double* b, int64_t ldb, double* x, int64_t ldx, void* ws, size_t bytes,
    void* stream)
{
    return trsm<double>(upper, transpose, unit, n, nrhs, a, lda, b, ldb, x, ldx, ws, bytes, stream);
}
B200LA_API int b200la_strsm(int upper, int transpose, int unit, int64_t n, int64_t nrhs, const float* a,
    int64_t lda, const float* b, int64_t ldb, float* x, int64_t ldx, void* ws, size_t bytes,
    void* stream)
{
    return trsm<float>(upper, transpose, unit, n, nrhs, a, lda, b, ldb, x, ldx, ws, bytes, stream);
}

B200LA_API size_t b200la_dgemm_workspace_size(int64_t, int64_t, int64_t) { return 0; }
B200LA_API size_t b200la_sgemm_workspace_size(int64_t, int64_t, int64_t) { return 0; }
B200LA_API int b200la_dgemm(int ta, int tb, int64_t rows, int64_t cols, int64_t depth, double alpha,
    const double* a, int64_t lda, const double* b, int64_t ldb, double beta, double* c, int64_t ldc,
    void* ws, size_t bytes, void* stream)
{
    (void)ws;
    (void)bytes;
    return gemm<double>(ta, tb, rows, cols, depth, alpha, a, lda, b, ldb, beta, c, ldc, stream);
}
B200LA_API int b200la_sgemm(int ta, int tb, int64_t rows, int64_t cols, int64_t depth, float alpha,
    const float* a, int64_t lda, const float* b, int64_t ldb, float beta, float* c, int64_t ldc,
    void* ws, size_t bytes, void* stream)
{
    (void)ws;
    (void)bytes;
    return gemm<float>(ta, tb, rows, cols, depth, alpha, a, lda, b, ldb, beta, c, ldc, stream);
}
}

// ---------------------------------------------------------------------------
// Allocation-free linear solve (b200la_dgesv_noalloc).
//
// For callers that cannot allocate device memory themselves -- a host-language
// binding or plugin host that only hands over the device pointers of the
// matrix, pivots and right-hand side, or a service that forbids allocation
// once it is running -- the scratch of the LU solve lives in one fixed
// file-scope device array instead of a caller workspace.  Every GPU that
// loads this library holds that array (1 MiB) until the process exits.
// ---------------------------------------------------------------------------
namespace b200la
{
namespace
{
constexpr int64_t kNoAllocMaxOrder     = 16384;
constexpr size_t  kNoAllocScratchBytes = 1024 * 1024;
}  // namespace
}  // namespace b200la

static __device__ __align__(256) unsigned char g_noalloc_scratch[b200la::kNoAllocScratchBytes];

namespace b200la
{
namespace
{
std::mutex g_noalloc_mutex;
void*      g_noalloc_address[64] = {};

// Device address of g_noalloc_scratch on the current device.  The host-side
// name of the array is only a stand-in, so the address is looked up once per
// device (with that device current) and cached.
int noalloc_scratch(void** out)
{
    int dev = 0;
    B200LA_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64)
    {
        return set_error(B200LA_NOT_SUPPORTED, "dgesv_noalloc: device index %d out of range", dev);
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_address[dev] == nullptr)
    {
        void*             p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
        {
            return cuda_check(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
        }
        g_noalloc_address[dev] = p;
    }
    *out = g_noalloc_address[dev];
    return B200LA_SUCCESS;
}
}  // namespace
}  // namespace b200la

extern "C" B200LA_API int b200la_dgesv_noalloc(double* m, int64_t* pivot, int64_t n, double* x,
    int mode, void* stream)
{
    using namespace b200la;
    if (n > kNoAllocMaxOrder)
    {
        return set_error(B200LA_INVALID_ARGUMENT,
            "dgesv_noalloc: order %lld exceeds the fixed scratch limit of %lld; use b200la_dgesv "
            "with a caller-provided workspace",
            (long long)n, (long long)kNoAllocMaxOrder);
    }
    const size_t need = gesv_ws_size<double>(n, mode);
    if (need > kNoAllocScratchBytes)
    {
        return set_error(B200LA_NOT_SUPPORTED, "dgesv_noalloc: needs %zu bytes of scratch, has %zu",
            need, kNoAllocScratchBytes);
    }
    const bool chol = mode == B200LA_CHOLESKY_LINEAR_SOLVER || mode == B200LA_CHOLESKY_UPFRONT_LINEAR_SOLVER;
    if (m == nullptr || x == nullptr || (pivot == nullptr && !chol) || n <= 0 ||
        (mode != B200LA_LU_LINEAR_SOLVER && mode != B200LA_LU_UPFRONT_LINEAR_SOLVER && !chol))
    {
        // argument errors are reported by the shared checks, before any
        // device work
        return gesv<double>(m, pivot, n, x, mode, nullptr, 0, stream);
    }
    {
        const int st = prepare_device();
        if (st != B200LA_SUCCESS)
        {
            return st;
        }
    }
    void* scratch = nullptr;
    const int st  = noalloc_scratch(&scratch);
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    return gesv<double>(m, pivot, n, x, mode, scratch, kNoAllocScratchBytes, stream);
}
