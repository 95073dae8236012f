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

// Failure-detection check of the bounded device waits: the forward
// triangular solve of b200la_dgesv's solve step with block 0 never claimed
// (its ticket is started at 1), so every other block waits for a block that
// nothing publishes until wait_ns runs out.  The factors are not read past
// the first wait.  Returns what the workspace's status block reports
// (B200LA_DEVICE_TIMEOUT when the waits ran out).
B200LA_API int b200la_test_wait_expiry(const double* lu, int64_t n, double* x, uint64_t wait_ns, void* ws,
    size_t bytes, void* stream)
{
    if (lu == nullptr || x == nullptr || n < 2 * kTvRows || n > INT_MAX)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "test_wait_expiry: needs factors, x and n >= %d", 2 * kTvRows);
    }
    if (wait_ns < 100000ull || wait_ns > kWaitLimitNs)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "test_wait_expiry: wait limit outside [100 us, 2 s]");
    }
    const size_t need = gesv_ws_size<double>(n, B200LA_LU_LINEAR_SOLVER);
    if (ws == nullptr || bytes < need)
    {
        return set_error(B200LA_WORKSPACE_TOO_SMALL, "test_wait_expiry: workspace too small (%zu < %zu)", bytes,
            need);
    }
    int st = prepare<double>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    Arena             a(ws, bytes);
    GetrfPlan<double> gp = plan_getrf<double>(a);
    SolvePlan<double> sp = plan_solve<double>(a, n, 1);
    cudaStream_t      s  = as_stream(stream);
    k_status_init<<<1, 32, 0, s>>>(gp.st, gp.perm);
    B200LA_LAUNCH_CHECK();
    const int32_t withheld = 1;
    B200LA_CUDA(cudaMemcpyAsync(sp.ticket, &withheld, sizeof(withheld), cudaMemcpyHostToDevice, s));
    const int nb = (int)((n + kTvRows - 1) / kTvRows);
    k_trsv_blocks<double, true><<<nb, kTvThreads, 0, s>>>(lu, n, x, (int)n, 0, nullptr, sp.xll, tv_next_epoch(),
        sp.ticket, gp.st, wait_ns);
    B200LA_LAUNCH_CHECK();
    k_status_finish<<<1, 32, 0, s>>>(gp.st);
    B200LA_LAUNCH_CHECK();
    return read_status(gp.st, nullptr, s);
}

// Latency floor of the cluster panel's per-column exchange (measurement
// hook): k_panel_exchange_floor for `columns` columns, FP64 (elem_bytes 8)
// or FP32 (4) records of a 64- or 32-column panel, in the cluster size the
// panel kernel uses.  Synchronizes `stream`; *ns_per_column receives the
// device-timed nanoseconds per column.  Workspace: 256 bytes.
B200LA_API int b200la_panel_exchange_floor(int elem_bytes, int width, int columns, double* ns_per_column, void* ws,
    size_t bytes, void* stream)
{
    if (ns_per_column == nullptr || ws == nullptr || bytes < 256 || columns < 1 || columns > 1 << 20 ||
        (elem_bytes != 4 && elem_bytes != 8) || (width != 32 && width != 64))
    {
        return set_error(B200LA_INVALID_ARGUMENT, "panel_exchange_floor: bad arguments");
    }
    int st = elem_bytes == 8 ? prepare<double>() : prepare<float>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    int cl = 0, gmax = 0;
    st = elem_bytes == 8 ? panel_config<double>(cl, gmax) : panel_config<float>(cl, gmax);
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    if (cl <= 0)
    {
        return set_error(B200LA_NOT_SUPPORTED, "panel_exchange_floor: no usable cluster size");
    }
    cudaStream_t        s  = as_stream(stream);
    unsigned long long* ns = static_cast<unsigned long long*>(ws);
    cudaLaunchConfig_t  cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim              = dim3(cl);
    cfg.blockDim             = dim3(kPanelThreads);
    cfg.stream               = s;
    attr[0].id               = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cl;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs                = attr;
    cfg.numAttrs             = 1;
    if (elem_bytes == 8 && width == 64)
    {
        B200LA_CUDA(cudaLaunchKernelEx(&cfg, k_panel_exchange_floor<double, 64>, columns, ns));
    }
    else if (elem_bytes == 8)
    {
        B200LA_CUDA(cudaLaunchKernelEx(&cfg, k_panel_exchange_floor<double, 32>, columns, ns));
    }
    else if (width == 64)
    {
        B200LA_CUDA(cudaLaunchKernelEx(&cfg, k_panel_exchange_floor<float, 64>, columns, ns));
    }
    else
    {
        B200LA_CUDA(cudaLaunchKernelEx(&cfg, k_panel_exchange_floor<float, 32>, columns, ns));
    }
    unsigned long long h = 0;
    B200LA_CUDA(cudaMemcpyAsync(&h, ns, sizeof(h), cudaMemcpyDeviceToHost, s));
    B200LA_CUDA(cudaStreamSynchronize(s));
    *ns_per_column = (double)h / columns;
    return B200LA_SUCCESS;
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
// Driver entry points for identifying the current context (resolved through
// the runtime, so the library does not link libcuda).
using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn      = int (*)(void*, unsigned long long*);

struct NoAllocCache
{
    unsigned long long ctx_id;  // 0: free slot
    void*              address;
};

std::mutex   g_noalloc_mutex;
NoAllocCache g_noalloc_cache[64] = {};

// Unique id of the current context (cuCtxGetId), 0 if it cannot be had.
unsigned long long current_context_id()
{
    static CtxGetCurrentFn get_current = [] {
        void*                           p = nullptr;
        cudaDriverEntryPointQueryResult q;
        return (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess)
                   ? reinterpret_cast<CtxGetCurrentFn>(p)
                   : nullptr;
    }();
    static CtxGetIdFn get_id = [] {
        void*                           p = nullptr;
        cudaDriverEntryPointQueryResult q;
        return (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
                   q == cudaDriverEntryPointSuccess)
                   ? reinterpret_cast<CtxGetIdFn>(p)
                   : nullptr;
    }();
    void*              ctx = nullptr;
    unsigned long long id  = 0;
    if (get_current == nullptr || get_id == nullptr || get_current(&ctx) != 0 || ctx == nullptr ||
        get_id(ctx, &id) != 0)
    {
        return 0;
    }
    return id;
}

// Device address of g_noalloc_scratch in the current context.  The host-side
// name of the array is only a stand-in, so the address is looked up with the
// device current (cudaGetSymbolAddress) the first time a context calls, and
// cached under that context's unique id: a context created later (after a
// cudaDeviceReset, say, which unloads the module and may place the array
// elsewhere) has a new id and gets its own lookup.  Without a context id
// the address is looked up on every call.
int noalloc_scratch(void** out)
{
    int dev = 0;
    B200LA_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64)
    {
        return set_error(B200LA_NOT_SUPPORTED, "dgesv_noalloc: device index %d out of range", dev);
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    const unsigned long long    id = current_context_id();
    if (id != 0 && g_noalloc_cache[dev].ctx_id == id)
    {
        *out = g_noalloc_cache[dev].address;
        return B200LA_SUCCESS;
    }
    void*             p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess)
    {
        return cuda_check(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    }
    // cudaGetSymbolAddress makes the primary context current if none was:
    // key the entry on the context it answered for
    const unsigned long long id_now = id != 0 ? id : current_context_id();
    g_noalloc_cache[dev]            = NoAllocCache{id_now, p};
    *out                            = p;
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
