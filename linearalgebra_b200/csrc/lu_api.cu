// Host drivers and extern "C" entry points for lu_decomposition,
// linear_solver (LU modes), the multi-RHS getrs extension,
// triangular_solver and multiplication.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <cstdlib>
#include <mutex>

#include "lu_kernels.cuh"
#include "solve_kernels.cuh"

namespace b200la
{
int require_sm100();

namespace
{
constexpr size_t kPanelSmemMax = 200 * 1024;


// Cluster size usable by k_panel_cluster on each device (0: none).
template <typename T> int& cluster_size_slot(int dev)
{
    static int sizes[64] = {};
    return sizes[dev];
}

template <typename T> int probe_cluster_size()
{
    for (int cl : {16, 8})
    {
        cudaLaunchConfig_t  cfg = {};
        cudaLaunchAttribute attr[1];
        cfg.gridDim                    = dim3(cl);
        cfg.blockDim                   = dim3(kPanelThreads);
        cfg.dynamicSmemBytes           = kPanelSmemMax;
        attr[0].id                     = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x       = cl;
        attr[0].val.clusterDim.y       = 1;
        attr[0].val.clusterDim.z       = 1;
        cfg.attrs                      = attr;
        cfg.numAttrs                   = 1;
        int clusters                   = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, (const void*)k_panel_cluster<T>, &cfg) ==
                cudaSuccess &&
            clusters > 0)
        {
            return cl;
        }
        cudaGetLastError();
    }
    return 0;
}

// Raise the dynamic shared-memory limits once per device and type.
template <typename T> int ensure_kernel_attributes()
{
    static std::mutex m;
    static bool       done[64] = {};
    int               dev      = 0;
    B200LA_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(m);
    if (dev >= 0 && dev < 64 && done[dev])
    {
        return B200LA_SUCCESS;
    }
    B200LA_CUDA(cudaFuncSetAttribute(
        k_panel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelSmemMax));
    B200LA_CUDA(cudaFuncSetAttribute(
        k_panel_cluster<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelSmemMax));
    B200LA_CUDA(cudaFuncSetAttribute(
        k_panel_cluster<T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    if (dev >= 0 && dev < 64)
    {
        cluster_size_slot<T>(dev) = probe_cluster_size<T>();
    }
    B200LA_CUDA(cudaFuncSetAttribute(
        k_laswp_trsm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)laswp_smem_bytes<T>()));
    B200LA_CUDA(cudaFuncSetAttribute(
        k_trailing<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trailing_smem_bytes<T>()));
    B200LA_CUDA(cudaFuncSetAttribute(k_gemm<T, false, false>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem_bytes<T>()));
    B200LA_CUDA(cudaFuncSetAttribute(k_gemm<T, true, false>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem_bytes<T>()));
    B200LA_CUDA(cudaFuncSetAttribute(k_gemm<T, false, true>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem_bytes<T>()));
    B200LA_CUDA(cudaFuncSetAttribute(k_gemm<T, true, true>,
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gemm_smem_bytes<T>()));
    if (dev >= 0 && dev < 64)
    {
        done[dev] = true;
    }
    return B200LA_SUCCESS;
}

int prepare_device()
{
    return require_sm100();
}

template <typename T> int prepare()
{
    int st = prepare_device();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    return ensure_kernel_attributes<T>();
}

// ---------------------------------------------------------------------------
// Workspace plans.  The same function sizes (Arena()) and carves
// (Arena(base, bytes)).
// ---------------------------------------------------------------------------
template <typename T> struct GetrfPlan
{
    DeviceStatus* st;
    uint64_t*     hdr;
    uint64_t*     payload;
    uint64_t*     diag;
    PermList*     perm;
};

template <typename T> GetrfPlan<T> plan_getrf(Arena& a)
{
    GetrfPlan<T> p;
    p.st      = a.next<DeviceStatus>(1);
    p.hdr     = a.next<uint64_t>(panel_hdr_words<T>());
    p.payload = a.next<uint64_t>(panel_payload_words<T>());
    p.diag    = a.next<uint64_t>(panel_diag_words<T>());
    p.perm    = a.next<PermList>(1);
    return p;
}

template <typename T> struct SolvePlan
{
    int32_t* perm;
    T*       y;
};

template <typename T> SolvePlan<T> plan_solve(Arena& a, int64_t n, int64_t nrhs)
{
    SolvePlan<T> p;
    p.perm = a.next<int32_t>((size_t)n);
    p.y    = a.next<T>((size_t)n * (size_t)nrhs);
    return p;
}

inline cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

inline int grid_1d(int64_t total, int threads)
{
    const int64_t g = (total + threads - 1) / threads;
    return (int)(g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g));
}

// ---------------------------------------------------------------------------
// LU factorization (asynchronous).
// ---------------------------------------------------------------------------
template <typename T>
int enqueue_getrf(T* m, int n, int64_t* pivot, const GetrfPlan<T>& p, cudaStream_t s)
{
    // the exchange words carry column flags: clear them so no word of an
    // earlier factorization can validate
    B200LA_CUDA(cudaMemsetAsync(p.hdr, 0, sizeof(uint64_t) * panel_hdr_words<T>(), s));
    B200LA_CUDA(cudaMemsetAsync(p.payload, 0, sizeof(uint64_t) * panel_payload_words<T>(), s));
    B200LA_CUDA(cudaMemsetAsync(p.diag, 0, sizeof(uint64_t) * panel_diag_words<T>(), s));
    prof_begin(KC_SOLVE, s);
    k_status_init<<<1, 32, 0, s>>>(p.st, p.perm);
    prof_end(KC_SOLVE, s);
    B200LA_LAUNCH_CHECK();
    const int sms  = device_sm_count();
    const int gmax = sms < kMaxPanelCtas ? sms : kMaxPanelCtas;
    int       dev  = 0;
    B200LA_CUDA(cudaGetDevice(&dev));
    // B200LA_FORCE_GRID_PANEL=1 keeps every panel on the grid-wide kernel
    // (used by the tests to check both panel paths)
    const char* force_grid = getenv("B200LA_FORCE_GRID_PANEL");
    const int   cl = (force_grid != nullptr && force_grid[0] == '1')
                       ? 0
                       : ((dev >= 0 && dev < 64) ? cluster_size_slot<T>(dev) : 0);
    PanelWs<T> ws{p.hdr, p.payload, p.diag, p.perm};
    DeviceStatus* st = p.st;
    for (int k = 0; k < n; k += kNB)
    {
        int       w   = n - k < kNB ? n - k : kNB;
        const int R   = n - k;
        // the panel inside one thread-block cluster when its rows fit there
        if (cl > 0)
        {
            const int    rpc_c  = (R + cl - 1) / cl;
            const size_t smem_c = (size_t)rpc_c * (kNB + 1) * sizeof(T);
            if (smem_c <= kPanelSmemMax)
            {
                cudaLaunchConfig_t  cfg = {};
                cudaLaunchAttribute attr[1];
                cfg.gridDim              = dim3(cl);
                cfg.blockDim             = dim3(kPanelThreads);
                cfg.dynamicSmemBytes     = smem_c;
                cfg.stream               = s;
                attr[0].id               = cudaLaunchAttributeClusterDimension;
                attr[0].val.clusterDim.x = cl;
                attr[0].val.clusterDim.y = 1;
                attr[0].val.clusterDim.z = 1;
                cfg.attrs                = attr;
                cfg.numAttrs             = 1;
                prof_begin(KC_PANEL, s);
                B200LA_CUDA(cudaLaunchKernelEx(&cfg, k_panel_cluster<T>, m, n, k, w, rpc_c, pivot, p.perm, p.st));
                prof_end(KC_PANEL, s);
                goto panel_done;
            }
        }
        {
        int       G   = (R + 15) / 16;
        G             = G < 1 ? 1 : (G > gmax ? gmax : G);
        int rpc       = (R + G - 1) / G;
        G             = (R + rpc - 1) / rpc;
        size_t smem   = (size_t)rpc * (kNB + 1) * sizeof(T);
        int    in_smem = smem <= kPanelSmemMax ? 1 : 0;
        if (!in_smem)
        {
            smem = 0;
        }
        int   kk     = k;
        int   nn     = n;
        void* args[] = {&m, &nn, &kk, &w, &rpc, &in_smem, &pivot, &ws, &st};
        prof_begin(KC_PANEL, s);
        B200LA_CUDA(cudaLaunchCooperativeKernel(
            (const void*)k_panel<T>, dim3(G), dim3(kPanelThreads), args, smem, s));
        prof_end(KC_PANEL, s);
        }
    panel_done:
        const int rest = n - k - w;
        const int nl   = (k + kSwapCols - 1) / kSwapCols;
        const int nr   = (rest + kSwapCols - 1) / kSwapCols;
        if (nl + nr > 0)
        {
            prof_begin(KC_SWAP, s);
            k_laswp_trsm<T><<<nl + nr, kSwapThreads, laswp_smem_bytes<T>(), s>>>(m, n, k, w, p.perm, nl);
            prof_end(KC_SWAP, s);
            B200LA_LAUNCH_CHECK();
        }
        if (rest > 0)
        {
            dim3 grid((rest + kChunkN - 1) / kChunkN, (rest + kBandM - 1) / kBandM);
            prof_begin(KC_TRAILING, s);
            k_trailing<T><<<grid, 128, trailing_smem_bytes<T>(), s>>>(m, n, k, w);
            prof_end(KC_TRAILING, s);
            B200LA_LAUNCH_CHECK();
        }
    }
    prof_begin(KC_SOLVE, s);
    k_status_finish<<<1, 32, 0, s>>>(p.st);
    prof_end(KC_SOLVE, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

template <typename T> size_t getrf_ws_size(int64_t)
{
    Arena a;
    plan_getrf<T>(a);
    return a.size();
}

template <typename T>
int check_getrf_args(const T* m, int64_t n, const int64_t* pivot, void* ws, size_t bytes)
{
    if (m == nullptr || pivot == nullptr)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "lu_decomposition: m and pivot must not be null");
    }
    if (n <= 0)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "lu_decomposition: lda must be positive (got %lld)",
            (long long)n);
    }
    if (n > INT_MAX / 2)
    {
        return set_error(B200LA_NOT_SUPPORTED, "lu_decomposition: order %lld is too large",
            (long long)n);
    }
    const size_t need = getrf_ws_size<T>(n);
    if (ws == nullptr || bytes < need)
    {
        return set_error(B200LA_WORKSPACE_TOO_SMALL,
            "lu_decomposition: workspace is null or too small (%zu < %zu bytes)", bytes, need);
    }
    return B200LA_SUCCESS;
}

template <typename T>
int getrf_async(T* m, int64_t n, int64_t* pivot, void* ws, size_t bytes, void* stream)
{
    int st = check_getrf_args(m, n, pivot, ws, bytes);
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    st = prepare<T>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    Arena        a(ws, bytes);
    GetrfPlan<T> p = plan_getrf<T>(a);
    return enqueue_getrf<T>(m, (int)n, pivot, p, as_stream(stream));
}

int read_status(const DeviceStatus* dst, int* info, cudaStream_t s)
{
    DeviceStatus h;
    B200LA_CUDA(cudaMemcpyAsync(&h, dst, sizeof(h), cudaMemcpyDeviceToHost, s));
    B200LA_CUDA(cudaStreamSynchronize(s));
    if (h.error == DEV_WAIT_TIMEOUT)
    {
        return set_error(B200LA_DEVICE_TIMEOUT,
            "a bounded device-side wait gave up (site %d); results are incomplete", h.error_site);
    }
    if (h.error == DEV_BAD_PIVOT)
    {
        return set_error(B200LA_INVALID_ARGUMENT,
            "pivot vector holds an entry outside [i+1, n]; those entries were ignored");
    }
    if (h.error != 0)
    {
        return set_error(B200LA_CUDA_ERROR, "device status %d", h.error);
    }
    if (info)
    {
        *info = (int)h.info;
    }
    return h.info == 0 ? B200LA_SUCCESS : B200LA_SINGULAR;
}

template <typename T>
int getrf_sync(T* m, int64_t n, int64_t* pivot, void* ws, size_t bytes, int* info, void* stream)
{
    int st = getrf_async<T>(m, n, pivot, ws, bytes, stream);
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    Arena        a(ws, bytes);
    GetrfPlan<T> p = plan_getrf<T>(a);
    return read_status(p.st, info, as_stream(stream));
}

// ---------------------------------------------------------------------------
// Triangular solves, in place on X (X already holds the right-hand sides).
// ---------------------------------------------------------------------------
template <typename T>
int enqueue_trsm_inplace(bool upper, bool transpose, bool unit, int n, int nrhs, const T* a,
    int64_t lda, T* x, int64_t ldx, const DeviceStatus* gate, cudaStream_t s)
{
    const bool eff_upper = upper != transpose;
    const int  nblocks   = (n + kTrsmBlock - 1) / kTrsmBlock;
    for (int step = 0; step < nblocks; ++step)
    {
        int r0, bw, u0, um;
        if (!eff_upper)
        {
            r0 = step * kTrsmBlock;
            bw = n - r0 < kTrsmBlock ? n - r0 : kTrsmBlock;
            u0 = r0 + bw;
            um = n - u0;
        }
        else
        {
            const int hi = n - step * kTrsmBlock;
            r0           = hi - kTrsmBlock > 0 ? hi - kTrsmBlock : 0;
            bw           = hi - r0;
            u0           = 0;
            um           = r0;
        }
        prof_begin(KC_SOLVE, s);
        k_trsm_diag<T><<<(nrhs + kTrsmCols - 1) / kTrsmCols, kTrsmCols, 0, s>>>(
            a, lda, transpose, eff_upper, unit, r0, bw, x, ldx, nrhs, gate);
        prof_end(KC_SOLVE, s);
        B200LA_LAUNCH_CHECK();
        if (um > 0)
        {
            dim3 grid((nrhs + kUpdCols - 1) / kUpdCols, (um + 63) / 64);
            prof_begin(KC_SOLVE, s);
            k_trsm_update<T><<<grid, 256, 0, s>>>(a, lda, transpose, r0, bw, u0, um, x, ldx, nrhs, gate);
            prof_end(KC_SOLVE, s);
            B200LA_LAUNCH_CHECK();
        }
    }
    return B200LA_SUCCESS;
}

// Solve with LU factors: Y = P X, L Y' = Y, U X = Y'.  x is n x nrhs (ldx).
template <typename T>
int enqueue_getrs(const T* lu, const int64_t* pivot, int n, int nrhs, T* x, int64_t ldx,
    const SolvePlan<T>& sp, DeviceStatus* st, const DeviceStatus* gate, cudaStream_t s)
{
    const size_t perm_smem = (size_t)n * sizeof(int32_t);
    const int    use_smem  = perm_smem <= 48 * 1024 ? 1 : 0;
    prof_begin(KC_SOLVE, s);
    k_perm_from_pivots<<<1, 256, use_smem ? perm_smem : 0, s>>>(pivot, n, sp.perm, use_smem, st, gate);
    prof_end(KC_SOLVE, s);
    B200LA_LAUNCH_CHECK();
    const int64_t total = (int64_t)n * nrhs;
    prof_begin(KC_SOLVE, s);
    k_gather_rows<T><<<grid_1d(total, 256), 256, 0, s>>>(x, ldx, sp.perm, sp.y, nrhs, n, nrhs, gate);
    prof_end(KC_SOLVE, s);
    B200LA_LAUNCH_CHECK();
    int rc = enqueue_trsm_inplace<T>(false, false, true, n, nrhs, lu, n, sp.y, nrhs, gate, s);
    if (rc != B200LA_SUCCESS)
    {
        return rc;
    }
    rc = enqueue_trsm_inplace<T>(true, false, false, n, nrhs, lu, n, sp.y, nrhs, gate, s);
    if (rc != B200LA_SUCCESS)
    {
        return rc;
    }
    prof_begin(KC_SOLVE, s);
    k_copy2d<T><<<grid_1d(total, 256), 256, 0, s>>>(sp.y, nrhs, x, ldx, n, nrhs, gate);
    prof_end(KC_SOLVE, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

template <typename T> size_t gesv_ws_size(int64_t n, int mode)
{
    if (n <= 0 || (mode != B200LA_LU_LINEAR_SOLVER && mode != B200LA_LU_UPFRONT_LINEAR_SOLVER))
    {
        return 0;
    }
    Arena a;
    plan_getrf<T>(a);
    plan_solve<T>(a, n, 1);
    return a.size();
}

template <typename T>
int gesv(T* m, int64_t* pivot, int64_t n, T* x, int mode, void* ws, size_t bytes, void* stream)
{
    if (m == nullptr || x == nullptr)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "linear_solver::apply: m and x must not be null");
    }
    if (n <= 0)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "linear_solver::apply: lda must be positive");
    }
    if (mode != B200LA_LU_LINEAR_SOLVER && mode != B200LA_LU_UPFRONT_LINEAR_SOLVER)
    {
        return set_error(B200LA_NOT_SUPPORTED,
            "linear_solver: only the LU modes are provided by this backend (mode %d)", mode);
    }
    if (pivot == nullptr)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "linear_solver: LU modes need a pivot array");
    }
    if (n > INT_MAX / 2)
    {
        return set_error(B200LA_NOT_SUPPORTED, "linear_solver: order too large");
    }
    const size_t need = gesv_ws_size<T>(n, mode);
    if (ws == nullptr || bytes < need)
    {
        return set_error(B200LA_WORKSPACE_TOO_SMALL,
            "linear_solver: workspace is null or too small (%zu < %zu bytes)", bytes, need);
    }
    int st = prepare<T>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    Arena         a(ws, bytes);
    GetrfPlan<T>  gp = plan_getrf<T>(a);
    SolvePlan<T>  sp = plan_solve<T>(a, n, 1);
    cudaStream_t  s  = as_stream(stream);
    if (mode == B200LA_LU_LINEAR_SOLVER)
    {
        st = enqueue_getrf<T>(m, (int)n, pivot, gp, s);
    }
    else
    {
        prof_begin(KC_SOLVE, s);
        k_status_init<<<1, 32, 0, s>>>(gp.st, gp.perm);
        prof_end(KC_SOLVE, s);
        B200LA_LAUNCH_CHECK();
        st = B200LA_SUCCESS;
    }
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    return enqueue_getrs<T>(m, pivot, (int)n, 1, x, 1, sp, gp.st, gp.st, s);
}

template <typename T> size_t getrs_ws_size(int64_t n, int64_t nrhs)
{
    if (n <= 0 || nrhs <= 0)
    {
        return 0;
    }
    Arena a;
    plan_getrf<T>(a);
    plan_solve<T>(a, n, nrhs);
    return a.size();
}

template <typename T>
int getrs(const T* lu, const int64_t* pivot, int64_t n, int64_t nrhs, T* x, int64_t ldx, void* ws,
    size_t bytes, void* stream)
{
    if (lu == nullptr || pivot == nullptr || x == nullptr)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "getrs: null pointer");
    }
    if (n <= 0 || nrhs <= 0 || ldx < nrhs || n > INT_MAX / 2 || nrhs > INT_MAX / 2)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "getrs: invalid sizes");
    }
    const size_t need = getrs_ws_size<T>(n, nrhs);
    if (ws == nullptr || bytes < need)
    {
        return set_error(B200LA_WORKSPACE_TOO_SMALL, "getrs: workspace too small (%zu < %zu)", bytes, need);
    }
    int st = prepare<T>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    Arena        a(ws, bytes);
    GetrfPlan<T> gp = plan_getrf<T>(a);
    SolvePlan<T> sp = plan_solve<T>(a, n, nrhs);
    cudaStream_t s  = as_stream(stream);
    prof_begin(KC_SOLVE, s);
    k_status_init<<<1, 32, 0, s>>>(gp.st, gp.perm);
    prof_end(KC_SOLVE, s);
    B200LA_LAUNCH_CHECK();
    return enqueue_getrs<T>(lu, pivot, (int)n, (int)nrhs, x, ldx, sp, gp.st, gp.st, s);
}

// ---------------------------------------------------------------------------
// triangular_solver
// ---------------------------------------------------------------------------
template <typename T>
int check_trsm(int64_t n, int64_t nrhs, const T* a, int64_t lda, const T* b, int64_t ldb, const T* x,
    int64_t ldx)
{
    if (n <= 0 || nrhs <= 0)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "triangular_solver: dimensions must be positive");
    }
    if (n > INT_MAX || nrhs > INT_MAX)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "checked_narrow: value does not fit in target type");
    }
    if (!a || !b || !x)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "triangular_solver: matrices must not be null");
    }
    if ((const void*)a == (const void*)b || (const void*)a == (const void*)x ||
        (const void*)b == (const void*)x)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "triangular_solver: matrices must use distinct buffers");
    }
    if (lda < n || ldb < nrhs || ldx < nrhs)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "triangular_solver: invalid row stride");
    }
    const int64_t limit = INT64_MAX / n;
    if (lda > limit || ldb > limit || ldx > limit)
    {
        return set_error(B200LA_INVALID_ARGUMENT,
            "triangular_solver: row stride span exceeds supported range");
    }
    return B200LA_SUCCESS;
}

template <typename T>
int trsm(int upper, int transpose, int unit, int64_t n, int64_t nrhs, const T* a, int64_t lda,
    const T* b, int64_t ldb, T* x, int64_t ldx, void* ws, size_t bytes, void* stream)
{
    int st = check_trsm<T>(n, nrhs, a, lda, b, ldb, x, ldx);
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    (void)ws;
    (void)bytes;
    st = prepare<T>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    cudaStream_t  s     = as_stream(stream);
    const int64_t total = n * nrhs;
    prof_begin(KC_SOLVE, s);
    k_copy2d<T><<<grid_1d(total, 256), 256, 0, s>>>(b, ldb, x, ldx, (int)n, (int)nrhs, nullptr);
    prof_end(KC_SOLVE, s);
    B200LA_LAUNCH_CHECK();
    return enqueue_trsm_inplace<T>(upper != 0, transpose != 0, unit != 0, (int)n, (int)nrhs, a, lda, x,
        ldx, nullptr, s);
}

// ---------------------------------------------------------------------------
// multiplication
// ---------------------------------------------------------------------------
template <typename T>
int gemm(int ta, int tb, int64_t rows, int64_t cols, int64_t depth, T alpha, const T* a, int64_t lda,
    const T* b, int64_t ldb, T beta, T* c, int64_t ldc, void* stream)
{
    if (!a || !b || !c)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "multiplication::apply: a, b, and c must not be null");
    }
    if (rows <= 0 || cols <= 0 || depth <= 0 || lda <= 0 || ldb <= 0 || ldc <= 0)
    {
        return set_error(B200LA_INVALID_ARGUMENT,
            "multiplication::apply: rows/columns/depth/lda/ldb/ldc must be positive");
    }
    if (rows > INT_MAX / 2 || cols > INT_MAX / 2 || depth > INT_MAX / 2)
    {
        return set_error(B200LA_NOT_SUPPORTED, "multiplication: dimension too large");
    }
    int st = prepare<T>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    cudaStream_t s = as_stream(stream);
    if (alpha == T(0))
    {
        if (beta != T(1))
        {
            prof_begin(KC_GEMM, s);
            k_scale2d<T><<<grid_1d(rows * cols, 256), 256, 0, s>>>(c, ldc, (int)rows, (int)cols, beta);
            prof_end(KC_GEMM, s);
            B200LA_LAUNCH_CHECK();
        }
        return B200LA_SUCCESS;
    }
    dim3         grid((unsigned)((cols + 63) / 64), (unsigned)((rows + 127) / 128));
    const size_t smem = gemm_smem_bytes<T>();
    const int    r = (int)rows, co = (int)cols, d = (int)depth;
    prof_begin(KC_GEMM, s);
    if (!ta && !tb)
        k_gemm<T, false, false><<<grid, 128, smem, s>>>(r, co, d, alpha, a, lda, b, ldb, beta, c, ldc);
    else if (ta && !tb)
        k_gemm<T, true, false><<<grid, 128, smem, s>>>(r, co, d, alpha, a, lda, b, ldb, beta, c, ldc);
    else if (!ta && tb)
        k_gemm<T, false, true><<<grid, 128, smem, s>>>(r, co, d, alpha, a, lda, b, ldb, beta, c, ldc);
    else
        k_gemm<T, true, true><<<grid, 128, smem, s>>>(r, co, d, alpha, a, lda, b, ldb, beta, c, ldc);
    prof_end(KC_GEMM, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

}  // namespace
}  // namespace b200la

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
    if (m == nullptr || x == nullptr || pivot == nullptr || n <= 0 ||
        (mode != B200LA_LU_LINEAR_SOLVER && mode != B200LA_LU_UPFRONT_LINEAR_SOLVER))
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
