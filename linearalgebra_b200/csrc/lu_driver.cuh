// Host-side helpers shared by the LU drivers (plain FP64/FP32 LU-solve path
// and the mixed-precision solver): workspace plans, kernel attributes, panel
// launch, triangular-solve sequencing.
#pragma once

#include <cuda_runtime.h>

#include <climits>
#include <cstdint>
#include <cstdlib>
#include <mutex>

#include "cholesky.cuh"
#include "dmma.cuh"
#include "lu_kernels.cuh"
#include "solve_kernels.cuh"
#include "trsv.cuh"

namespace b200la
{
int require_sm100();

constexpr size_t kPanelSmemMax = 200 * 1024;
// dynamic shared memory of the 64-column cluster panel (the probe's kernel):
// sm_100's 227 KB per CTA less 6 KB for its static arrays
constexpr size_t kClusterSmemMax = cluster_dyn_max<double, 64>();
constexpr int    kLeanPanelCtas = 48;  // grid panel CTAs beside a concurrent trailing update


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
        cfg.dynamicSmemBytes           = kClusterSmemMax;
        attr[0].id                     = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x       = cl;
        attr[0].val.clusterDim.y       = 1;
        attr[0].val.clusterDim.z       = 1;
        cfg.attrs                      = attr;
        cfg.numAttrs                   = 1;
        int clusters                   = 0;
        if (cudaOccupancyMaxActiveClusters(&clusters, (const void*)k_panel_cluster<T, 64>, &cfg) ==
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
        k_perm_from_pivots<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    B200LA_CUDA(cudaFuncSetAttribute(
        k_panel_cluster<T, 64>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cluster_dyn_max<T, 64>()));
    B200LA_CUDA(cudaFuncSetAttribute(k_panel_cluster<T, 64>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    B200LA_CUDA(cudaFuncSetAttribute(
        k_panel_cluster<T, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cluster_dyn_max<T, 32>()));
    B200LA_CUDA(cudaFuncSetAttribute(k_panel_cluster<T, 32>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    B200LA_CUDA(cudaFuncSetAttribute(
        k_panel_exchange_floor<T, 64>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    B200LA_CUDA(cudaFuncSetAttribute(
        k_panel_exchange_floor<T, 32>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    if (dev >= 0 && dev < 64)
    {
        cluster_size_slot<T>(dev) = probe_cluster_size<T>();
    }
    B200LA_CUDA(cudaFuncSetAttribute(
        k_laswp_trsm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)laswp_smem_bytes<T>()));
    B200LA_CUDA(cudaFuncSetAttribute(
        k_trailing<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)trailing_smem_bytes<T>()));
    B200LA_CUDA(cudaFuncSetAttribute(
        k_dmma_update<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDmSmem));
    B200LA_CUDA(cudaFuncSetAttribute(
        k_dmma_update<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDmSmem));
    B200LA_CUDA(cudaFuncSetAttribute(k_dmma_band<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBandSmem));
    B200LA_CUDA(cudaFuncSetAttribute(k_dmma_gemm<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDmSmem));
    B200LA_CUDA(cudaFuncSetAttribute(k_chol_diag<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)chol_smem_bytes<T>()));
    B200LA_CUDA(cudaFuncSetAttribute(k_chol_trsm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)chol_trsm_smem_bytes<T>()));
    B200LA_CUDA(cudaFuncSetAttribute(k_chol_syrk<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)chol_smem_bytes<T>()));
    B200LA_CUDA(cudaFuncSetAttribute(k_dmma_gemm<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDmSmem));
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

// Shared memory for k_perm_from_pivots: the whole permutation when it fits
// in 200 KB (n <= 51200), else 0 (the kernel then works in global memory).
inline size_t perm_smem_bytes(int n)
{
    const size_t b = (size_t)n * sizeof(int32_t);
    return b <= 200 * 1024 ? b : 0;
}

inline int prepare_device()
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
    int32_t*  perm;
    T*        y;
    // one-launch triangular solves (FP64, one right-hand side)
    uint64_t* xll;    // flagged copies of solved blocks (16 bytes per row)
    int32_t*  ticket; // block ticket of k_trsv_blocks
};

template <typename T> SolvePlan<T> plan_solve(Arena& a, int64_t n, int64_t nrhs)
{
    SolvePlan<T> p{};
    p.perm = a.next<int32_t>((size_t)n);
    p.y    = a.next<T>((size_t)n * (size_t)nrhs);
    if (sizeof(T) == 8 && nrhs == 1)
    {
        const size_t nb = (size_t)((n + kTvRows - 1) / kTvRows);
        p.ticket        = a.next<int32_t>(32);
        p.xll           = a.next<uint64_t>(nb * kTvRows * 2);
    }
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
// Factor panel [k, k+w) of rows [k, n): inside one thread-block cluster when
// its rows fit there (cl > 0), else with the grid-wide kernel.
// Whether a panel of `rows` rows and width w fits the cluster panel kernel
// on a cluster of `cl` CTAs.
template <typename T> bool cluster_panel_fits(int rows, int w, int cl)
{
    if (cl <= 0)
    {
        return false;
    }
    const size_t rpc = (size_t)((rows + cl - 1) / cl);
    return w <= 32 ? rpc * cluster_row_bytes<T, 32>() <= cluster_dyn_max<T, 32>()
                   : rpc * cluster_row_bytes<T, 64>() <= cluster_dyn_max<T, 64>();
}

// Whether launch_panel takes the fusing cluster kernel for this panel and
// can apply a previous panel of width prev_w first (both at most 32 wide).
template <typename T> bool panel_can_fuse(int rows, int w, int prev_w, int cl)
{
    return cluster_fuses<T, 32>() && w <= 32 && prev_w >= 1 && prev_w <= 32 && cluster_panel_fits<T>(rows, w, cl);
}

// pperm / pk: the previous panel's interchange list and first column, whose
// interchanges, U12 and update on this panel's columns the panel kernel then
// applies first (only where panel_can_fuse; an error otherwise).
template <typename T>
int launch_panel(T* m, int n, int k, int w, int64_t* pivot, const GetrfPlan<T>& p, int cl, int gmax,
    cudaStream_t s, bool lean = false, const PermList* pperm = nullptr, int pk = -1)
{
    if (pperm != nullptr && !panel_can_fuse<T>(n - k, w, k - pk, cl))
    {
        return set_error(B200LA_NOT_SUPPORTED, "panel: the fused update needs the FP32 32-column cluster kernel");
    }
    const int R = n - k;
    PanelWs<T> ws{p.hdr, p.payload, p.diag, p.perm};
    DeviceStatus* st = p.st;
    // the panel inside one thread-block cluster when its rows fit there
    if (cluster_panel_fits<T>(R, w, cl))
    {
        const int           rpc = (R + cl - 1) / cl;
        cudaLaunchConfig_t  cfg = {};
        cudaLaunchAttribute attr[1];
        cfg.gridDim              = dim3(cl);
        cfg.blockDim             = dim3(kPanelThreads);
        cfg.dynamicSmemBytes     = (size_t)rpc * (w <= 32 ? cluster_row_bytes<T, 32>() : cluster_row_bytes<T, 64>());
        cfg.stream               = s;
        attr[0].id               = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cl;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs                = attr;
        cfg.numAttrs             = 1;
        prof_begin(KC_PANEL, s);
        if (w <= 32)
        {
            B200LA_CUDA(cudaLaunchKernelEx(&cfg, k_panel_cluster<T, 32>, m, n, k, w, rpc, pivot, p.perm, p.st,
                pperm, pk));
        }
        else
        {
            B200LA_CUDA(cudaLaunchKernelEx(&cfg, k_panel_cluster<T, 64>, m, n, k, w, rpc, pivot, p.perm, p.st,
                (const PermList*)nullptr, -1));
        }
        prof_end(KC_PANEL, s);
        return B200LA_SUCCESS;
    }
    {
        int       G   = (R + 15) / 16;
        if (lean)
        {
            // beside a concurrent trailing update: the fewest CTAs that hold
            // the panel in shared memory (at least kLeanPanelCtas), so the
            // update keeps the other SMs
            const int rows_fit = (int)(kPanelSmemMax / (panel_ldl<T>() * sizeof(T)));
            const int g_fit    = (R + rows_fit - 1) / rows_fit;
            G                  = G < kLeanPanelCtas ? G : (g_fit > kLeanPanelCtas ? g_fit : kLeanPanelCtas);
        }
        G             = G < 1 ? 1 : (G > gmax ? gmax : G);
        int rpc       = (R + G - 1) / G;
        G             = (R + rpc - 1) / rpc;
        size_t smem   = (size_t)rpc * panel_ldl<T>() * sizeof(T);
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

    return B200LA_SUCCESS;
}

// Cluster size for the cluster panel kernel on the current device (0: the
// grid-wide kernel only) and the grid kernel's CTA limit.
// B200LA_FORCE_GRID_PANEL=1 keeps every panel on the grid-wide kernel (used
// by the tests to check both panel paths).
template <typename T> int panel_config(int& cl, int& gmax)
{
    const int sms = device_sm_count();
    gmax          = sms < kMaxPanelCtas ? sms : kMaxPanelCtas;
    int dev       = 0;
    B200LA_CUDA(cudaGetDevice(&dev));
    const char* force_grid = getenv("B200LA_FORCE_GRID_PANEL");
    cl = (force_grid != nullptr && force_grid[0] == '1')
             ? 0
             : ((dev >= 0 && dev < 64) ? cluster_size_slot<T>(dev) : 0);
    return B200LA_SUCCESS;
}

template <typename T> int clear_panel_exchange(const GetrfPlan<T>& p, cudaStream_t s)
{
    // the exchange words carry column flags: clear them so no word of an
    // earlier factorization can validate
    B200LA_CUDA(cudaMemsetAsync(p.hdr, 0, sizeof(uint64_t) * panel_hdr_words<T>(), s));
    B200LA_CUDA(cudaMemsetAsync(p.payload, 0, sizeof(uint64_t) * panel_payload_words<T>(), s));
    B200LA_CUDA(cudaMemsetAsync(p.diag, 0, sizeof(uint64_t) * panel_diag_words<T>(), s));
    return B200LA_SUCCESS;
}

// The high-priority stream the next panel runs on while the current
// trailing update finishes (one per device, created on first use).
inline cudaStream_t panel_side_stream(int* rc)
{
    static std::mutex   mu;
    static cudaStream_t streams[64] = {};
    int                 dev         = 0;
    *rc                             = B200LA_SUCCESS;
    cudaError_t e                   = cudaGetDevice(&dev);
    if (e != cudaSuccess)
    {
        *rc = cuda_check(e, "cudaGetDevice");
        return nullptr;
    }
    if (dev < 0 || dev >= 64)
    {
        *rc = set_error(B200LA_NOT_SUPPORTED, "device index %d out of range", dev);
        return nullptr;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (streams[dev] == nullptr)
    {
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        e = cudaStreamCreateWithPriority(&streams[dev], cudaStreamNonBlocking, greatest);
        if (e != cudaSuccess)
        {
            streams[dev] = nullptr;
            *rc          = cuda_check(e, "cudaStreamCreateWithPriority");
            return nullptr;
        }
    }
    return streams[dev];
}

// B200LA_LU_LOOKAHEAD=0 turns the look-ahead off (used to check that it
// leaves every bit unchanged).
inline bool lu_lookahead_enabled()
{
    const char* e = getenv("B200LA_LU_LOOKAHEAD");
    return !(e != nullptr && e[0] == '0');
}

// Trailing update A22[:, c0:c1] -= L21 U12[:, c0:c1] of panel (k, w); the
// columns c0, c1 are relative to the first trailing column k + w.
template <typename T>
int launch_trailing(T* m, int n, int k, int w, int c0, int c1, cudaStream_t s)
{
    const int rest = n - k - w;
    prof_begin(KC_TRAILING, s);
    if constexpr (sizeof(T) == 8)
    {
        // A22 -= L21 U12 on the tensor cores, delta from zero then
        // subtracted: the same bits as k_trailing's fma loop.
        static_assert(kNB <= kBandK, "the band kernel holds one panel's L21 slice");
        const double* l21 = m + (int64_t)(k + w) * n + k;
        const double* u12 = m + (int64_t)k * n + k + w + c0;
        double*       a22 = m + (int64_t)(k + w) * n + k + w + c0;
        const int     nc  = c1 - c0;
        k_dmma_band<0><<<band_grid(rest, nc, device_sm_count()), kDmThreads, kBandSmem, s>>>(
            rest, nc, w, l21, n, u12, n, a22, n, dm_vec16(l21, n, u12, n, a22, n), nullptr);
    }
    else
    {
        // k_trailing covers columns [0, ncols) of A22; only whole updates here
        dim3 grid((c1 + kChunkN - 1) / kChunkN, (rest + kBandM - 1) / kBandM);
        k_trailing<T><<<grid, 128, trailing_smem_bytes<T>(), s>>>(m, n, k, w, c1, 0);
    }
    prof_end(KC_TRAILING, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

template <typename T>
int enqueue_getrf(T* m, int n, int64_t* pivot, const GetrfPlan<T>& p, cudaStream_t s)
{
    {
        const int rc = clear_panel_exchange<T>(p, s);
        if (rc != B200LA_SUCCESS)
        {
            return rc;
        }
    }
    prof_begin(KC_SOLVE, s);
    k_status_init<<<1, 32, 0, s>>>(p.st, p.perm);
    prof_end(KC_SOLVE, s);
    B200LA_LAUNCH_CHECK();
    int cl = 0, gmax = 0;
    {
        const int rc = panel_config<T>(cl, gmax);
        if (rc != B200LA_SUCCESS)
        {
            return rc;
        }
    }
    // Look-ahead (FP64): after panel k's interchanges and U12, the trailing
    // update of the next panel's columns runs first; panel k+1 then factors
    // on the side stream while the rest of the update runs here.  Every
    // element sees the same operations in the same order as without it.
    const bool   ahead = sizeof(T) == 8 && lu_lookahead_enabled() && n > 2 * kNB;
    cudaStream_t side  = nullptr;
    cudaEvent_t  ev_cols = nullptr, ev_panel = nullptr;
    if (ahead)
    {
        int rc = B200LA_SUCCESS;
        side   = panel_side_stream(&rc);
        if (rc != B200LA_SUCCESS)
        {
            return rc;
        }
        B200LA_CUDA(cudaEventCreateWithFlags(&ev_cols, cudaEventDisableTiming));
        B200LA_CUDA(cudaEventCreateWithFlags(&ev_panel, cudaEventDisableTiming));
    }
    struct EventGuard
    {
        cudaEvent_t a, b;
        ~EventGuard()
        {
            if (a)
                cudaEventDestroy(a);
            if (b)
                cudaEventDestroy(b);
        }
    } guard{ev_cols, ev_panel};

    {
        const int w0  = n < kNB ? n : kNB;
        const int prc = launch_panel<T>(m, n, 0, w0, pivot, p, cl, gmax, s);
        if (prc != B200LA_SUCCESS)
        {
            return prc;
        }
    }
    for (int k = 0; k < n; k += kNB)
    {
        const int w    = n - k < kNB ? n - k : kNB;
        const int rest = n - k - w;
        const int nl   = (k + kSwapCols - 1) / kSwapCols;
        const int nr   = (rest + kSwapCols - 1) / kSwapCols;
        if (nl + nr > 0)
        {
            prof_begin(KC_SWAP, s);
            k_laswp_trsm<T><<<nl + nr, kSwapThreads, laswp_smem_bytes<T>(), s>>>(m, n, k, w, p.perm, nl, n, 0, k, n,
                k + w);
            prof_end(KC_SWAP, s);
            B200LA_LAUNCH_CHECK();
        }
        if (rest <= 0)
        {
            break;
        }
        const int kn = k + w;  // the next panel
        const int wn = rest < kNB ? rest : kNB;
        int       rc = B200LA_SUCCESS;
        if (ahead && rest > wn)
        {
            rc = launch_trailing<T>(m, n, k, w, 0, wn, s);
            if (rc != B200LA_SUCCESS)
            {
                return rc;
            }
            B200LA_CUDA(cudaEventRecord(ev_cols, s));
            B200LA_CUDA(cudaStreamWaitEvent(side, ev_cols, 0));
            rc = launch_panel<T>(m, n, kn, wn, pivot, p, cl, gmax, side, true);
            if (rc != B200LA_SUCCESS)
            {
                return rc;
            }
            B200LA_CUDA(cudaEventRecord(ev_panel, side));
            rc = launch_trailing<T>(m, n, k, w, wn, rest, s);
            if (rc != B200LA_SUCCESS)
            {
                return rc;
            }
            B200LA_CUDA(cudaStreamWaitEvent(s, ev_panel, 0));
        }
        else
        {
            rc = launch_trailing<T>(m, n, k, w, 0, rest, s);
            if (rc != B200LA_SUCCESS)
            {
                return rc;
            }
            rc = launch_panel<T>(m, n, kn, wn, pivot, p, cl, gmax, s);
            if (rc != B200LA_SUCCESS)
            {
                return rc;
            }
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

inline int read_status(const DeviceStatus* dst, int* info, cudaStream_t s)
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
template <typename TA, typename T = TA>
int enqueue_trsm_inplace(bool upper, bool transpose, bool unit, int n, int nrhs, const TA* a,
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
        k_trsm_diag<TA, T><<<(nrhs + kTrsmCols - 1) / kTrsmCols, kTrsmCols, 0, s>>>(
            a, lda, transpose, eff_upper, unit, r0, bw, x, ldx, nrhs, gate);
        prof_end(KC_SOLVE, s);
        B200LA_LAUNCH_CHECK();
        if (um > 0)
        {
            dim3 grid((nrhs + kUpdCols - 1) / kUpdCols, (um + 63) / 64);
            prof_begin(KC_SOLVE, s);
            k_trsm_update<TA, T><<<grid, 256, 0, s>>>(a, lda, transpose, r0, bw, u0, um, x, ldx, nrhs, gate);
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
    const size_t perm_smem = perm_smem_bytes(n);
    const int    use_smem  = perm_smem > 0 ? 1 : 0;
    prof_begin(KC_SOLVE, s);
    k_perm_from_pivots<0><<<1, 256, perm_smem, s>>>(pivot, n, sp.perm, use_smem, st, gate);
    prof_end(KC_SOLVE, s);
    B200LA_LAUNCH_CHECK();
    const int64_t total = (int64_t)n * nrhs;
    prof_begin(KC_SOLVE, s);
    k_gather_rows<T><<<grid_1d(total, 256), 256, 0, s>>>(x, ldx, sp.perm, sp.y, nrhs, n, nrhs, gate);
    prof_end(KC_SOLVE, s);
    B200LA_LAUNCH_CHECK();
    if constexpr (sizeof(T) == 8)
    {
        if (nrhs == 1 && sp.xll != nullptr)
        {
            // L then U, each in one launch: 64-row blocks claimed in solve
            // order, solved blocks published as flagged words (bounded
            // waits), each diagonal block solved by substitution.  On an
            // exactly singular factorization (gate set) this works on
            // scratch only and the final copy below is skipped.
            const int nb = (n + kTvRows - 1) / kTvRows;
            for (int pass = 0; pass < 2; ++pass)
            {
                B200LA_CUDA(cudaMemsetAsync(sp.ticket, 0, sizeof(int32_t), s));
                const uint32_t epoch = tv_next_epoch();
                prof_begin(KC_SOLVE, s);
                k_trsv_blocks<double, true><<<nb, kTvThreads, 0, s>>>(lu, n, sp.y, n, pass, nullptr, sp.xll, epoch,
                    sp.ticket, st, kWaitLimitNs);
                prof_end(KC_SOLVE, s);
                B200LA_LAUNCH_CHECK();
            }
            prof_begin(KC_SOLVE, s);
            k_copy2d<T><<<grid_1d(total, 256), 256, 0, s>>>(sp.y, nrhs, x, ldx, n, nrhs, gate);
            prof_end(KC_SOLVE, s);
            B200LA_LAUNCH_CHECK();
            return B200LA_SUCCESS;
        }
    }
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

// Blocked lower Cholesky of m (n x n, row-major) in the reference's order
// (cholesky.cuh); upper: then transposed into the upper triangle.  The status
// block gets the first non-positive pivot; later kernels are gated on it.
// Look-ahead: the trailing update of block k is split into its first tile
// column (the next block's columns) and the rest; the next block's diagonal
// and panel kernels run on a side stream beside the rest.
template <typename T> int launch_chol_block(T* m, int n, int k, DeviceStatus* st, cudaStream_t s)
{
    const int bs    = n - k < kCholNB ? n - k : kCholNB;
    const int below = n - k - bs;
    prof_begin(KC_CHOL_AUX, s);
    k_chol_diag<T><<<1, kCholNB, chol_smem_bytes<T>(), s>>>(m, n, k, bs, st);
    prof_end(KC_CHOL_AUX, s);
    B200LA_LAUNCH_CHECK();
    if (below > 0)
    {
        prof_begin(KC_CHOL_AUX, s);
        k_chol_trsm<T><<<(below + kCholTrsmRows - 1) / kCholTrsmRows, kCholTrsmRows, chol_trsm_smem_bytes<T>(),
            s>>>(m, n, k, st);
        prof_end(KC_CHOL_AUX, s);
        B200LA_LAUNCH_CHECK();
    }
    return B200LA_SUCCESS;
}

template <typename T> int launch_chol_syrk(T* m, int n, int k, int set, DeviceStatus* st, cudaStream_t s)
{
    const int64_t tiles = (n - k - kCholNB + kSyrkTile - 1) / kSyrkTile;
    const int64_t grid  = set == kSyrkFirst ? tiles : set == kSyrkRest ? tiles * (tiles - 1) / 2 : tiles * (tiles + 1) / 2;
    if (grid <= 0)
    {
        return B200LA_SUCCESS;
    }
    prof_begin(KC_CHOL_UPD, s);
    k_chol_syrk<T><<<(unsigned)grid, 256, chol_smem_bytes<T>(), s>>>(m, n, k, set, st);
    prof_end(KC_CHOL_UPD, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

template <typename T> int enqueue_potrf(T* m, int n, bool upper, DeviceStatus* st, cudaStream_t s)
{
    prof_begin(KC_CHOL_AUX, s);
    k_status_init<<<1, 32, 0, s>>>(st, nullptr);
    prof_end(KC_CHOL_AUX, s);
    B200LA_LAUNCH_CHECK();
    const bool   ahead = lu_lookahead_enabled() && n > 2 * kCholNB;
    cudaStream_t side  = nullptr;
    cudaEvent_t  ev_cols = nullptr, ev_block = nullptr;
    if (ahead)
    {
        int rc = B200LA_SUCCESS;
        side   = panel_side_stream(&rc);
        if (rc != B200LA_SUCCESS)
        {
            return rc;
        }
        B200LA_CUDA(cudaEventCreateWithFlags(&ev_cols, cudaEventDisableTiming));
        B200LA_CUDA(cudaEventCreateWithFlags(&ev_block, cudaEventDisableTiming));
    }
    struct EventGuard
    {
        cudaEvent_t a, b;
        ~EventGuard()
        {
            if (a)
                cudaEventDestroy(a);
            if (b)
                cudaEventDestroy(b);
        }
    } guard{ev_cols, ev_block};
    int rc = launch_chol_block<T>(m, n, 0, st, s);
    for (int k = 0; rc == B200LA_SUCCESS && n - k > kCholNB; k += kCholNB)
    {
        if (ahead)
        {
            rc = launch_chol_syrk<T>(m, n, k, kSyrkFirst, st, s);
            if (rc != B200LA_SUCCESS)
            {
                break;
            }
            B200LA_CUDA(cudaEventRecord(ev_cols, s));
            B200LA_CUDA(cudaStreamWaitEvent(side, ev_cols, 0));
            rc = launch_chol_block<T>(m, n, k + kCholNB, st, side);
            if (rc != B200LA_SUCCESS)
            {
                break;
            }
            B200LA_CUDA(cudaEventRecord(ev_block, side));
            rc = launch_chol_syrk<T>(m, n, k, kSyrkRest, st, s);
            B200LA_CUDA(cudaStreamWaitEvent(s, ev_block, 0));
        }
        else
        {
            rc = launch_chol_syrk<T>(m, n, k, kSyrkAll, st, s);
            if (rc == B200LA_SUCCESS)
            {
                rc = launch_chol_block<T>(m, n, k + kCholNB, st, s);
            }
        }
    }
    if (rc != B200LA_SUCCESS)
    {
        return rc;
    }
    if (upper)
    {
        prof_begin(KC_CHOL_AUX, s);
        k_chol_to_upper<T><<<grid_1d((int64_t)n * n, 256), 256, 0, s>>>(m, n, st);
        prof_end(KC_CHOL_AUX, s);
        B200LA_LAUNCH_CHECK();
    }
    prof_begin(KC_CHOL_AUX, s);
    k_status_finish<<<1, 32, 0, s>>>(st);
    prof_end(KC_CHOL_AUX, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

// Solve with a lower Cholesky factor in place on x (n x nrhs, row stride
// ldx): L y = x, then L^T x = y.  Gated on the factorization's status.
template <typename T>
int enqueue_potrs(const T* l, int n, int nrhs, T* x, int64_t ldx, const SolvePlan<T>& sp, DeviceStatus* st,
    const DeviceStatus* gate, cudaStream_t s)
{
    if constexpr (sizeof(T) == 8)
    {
        if (nrhs == 1 && sp.xll != nullptr)
        {
            // L y = x, then L^T x = y, each in one launch (k_trsv_blocks, the
            // Cholesky variant) on scratch; the result is copied back only if
            // the factorization succeeded
            const int nb = (n + kTvRows - 1) / kTvRows;
            prof_begin(KC_SOLVE, s);
            k_copy2d<T><<<grid_1d(n, 256), 256, 0, s>>>(x, ldx, sp.y, 1, n, 1, nullptr);
            prof_end(KC_SOLVE, s);
            B200LA_LAUNCH_CHECK();
            for (int pass = 0; pass < 2; ++pass)
            {
                B200LA_CUDA(cudaMemsetAsync(sp.ticket, 0, sizeof(int32_t), s));
                const uint32_t epoch = tv_next_epoch();
                prof_begin(KC_SOLVE, s);
                k_trsv_blocks<double, true, true><<<nb, kTvThreads, 0, s>>>(l, n, sp.y, n, pass, nullptr, sp.xll,
                    epoch, sp.ticket, st, kWaitLimitNs);
                prof_end(KC_SOLVE, s);
                B200LA_LAUNCH_CHECK();
            }
            prof_begin(KC_SOLVE, s);
            k_copy2d<T><<<grid_1d(n, 256), 256, 0, s>>>(sp.y, 1, x, ldx, n, 1, gate);
            prof_end(KC_SOLVE, s);
            B200LA_LAUNCH_CHECK();
            return B200LA_SUCCESS;
        }
    }
    int rc = enqueue_trsm_inplace<T>(false, false, false, n, nrhs, l, n, x, ldx, gate, s);
    if (rc != B200LA_SUCCESS)
    {
        return rc;
    }
    return enqueue_trsm_inplace<T>(false, true, false, n, nrhs, l, n, x, ldx, gate, s);
}

template <typename T> size_t gesv_ws_size(int64_t n, int mode)
{
    if (n <= 0 || mode < B200LA_LU_LINEAR_SOLVER || mode > B200LA_CHOLESKY_UPFRONT_LINEAR_SOLVER)
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
    if (mode < B200LA_LU_LINEAR_SOLVER || mode > B200LA_CHOLESKY_UPFRONT_LINEAR_SOLVER)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "unsupported linear_solver_type (%d)", mode);
    }
    const bool chol = mode == B200LA_CHOLESKY_LINEAR_SOLVER || mode == B200LA_CHOLESKY_UPFRONT_LINEAR_SOLVER;
    if (!chol && pivot == nullptr)
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
    if (chol)
    {
        // linear_solver_native.cpp: CHOLESKY factors (lower) and solves only
        // if the matrix is positive definite; CHOLESKY_UPFRONT solves with
        // the given lower factor
        if (mode == B200LA_CHOLESKY_LINEAR_SOLVER)
        {
            st = enqueue_potrf<T>(m, (int)n, false, gp.st, s);
        }
        else
        {
            prof_begin(KC_SOLVE, s);
            k_status_init<<<1, 32, 0, s>>>(gp.st, nullptr);
            prof_end(KC_SOLVE, s);
            B200LA_LAUNCH_CHECK();
            st = B200LA_SUCCESS;
        }
        if (st != B200LA_SUCCESS)
        {
            return st;
        }
        return enqueue_potrs<T>(m, (int)n, 1, x, 1, sp, gp.st, gp.st, s);
    }
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

template <typename T>
int potrf(T* m, int64_t n, int upper, void* ws, size_t bytes, int* info, void* stream)
{
    if (m == nullptr)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "cholesky_decomposition::apply: C must not be null");
    }
    if (n <= 0)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "cholesky_decomposition::apply: lda must be positive");
    }
    if (upper != 0 && upper != 1)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "Unsupported enum type!");
    }
    if (n > INT_MAX / 2)
    {
        return set_error(B200LA_NOT_SUPPORTED, "cholesky_decomposition: order too large");
    }
    const size_t need = getrf_ws_size<T>(n);
    if (ws == nullptr || bytes < need)
    {
        return set_error(B200LA_WORKSPACE_TOO_SMALL,
            "cholesky_decomposition: workspace is null or too small (%zu < %zu bytes)", bytes, need);
    }
    int st = prepare<T>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    Arena        a(ws, bytes);
    GetrfPlan<T> p = plan_getrf<T>(a);
    cudaStream_t s = as_stream(stream);
    st             = enqueue_potrf<T>(m, (int)n, upper != 0, p.st, s);
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    return read_status(p.st, info, s);
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
    const int r = (int)rows, co = (int)cols, d = (int)depth;
    if constexpr (sizeof(T) == 8)
    {
        if (!tb)
        {
            // op(b) = b: the reference's loop is an fma chain per element in
            // k order from beta c, which the FP64 tensor cores reproduce
            const int  v16 = dm_vec16(a, lda, b, ldb, c, ldc);
            const dim3 dgrid((unsigned)((cols + kDmTile - 1) / kDmTile), (unsigned)((rows + kDmTile - 1) / kDmTile));
            prof_begin(KC_GEMM, s);
            if (ta)
                k_dmma_gemm<true><<<dgrid, kDmThreads, kDmSmem, s>>>(r, co, d, alpha, a, lda, 0, b, ldb, 0, beta, c,
                    ldc, 0, v16);
            else
                k_dmma_gemm<false><<<dgrid, kDmThreads, kDmSmem, s>>>(r, co, d, alpha, a, lda, 0, b, ldb, 0, beta, c,
                    ldc, 0, v16);
            prof_end(KC_GEMM, s);
            B200LA_LAUNCH_CHECK();
            return B200LA_SUCCESS;
        }
    }
    dim3         grid((unsigned)((cols + 63) / 64), (unsigned)((rows + 127) / 128));
    const size_t smem = gemm_smem_bytes<T>();
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

// ---------------------------------------------------------------------------
// batched multiplication: c_i = a_i b_i for `count` packed dim x dim matrices
// (batched_matrix_multiplication, include/matrix_operation/
// multiplication_batched.h; the CUDA_BLAS kernel sums a b from zero in k
// order, multiplication_batched_cublas.cu:15-40).  FP64 on the tensor cores
// (the same fma chain), FP32 on the SIMT kernel (likewise).
// ---------------------------------------------------------------------------
template <typename T> int gemm_batched(int64_t dim, int64_t count, const T* a, const T* b, T* c, void* stream)
{
    if (a == nullptr || b == nullptr || c == nullptr)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "batched_matrix_multiplication: a, b, and c must not be null");
    }
    if (dim <= 0 || count <= 0)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "batched_matrix_multiplication: dim and count must be positive");
    }
    if (dim > INT_MAX / 2)
    {
        return set_error(B200LA_NOT_SUPPORTED, "batched_matrix_multiplication: dim too large");
    }
    int st = prepare<T>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    cudaStream_t  s      = as_stream(stream);
    const int     d      = (int)dim;
    const int64_t stride = dim * dim;
    constexpr int64_t kMaxZ = 65535;
    for (int64_t c0 = 0; c0 < count; c0 += kMaxZ)
    {
        const unsigned nz = (unsigned)(count - c0 < kMaxZ ? count - c0 : kMaxZ);
        const T*       ab = a + c0 * stride;
        const T*       bb = b + c0 * stride;
        T*             cb = c + c0 * stride;
        prof_begin(KC_GEMM, s);
        if constexpr (sizeof(T) == 8)
        {
            const int  v16 = dm_vec16(ab, dim, bb, dim, cb, dim) && (stride % 2) == 0;
            const dim3 grid((unsigned)((d + kDmTile - 1) / kDmTile), (unsigned)((d + kDmTile - 1) / kDmTile), nz);
            k_dmma_gemm<false><<<grid, kDmThreads, kDmSmem, s>>>(d, d, d, 1.0, ab, dim, stride, bb, dim, stride, 0.0,
                cb, dim, stride, v16);
        }
        else
        {
            const dim3 grid((unsigned)((d + 63) / 64), (unsigned)((d + 127) / 128), nz);
            k_gemm<T, false, false><<<grid, 128, gemm_smem_bytes<T>(), s>>>(d, d, d, T(1), ab, dim, bb, dim, T(0),
                cb, dim, stride, stride, stride);
        }
        prof_end(KC_GEMM, s);
        B200LA_LAUNCH_CHECK();
    }
    return B200LA_SUCCESS;
}

}  // namespace b200la
