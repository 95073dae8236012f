// Batched solver for many independent dense systems of uneven order
// (16 <= n <= 512), in ONE persistent kernel launch.
//
// Each CTA (512 threads) takes systems from an atomic work queue (the caller
// passes them largest first, so the tail of the launch is short) and, per
// system:
//   * copies A (FP64) into a factor buffer in the factorization type T
//     (float: FP32 factors + FP64 refinement; double: plain FP64 LU), with
//     ||A||_inf on the way;
//   * factors it with a blocked right-looking LU with partial pivoting:
//     panels of NB columns held in shared memory (one thread per row), the
//     panel's interchanges on the other columns, U12 by substitution and the
//     trailing update A22 -= L21 U12 with one thread per column;
//   * solves with the factors applied in FP64 (32-row blocks: one warp per
//     diagonal block, all threads for the updates), then refines in FP64:
//     r = b - A x, d = U^-1 L^-1 P r, x += d, until the normwise backward
//     error ||r|| / (||A|| ||x|| + ||b||) <= tol, the refinement stalls
//     (less than a factor 2 gained per correction) or max_iter corrections.
// With FP32 factors, a second launch of the same kernel with FP64 factors
// takes only the systems whose refinement did not converge (ill-conditioned
// ones); it skips every other system at the cost of one queue step.
// The panel width NB is taken per system from a per-size-bucket table chosen
// by the autotuner (16 or 32 for FP32; 16 for FP64).
// Per-system outputs: status (corrections used, or -(info) for an exactly
// singular U) and the final backward error.
#include <cuda_runtime.h>

#include <climits>
#include <cstdint>

#include "common.cuh"

namespace b200la
{
namespace
{
constexpr int kBT      = 512;  // threads per CTA = largest order handled
constexpr int kBMaxN   = 512;
constexpr int kBBuckets = 8;   // size buckets of 64
// status of a system whose refinement stalled or ran out of corrections; the
// FP64 pass picks these up.  Systems finished by that pass get 1000 + k.
constexpr int32_t kNotConverged = -1000000;
constexpr int32_t kEscalated    = 1000;

template <typename T> struct BatchTraits;
template <> struct BatchTraits<float>
{
    static constexpr int kMaxNB = 32;
};
template <> struct BatchTraits<double>
{
    static constexpr int kMaxNB = 16;
};

template <typename T> constexpr size_t batched_smem()
{
    constexpr int NB = BatchTraits<T>::kMaxNB;
    // panel [512][NB+1] + U12 staging [NB][512] + FP64 vectors (y, r, x) [3][512]
    // + pivots and row permutation [2][512]
    return sizeof(T) * ((size_t)kBMaxN * (NB + 1) + (size_t)NB * kBMaxN) + sizeof(double) * 3 * kBMaxN +
           sizeof(int) * 2 * kBMaxN;
}

__device__ __forceinline__ void bat_best(double& key, int& row, double* red_key, int* red_row)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        const double ok = __shfl_down_sync(0xffffffffu, key, off);
        const int    orow = __shfl_down_sync(0xffffffffu, row, off);
        if (ok > key || (ok == key && orow < row))
        {
            key = ok;
            row = orow;
        }
    }
    if (lane == 0)
    {
        red_key[warp] = key;
        red_row[warp] = row;
    }
    __syncthreads();
    if (threadIdx.x < 32)
    {
        key = threadIdx.x < (kBT / 32) ? red_key[threadIdx.x] : -2.0;
        row = threadIdx.x < (kBT / 32) ? red_row[threadIdx.x] : INT_MAX;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            const double ok = __shfl_down_sync(0xffffffffu, key, off);
            const int    orow = __shfl_down_sync(0xffffffffu, row, off);
            if (ok > key || (ok == key && orow < row))
            {
                key = ok;
                row = orow;
            }
        }
        if (threadIdx.x == 0)
        {
            red_key[kBT / 32] = key;
            red_row[kBT / 32] = row;
        }
    }
    __syncthreads();
    key = red_key[kBT / 32];
    row = red_row[kBT / 32];
}

// y <- T^-1 y for the unit-lower (upper = false) or upper triangle of the
// n x n factor f (row-major), y in shared memory (FP64).  32-row blocks.
template <typename T>
__device__ void bat_trsv(const T* __restrict__ f, int n, bool upper, double* y)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nblk = (n + 31) / 32;
    for (int bi = 0; bi < nblk; ++bi)
    {
        const int b  = upper ? nblk - 1 - bi : bi;
        const int b0 = b * 32;
        const int bw = min(32, n - b0);
        if (warp == 0)
        {
            double v = lane < bw ? y[b0 + lane] : 0.0;
            if (!upper)
            {
                for (int j = 0; j < bw; ++j)
                {
                    const double yj = __shfl_sync(0xffffffffu, v, j);
                    if (lane > j && lane < bw)
                    {
                        v = fma(-(double)f[(size_t)(b0 + lane) * n + b0 + j], yj, v);
                    }
                }
            }
            else
            {
                for (int j = bw - 1; j >= 0; --j)
                {
                    if (lane == j)
                    {
                        v = v / (double)f[(size_t)(b0 + j) * n + b0 + j];
                    }
                    const double yj = __shfl_sync(0xffffffffu, v, j);
                    if (lane < j)
                    {
                        v = fma(-(double)f[(size_t)(b0 + lane) * n + b0 + j], yj, v);
                    }
                }
            }
            if (lane < bw)
            {
                y[b0 + lane] = v;
            }
        }
        __syncthreads();
        // update the rows not yet solved
        const int i = threadIdx.x;
        if (i < n && (upper ? i < b0 : i >= b0 + bw))
        {
            const T* row = f + (size_t)i * n + b0;
            double   s   = 0.0;
            for (int j = 0; j < bw; ++j)
            {
                s = fma((double)row[j], y[b0 + j], s);
            }
            y[i] -= s;
        }
        __syncthreads();
    }
}

template <typename T>
__global__ void __launch_bounds__(kBT, 1) k_batched_gesv(int count, const int32_t* __restrict__ sizes,
    const int64_t* __restrict__ offa, const int64_t* __restrict__ offv, const int32_t* __restrict__ order,
    const double* __restrict__ A, const double* __restrict__ B, double* __restrict__ X, T* __restrict__ F,
    int max_iter, double tol, int fallback_only, const int32_t* __restrict__ nb_table, int32_t* __restrict__ status,
    double* __restrict__ berr, int32_t* __restrict__ queue)
{
    constexpr int MNB = BatchTraits<T>::kMaxNB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T(*P)[MNB + 1] = reinterpret_cast<T(*)[MNB + 1]>(smem_raw);                       // [512][MNB+1]
    T* U           = reinterpret_cast<T*>(smem_raw + sizeof(T) * kBMaxN * (MNB + 1));  // [MNB][512]
    double* yv     = reinterpret_cast<double*>(smem_raw + sizeof(T) * ((size_t)kBMaxN * (MNB + 1) + (size_t)MNB * kBMaxN));
    double* rv     = yv + kBMaxN;
    double* xv     = rv + kBMaxN;
    int*    piv    = reinterpret_cast<int*>(xv + kBMaxN);  // 0-based pivot row of each step
    int*    perm   = piv + kBMaxN;                          // final row permutation
    __shared__ double red_key[kBT / 32 + 1];
    __shared__ int    red_row[kBT / 32 + 1];
    __shared__ int    s_sys, s_first_zero;
    __shared__ unsigned long long s_norm[3];  // ||A||, max|r|, max|x|
    __shared__ int    spiv[MNB];

    const int tid = threadIdx.x;
    for (;;)
    {
        if (tid == 0)
        {
            s_sys = atomicAdd(queue, 1);
        }
        __syncthreads();
        const int q = s_sys;
        if (q >= count)
        {
            return;
        }
        const int     sys = order != nullptr ? order[q] : q;
        if (fallback_only && status[sys] != kNotConverged)
        {
            __syncthreads();
            continue;  // converged (or exactly singular) in the first pass
        }
        const int     n   = sizes[sys];
        const double* a   = A + offa[sys];
        T*            f   = F + offa[sys];
        const double* b   = B + offv[sys];
        double*       x   = X + offv[sys];
        int           NB  = nb_table[min((n - 1) / 64, kBBuckets - 1)];
        NB                = NB < 1 ? 1 : (NB > MNB ? MNB : NB);
        if (tid == 0)
        {
            s_first_zero = -1;
            s_norm[0] = s_norm[1] = s_norm[2] = 0ull;
        }
        __syncthreads();
        // ---- A -> F in T, ||A||_inf (a warp per row)
        {
            const int lane = tid & 31, warp = tid >> 5;
            for (int i = warp; i < n; i += kBT / 32)
            {
                double s = 0.0;
                for (int j = lane; j < n; j += 32)
                {
                    const double v     = a[(size_t)i * n + j];
                    f[(size_t)i * n + j] = (T)v;
                    s += fabs(v);
                }
#pragma unroll
                for (int off = 16; off > 0; off >>= 1)
                {
                    s += __shfl_down_sync(0xffffffffu, s, off);
                }
                if (lane == 0)
                {
                    atomicMax(&s_norm[0], (unsigned long long)__double_as_longlong(s));
                }
            }
        }
        __syncthreads();
        // ---- blocked LU with partial pivoting
        for (int k = 0; k < n; k += NB)
        {
            const int w = min(NB, n - k);
            const int R = n - k;
            // panel rows [k, n) x columns [k, k+w): one thread per row
            if (tid < R)
            {
                for (int c = 0; c < w; ++c)
                {
                    P[tid][c] = f[(size_t)(k + tid) * n + k + c];
                }
            }
            __syncthreads();
            for (int jj = 0; jj < w; ++jj)
            {
                double key = -2.0;
                int    row = INT_MAX;
                if (tid >= jj && tid < R)
                {
                    const T   v   = P[tid][jj];
                    const bool nan = v != v;
                    key = tid == jj ? (nan ? __longlong_as_double(0x7ff0000000000000ll) : (double)fabs(v))
                                    : (nan ? -1.0 : (double)fabs(v));
                    row = tid;
                }
                bat_best(key, row, red_key, red_row);
                const int p = row;
                if (tid == 0)
                {
                    spiv[jj] = p;
                }
                if (p != jj && tid < w)
                {
                    const T t  = P[jj][tid];
                    P[jj][tid] = P[p][tid];
                    P[p][tid]  = t;
                }
                __syncthreads();
                const T d = P[jj][jj];
                if (d == T(0))
                {
                    if (tid == 0 && s_first_zero < 0)
                    {
                        s_first_zero = k + jj;
                    }
                }
                else if (tid > jj && tid < R)
                {
                    const T l = P[tid][jj] / d;
                    P[tid][jj] = l;
                    for (int c = jj + 1; c < w; ++c)
                    {
                        P[tid][c] = fma(-l, P[jj][c], P[tid][c]);
                    }
                }
                __syncthreads();
            }
            // panel back to F; interchanges on the other columns
            if (tid < R)
            {
                for (int c = 0; c < w; ++c)
                {
                    f[(size_t)(k + tid) * n + k + c] = P[tid][c];
                }
            }
            for (int col = tid; col < n; col += kBT)
            {
                if (col >= k && col < k + w)
                {
                    continue;
                }
                for (int jj = 0; jj < w; ++jj)
                {
                    const int p = spiv[jj];
                    if (p != jj)
                    {
                        T* r1     = f + (size_t)(k + jj) * n + col;
                        T* r2     = f + (size_t)(k + p) * n + col;
                        const T t = *r1;
                        *r1       = *r2;
                        *r2       = t;
                    }
                }
            }
            if (tid == 0)
            {
                for (int jj = 0; jj < w; ++jj)
                {
                    piv[k + jj] = k + spiv[jj];
                }
            }
            __syncthreads();
            const int rest = n - k - w;
            if (rest > 0)
            {
                // U12 = L11^-1 A12, one thread per column, staged in U
                const int c = k + w + tid;
                if (tid < rest)
                {
                    T u[MNB];
#pragma unroll
                    for (int i = 0; i < MNB; ++i)
                    {
                        u[i] = i < w ? f[(size_t)(k + i) * n + c] : T(0);
                    }
#pragma unroll
                    for (int i = 1; i < MNB; ++i)
                    {
                        if (i < w)
                        {
#pragma unroll
                            for (int pp = 0; pp < i; ++pp)
                            {
                                u[i] = fma(-P[i][pp], u[pp], u[i]);
                            }
                        }
                    }
#pragma unroll
                    for (int i = 0; i < MNB; ++i)
                    {
                        if (i < w)
                        {
                            f[(size_t)(k + i) * n + c] = u[i];
                            U[i * kBMaxN + tid]      = u[i];
                        }
                    }
                }
                __syncthreads();
                // A22 -= L21 U12, one thread per column; L21 rows broadcast from P
                if (tid < rest)
                {
                    T u[MNB];
#pragma unroll
                    for (int i = 0; i < MNB; ++i)
                    {
                        u[i] = i < w ? U[i * kBMaxN + tid] : T(0);
                    }
                    for (int r = 0; r < rest; ++r)
                    {
                        const T* lrow = P[w + r];
                        T        acc  = T(0);
#pragma unroll
                        for (int i = 0; i < MNB; ++i)
                        {
                            if (i < w)
                            {
                                acc = fma(lrow[i], u[i], acc);
                            }
                        }
                        T* cell = f + (size_t)(k + w + r) * n + c;
                        *cell   = *cell - acc;
                    }
                }
                __syncthreads();
            }
        }
        if (s_first_zero >= 0)
        {
            if (tid == 0)
            {
                status[sys] = -(s_first_zero + 1);
                berr[sys]   = INFINITY;
            }
            __syncthreads();
            continue;
        }
        // row permutation of the pivot sequence (one thread, n <= 512 swaps)
        if (tid == 0)
        {
            for (int i = 0; i < n; ++i)
            {
                perm[i] = i;
            }
            for (int i = 0; i < n; ++i)
            {
                const int t = piv[i];
                const int v = perm[i];
                perm[i]     = perm[t];
                perm[t]     = v;
            }
        }
        __syncthreads();
        // ---- solve and refine in FP64
        double anorm, bnorm = 0.0;
        {
            const unsigned long long an = s_norm[0];
            anorm = __longlong_as_double((long long)an);
        }
        if (tid < n)
        {
            xv[tid] = 0.0;
            rv[tid] = b[tid];
        }
        __syncthreads();
        for (int i = 0; i < n; ++i)
        {
            bnorm = fmax(bnorm, fabs(rv[i]));
        }
        int    it       = 0;
        double eta      = INFINITY;
        double eta_prev = INFINITY;
        bool   done     = false;
        for (;;)
        {
            // d = U^-1 L^-1 P r
            if (tid < n)
            {
                yv[tid] = rv[perm[tid]];
            }
            __syncthreads();
            bat_trsv<T>(f, n, false, yv);
            bat_trsv<T>(f, n, true, yv);
            if (tid < n)
            {
                xv[tid] += yv[tid];
            }
            if (tid == 0)
            {
                s_norm[1] = 0ull;
                s_norm[2] = 0ull;
            }
            __syncthreads();
            // r = b - A x (a warp per row), max|r|, max|x|
            {
                const int lane = tid & 31, warp = tid >> 5;
                for (int i = warp; i < n; i += kBT / 32)
                {
                    double s = 0.0;
                    for (int j = lane; j < n; j += 32)
                    {
                        s = fma(a[(size_t)i * n + j], xv[j], s);
                    }
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1)
                    {
                        s += __shfl_down_sync(0xffffffffu, s, off);
                    }
                    if (lane == 0)
                    {
                        const double r = b[i] - s;
                        rv[i]          = r;
                        atomicMax(&s_norm[1], (unsigned long long)__double_as_longlong(fabs(r)));
                        atomicMax(&s_norm[2], (unsigned long long)__double_as_longlong(fabs(xv[i])));
                    }
                }
            }
            __syncthreads();
            const double rn  = __longlong_as_double((long long)s_norm[1]);
            const double xn  = __longlong_as_double((long long)s_norm[2]);
            const double den = anorm * xn + bnorm;
            eta              = den > 0 ? rn / den : 0.0;
            ++it;
            if (eta <= tol)
            {
                done = true;
                break;
            }
            // out of corrections, not a number, or stalled (less than a
            // factor 2 gained after the first correction)
            if (it > max_iter || !(eta == eta) || (it > 2 && eta > 0.5 * eta_prev))
            {
                break;
            }
            eta_prev = eta;
            __syncthreads();
        }
        if (tid < n)
        {
            x[tid] = xv[tid];
        }
        if (tid == 0)
        {
            status[sys] = done ? (fallback_only ? kEscalated + it - 1 : it - 1) : kNotConverged;
            berr[sys]   = eta;
        }
        __syncthreads();
    }
}

template <typename T> int set_batched_attr()
{
    static bool done[64] = {};
    int         dev      = 0;
    B200LA_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && done[dev])
        return B200LA_SUCCESS;
    B200LA_CUDA(cudaFuncSetAttribute(k_batched_gesv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)batched_smem<T>()));
    if (dev >= 0 && dev < 64)
        done[dev] = true;
    return B200LA_SUCCESS;
}
}  // namespace
int require_sm100();
}  // namespace b200la

using namespace b200la;

extern "C" {

B200LA_API size_t b200la_dgesv_batched_workspace_size(int64_t total_a, int64_t total_v, int precision)
{
    if (total_a <= 0 || total_v <= 0)
        return 0;
    Arena a;
    a.next<int32_t>(64);  // queue counters of the two passes
    // factors: FP32 in the first pass; the FP64 pass for systems whose FP32
    // refinement stalled reuses the same buffer as FP64
    a.next<double>((size_t)total_a);
    return a.size();
}

B200LA_API int b200la_dgesv_batched(int64_t count, const int32_t* sizes, const int64_t* offsets_a,
    const int64_t* offsets_v, const int32_t* order, const double* a, const double* b, double* x,
    int64_t total_a, int64_t total_v, int precision, const int32_t* nb_table, int max_iterations,
    double tolerance, int32_t* status, double* backward_error, void* workspace, size_t workspace_bytes,
    void* stream)
{
    if (count <= 0 || count > INT_MAX / 2 || !sizes || !offsets_a || !offsets_v || !a || !b || !x || !status ||
        !backward_error || !nb_table)
        return set_error(B200LA_INVALID_ARGUMENT, "dgesv_batched: null pointer or bad count");
    if (precision != B200LA_PREC_FP32 && precision != B200LA_PREC_FP64)
        return set_error(B200LA_NOT_SUPPORTED, "dgesv_batched: precision must be FP32 (refined) or FP64");
    if (max_iterations < 0 || !(tolerance > 0))
        return set_error(B200LA_INVALID_ARGUMENT, "dgesv_batched: invalid refinement options");
    const size_t need = b200la_dgesv_batched_workspace_size(total_a, total_v, precision);
    if (workspace == nullptr || workspace_bytes < need)
        return set_error(B200LA_WORKSPACE_TOO_SMALL, "dgesv_batched: workspace too small (%zu < %zu)",
            workspace_bytes, need);
    int rc = require_sm100();
    if (rc != B200LA_SUCCESS)
        return rc;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Arena        ar(workspace, workspace_bytes);
    int32_t*     queue = ar.next<int32_t>(64);
    const int grid = device_sm_count();
    B200LA_CUDA(cudaMemsetAsync(queue, 0, sizeof(int32_t) * 2, s));
    void* fbuf = ar.next<double>((size_t)total_a);
    if ((rc = set_batched_attr<double>()) != B200LA_SUCCESS)
        return rc;
    if (precision == B200LA_PREC_FP64)
    {
        prof_begin(KC_BATCHED, s);
        k_batched_gesv<double><<<grid, kBT, batched_smem<double>(), s>>>((int)count, sizes, offsets_a, offsets_v,
            order, a, b, x, (double*)fbuf, max_iterations, tolerance, 0, nb_table, status, backward_error, queue);
        prof_end(KC_BATCHED, s);
    }
    else
    {
        if ((rc = set_batched_attr<float>()) != B200LA_SUCCESS)
            return rc;
        prof_begin(KC_BATCHED, s);
        k_batched_gesv<float><<<grid, kBT, batched_smem<float>(), s>>>((int)count, sizes, offsets_a, offsets_v,
            order, a, b, x, (float*)fbuf, max_iterations, tolerance, 0, nb_table, status, backward_error, queue);
        prof_end(KC_BATCHED, s);
        B200LA_LAUNCH_CHECK();
        // FP64 factors for the systems whose FP32 refinement stalled
        prof_begin(KC_BATCHED, s);
        k_batched_gesv<double><<<grid, kBT, batched_smem<double>(), s>>>((int)count, sizes, offsets_a, offsets_v,
            order, a, b, x, (double*)fbuf, 3, tolerance, 1, nb_table, status, backward_error, queue + 1);
        prof_end(KC_BATCHED, s);
    }
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}
}
