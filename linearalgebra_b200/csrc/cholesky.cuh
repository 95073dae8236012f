// Cholesky factorization (lower; upper by transposition) for the Cholesky
// modes of linear_solver and for cholesky_decomposition, bit-identical to the
// reference's NATIVE code: src/matrix_operation/cpu/native/
// cholesky_decomposition_native.cpp (cholesky_decomposition_blocked_lower,
// block 64, and cholesky_decomposition_scalar_impl for the diagonal block).
//
// Rounding.  Every dot product of the reference (cholesky_dot, `sum += x*y`
// from zero) is compiled by g++ -O3 with AVX2+FMA into full vectors of
// products, each product rounded, added to the sum one by one in order, then
// one half vector the same way, and the last products fused into the sum.
// chol_dot reproduces that with separately rounded multiplies and adds
// (__dmul_rn / __dadd_rn cannot be contracted), so these updates run on the
// FP64 (or FP32) pipe, not the tensor cores, whose fused products would give
// other bits.  Per block k (bs = 64 rows, the last one shorter):
//   k_chol_diag   the diagonal block, row by row in the reference's order; a
//                 one-CTA wavefront computes entry (i, j) at step i + j (it
//                 needs row i's entries left of j and the finished row j);
//                 a non-positive pivot leaves the block exactly as the
//                 reference leaves it when it returns there;
//   k_chol_zero   zeros right of the diagonal block in its rows;
//   k_chol_trsm   A21 = A21 L11^-T, row by row (a thread per row);
//   k_chol_syrk   the trailing lower triangle, t_ij -= dot(a21_i, a21_j, 64).
// The first non-positive pivot goes to the status block (first_zero, then
// info = first_zero + 1) and gates every later kernel, as the reference
// returns at once.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"
#include "solve_kernels.cuh"

namespace b200la
{

constexpr int kCholNB = 64;

template <typename T> __device__ __forceinline__ T rn_mul(T a, T b);
template <> __device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
template <> __device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
template <typename T> __device__ __forceinline__ T rn_add(T a, T b);
template <> __device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
template <> __device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
template <typename T> __device__ __forceinline__ T rn_sub(T a, T b);
template <> __device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }
template <> __device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }

// The reference build's dot product (see the header comment): x, y with
// element strides 1, len terms.
template <typename T> __device__ __forceinline__ T chol_dot(const T* x, const T* y, int len)
{
    constexpr int vec  = 32 / (int)sizeof(T);
    constexpr int half = vec / 2;
    const int     main = len >= vec ? (len / vec) * vec : 0;
    T             s    = T(0);
    int           j    = 0;
    for (; j < main; ++j)
    {
        s = rn_add(s, rn_mul(x[j], y[j]));
    }
    if (len - j >= half)
    {
#pragma unroll
        for (int q = 0; q < half; ++q, ++j)
        {
            s = rn_add(s, rn_mul(x[j], y[j]));
        }
    }
    for (; j < len; ++j)
    {
        s = fma(x[j], y[j], s);
    }
    return s;
}

template <typename T> __device__ __forceinline__ T chol_sqrt(T v);
template <> __device__ __forceinline__ double chol_sqrt(double v) { return sqrt(v); }
template <> __device__ __forceinline__ float chol_sqrt(float v) { return sqrtf(v); }

// Dynamic shared memory of the kernels below: two padded 64 x 64 tiles.
template <typename T> constexpr size_t chol_smem_bytes() { return sizeof(T) * 2 * kCholNB * (kCholNB + 1); }

// The diagonal block [k, k+bs)^2, one CTA of kCholNB threads (thread i: row i).
template <typename T>
__global__ void __launch_bounds__(kCholNB) k_chol_diag(T* __restrict__ A, int n, int k, int bs, DeviceStatus* st)
{
    extern __shared__ __align__(16) unsigned char chol_smem[];
    T(*blk)[kCholNB + 1]  = reinterpret_cast<T(*)[kCholNB + 1]>(chol_smem);
    T(*orig)[kCholNB + 1] = blk + kCholNB;
    __shared__ int fail;
    if (gated(st))
    {
        return;
    }
    const int tid = threadIdx.x;
    for (int e = tid; e < bs * bs; e += kCholNB)
    {
        const int r = e / bs, c = e - (e / bs) * bs;
        const T   v = A[(int64_t)(k + r) * n + k + c];
        blk[r][c]   = v;
        orig[r][c]  = v;
    }
    if (tid == 0)
    {
        fail = -1;
    }
    __syncthreads();
    for (int t = 0; t <= 2 * (bs - 1); ++t)
    {
        const int i = tid, j = t - tid;
        if (i < bs && j >= 0 && j <= i)
        {
            if (j < i)
            {
                const T s = rn_sub(blk[i][j], chol_dot(&blk[i][0], &blk[j][0], j));
                blk[i][j] = s / blk[j][j];
            }
            else
            {
                const T s = rn_sub(blk[i][i], chol_dot(&blk[i][0], &blk[i][0], i));
                if (s <= T(0))
                {
                    fail = i;  // one diagonal per step
                }
                else
                {
                    blk[i][i] = chol_sqrt(s);
                }
            }
        }
        __syncthreads();
        if (fail >= 0)
        {
            break;
        }
    }
    const int f = fail;
    // write back; on a failure at row f the reference has finished rows < f
    // and row f's entries left of the diagonal, cleared the part above the
    // diagonal of columns <= f, and left everything else as it was
    for (int e = tid; e < bs * bs; e += kCholNB)
    {
        const int r = e / bs, c = e - (e / bs) * bs;
        T         v;
        if (c > r)
        {
            v = (f < 0 || c <= f) ? T(0) : orig[r][c];
        }
        else if (f < 0 || r < f || (r == f && c < r))
        {
            v = blk[r][c];
        }
        else
        {
            v = orig[r][c];
        }
        A[(int64_t)(k + r) * n + k + c] = v;
    }
    if (tid == 0 && f >= 0 && st->first_zero < 0)
    {
        st->first_zero = (int64_t)k + f;
    }
}

// Zeros right of the diagonal block in its rows: A[k..k+bs)[k+bs..n).
template <typename T> __global__ void k_chol_zero(T* __restrict__ A, int n, int k, int bs, const DeviceStatus* gate)
{
    if (gated(gate))
    {
        return;
    }
    const int     w     = n - k - bs;
    const int64_t total = (int64_t)bs * w;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    {
        const int r = (int)(e / w), c = (int)(e - (e / w) * w);
        A[(int64_t)(k + r) * n + k + bs + c] = T(0);
    }
}

// A21 = A21 L11^-T: rows [k+bs, n), thread per row; L11 and the CTA's rows
// staged in shared memory (padded rows).
template <typename T>
__global__ void __launch_bounds__(kCholNB) k_chol_trsm(T* __restrict__ A, int n, int k, int bs,
    const DeviceStatus* gate)
{
    extern __shared__ __align__(16) unsigned char chol_smem[];
    T(*l11)[kCholNB + 1]  = reinterpret_cast<T(*)[kCholNB + 1]>(chol_smem);
    T(*rows)[kCholNB + 1] = l11 + kCholNB;
    if (gated(gate))
    {
        return;
    }
    const int tid = threadIdx.x;
    const int r0  = k + bs + blockIdx.x * kCholNB;
    const int nr  = min(kCholNB, n - r0);
    for (int e = tid; e < bs * bs; e += kCholNB)
    {
        const int r = e / bs, c = e - (e / bs) * bs;
        l11[r][c]   = A[(int64_t)(k + r) * n + k + c];
    }
    for (int e = tid; e < nr * bs; e += kCholNB)
    {
        const int r = e / bs, c = e - (e / bs) * bs;
        rows[r][c]  = A[(int64_t)(r0 + r) * n + k + c];
    }
    __syncthreads();
    if (tid < nr)
    {
        T* row = &rows[tid][0];
        for (int j = 0; j < bs; ++j)
        {
            const T s = rn_sub(row[j], chol_dot(row, &l11[j][0], j));
            row[j]    = s / l11[j][j];
        }
    }
    __syncthreads();
    for (int e = tid; e < nr * bs; e += kCholNB)
    {
        const int r = e / bs, c = e - (e / bs) * bs;
        A[(int64_t)(r0 + r) * n + k + c] = rows[r][c];
    }
}

// Trailing lower triangle t_ij -= dot(a21_i, a21_j, bs), i >= j, over
// [k+bs, n)^2.  CTA tile 64 x 64 (tile (I, J), J <= I; tiles above the
// diagonal exit), 256 threads with 4 x 4 entries each; the two A21 slices in
// shared memory.  With bs = 64 every product is rounded and added in order
// (chol_dot's full-vector part covers all 64 terms).
constexpr int kSyrkTile = 64;
template <typename T>
__global__ void __launch_bounds__(256) k_chol_syrk(T* __restrict__ A, int n, int k, int bs, const DeviceStatus* gate)
{
    extern __shared__ __align__(16) unsigned char chol_smem[];
    T(*ai)[kCholNB + 1] = reinterpret_cast<T(*)[kCholNB + 1]>(chol_smem);
    T(*aj)[kCholNB + 1] = ai + kSyrkTile;
    const int I = blockIdx.y, J = blockIdx.x;
    if (J > I || gated(gate))
    {
        return;
    }
    const int base = k + bs;
    const int i0 = base + I * kSyrkTile, j0 = base + J * kSyrkTile;
    const int tid = threadIdx.x;
    for (int e = tid; e < kSyrkTile * bs; e += 256)
    {
        const int r = e / bs, c = e - (e / bs) * bs;
        ai[r][c]    = i0 + r < n ? A[(int64_t)(i0 + r) * n + k + c] : T(0);
        aj[r][c]    = j0 + r < n ? A[(int64_t)(j0 + r) * n + k + c] : T(0);
    }
    __syncthreads();
    const int tr = tid >> 4, tc = tid & 15;  // rows tr + 16a, columns tc + 16b
    T         acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
    {
#pragma unroll
        for (int b = 0; b < 4; ++b)
        {
            acc[a][b] = T(0);
        }
    }
    constexpr int vec  = 32 / (int)sizeof(T);
    constexpr int half = vec / 2;
    const int     main = bs >= vec ? (bs / vec) * vec : 0;
    const int     rend = main + (bs - main >= half ? half : 0);  // products rounded before [0, rend)
    for (int p = 0; p < bs; ++p)
    {
        T x[4], y[4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
        {
            x[a] = ai[tr + 16 * a][p];
            y[a] = aj[tc + 16 * a][p];
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
        {
#pragma unroll
            for (int b = 0; b < 4; ++b)
            {
                acc[a][b] = p < rend ? rn_add(acc[a][b], rn_mul(x[a], y[b])) : fma(x[a], y[b], acc[a][b]);
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
    {
        const int i = i0 + tr + 16 * a;
        if (i >= n)
        {
            continue;
        }
#pragma unroll
        for (int b = 0; b < 4; ++b)
        {
            const int j = j0 + tc + 16 * b;
            if (j <= i && j < n)
            {
                T* p  = A + (int64_t)i * n + j;
                *p    = rn_sub(*p, acc[a][b]);
            }
        }
    }
}

// Upper factor: U = L^T, the lower part cleared (the reference transposes its
// lower factor in place).  Thread per strictly-lower element.
template <typename T> __global__ void k_chol_to_upper(T* __restrict__ A, int n, const DeviceStatus* gate)
{
    if (gated(gate))
    {
        return;
    }
    const int64_t total = (int64_t)n * n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = (int)(e / n), j = (int)(e - (e / n) * n);
        if (j < i)
        {
            A[(int64_t)j * n + i] = A[(int64_t)i * n + j];
            A[(int64_t)i * n + j] = T(0);
        }
    }
}

}  // namespace b200la
