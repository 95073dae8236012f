// Cholesky factorization (lower; upper by transposition) for the Cholesky
// modes of linear_solver and for cholesky_decomposition, bit-identical to the
// reference's NATIVE code: src/matrix_operation/cpu/native/
// cholesky_decomposition_native.cpp (cholesky_decomposition_blocked_lower,
// block 64, and cholesky_decomposition_scalar_impl for the diagonal block).
//
// Rounding.  Every dot product of the reference (cholesky_dot, `sum += x*y`
// from zero) is compiled by g++ -O3 with AVX2+FMA into full vectors of
// products, each product rounded, added to the sum one by one in order, then
// one half vector the same way, and the last products fused into the sum;
// the pivot's dot(a_i, a_i, i) in double has no half vector
// (chol_rend_pivot).
// chol_dot reproduces that with separately rounded multiplies and adds
// (__dmul_rn / __dadd_rn cannot be contracted), so these updates run on the
// FP64 (or FP32) pipe, not the tensor cores, whose fused products would give
// other bits.  Per block k (bs = 64 rows, the last one shorter):
//   k_chol_diag   the diagonal block, one CTA, column by column: every dot
//                 product of the reference is accumulated term by term in
//                 its order as the columns it needs are finished; a
//                 non-positive pivot leaves the block exactly as the
//                 reference leaves it when it returns there;
//   k_chol_trsm   A21 = A21 L11^-T, a thread per row, term by term likewise,
//                 and zeros right of the diagonal block in its rows;
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

// The number of leading terms chol_dot rounds separately for a dot of len
// terms (the rest are fused): whole vectors, then one half vector if the
// remainder holds one.
template <typename T> __host__ __device__ constexpr int chol_rend(int len)
{
    constexpr int vec  = 32 / (int)sizeof(T);
    constexpr int half = vec / 2;
    const int     main = len >= vec ? (len / vec) * vec : 0;
    return main + (len - main >= half ? half : 0);
}

// s += x y in the reference's rounding for term `term` of a dot of `len`
// terms (both compile-time after unrolling).
template <typename T> __device__ __forceinline__ T chol_term(T s, T x, T y, int term, int len)
{
    return term < chol_rend<T>(len) ? rn_add(s, rn_mul(x, y)) : fma(x, y, s);
}

// The pivot's reduction dot(a_i, a_i, i) is compiled differently in the
// reference build (the same row as both operands): for double, whole vectors
// of 4 products rounded and the rest (up to 3) fused, no half vector; for
// float as chol_rend.  Established by probing the reference build one call
// site and length at a time.
template <typename T> __host__ __device__ constexpr int chol_rend_pivot(int len)
{
    return sizeof(T) == 8 ? (len / 4) * 4 : chol_rend<T>(len);
}

// Term `term` of row i's sum s_ij (dot of length j) in the diagonal block:
// the pivot's pattern when j == i (is_pivot, known at run time), the common
// one otherwise.  The two differ only for a few (term, j) pairs, which are
// known at compile time after unrolling; only those carry a select.
template <typename T>
__device__ __forceinline__ T chol_term_blk(T s, T x, T y, int term, int len, bool is_pivot)
{
    if (term >= chol_rend_pivot<T>(len) && term < chol_rend<T>(len))
    {
        return is_pivot ? fma(x, y, s) : rn_add(s, rn_mul(x, y));
    }
    return chol_term(s, x, y, term, len);
}

// Dynamic shared memory of the kernels below (padded rows of kCholNB + 1).
constexpr int kCholTrsmRows = 128;  // rows of A21 per k_chol_trsm CTA
template <typename T> constexpr size_t chol_smem_bytes() { return sizeof(T) * 2 * kCholNB * (kCholNB + 1); }
template <typename T> constexpr size_t chol_trsm_smem_bytes()
{
    return sizeof(T) * (kCholNB + kCholTrsmRows) * (kCholNB + 1);
}

// Element-wise asynchronous copies global -> shared (zero-filled when not
// valid), so a CTA issues all of its staging loads before it waits.
template <int BYTES> __device__ __forceinline__ void chol_cp_async(void* dst, const void* src, bool valid)
{
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(src), "n"(BYTES),
        "r"(valid ? BYTES : 0)
        : "memory");
}
__device__ __forceinline__ void chol_cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void chol_cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// The diagonal block [k, k+bs)^2, one CTA of kCholNB threads (thread i: row
// i).  Column-by-column (right-looking): at column c the pivot is
// sqrt(a_cc - s_cc), rows below get l_ic = (a_ic - s_ic) / l_cc, then every
// row adds its term c to s_ij (j > c).  Each s_ij therefore receives the
// terms l_i0 l_j0, l_i1 l_j1, ... in the reference's order and rounding (its
// row-by-row loop computes the same dot product from zero), so the factor
// is the same bits, with a critical path of bs steps instead of one dot
// product per entry.  The partial sums live in registers (s[j], row tid).
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
    for (int e = tid; e < kCholNB * kCholNB; e += kCholNB)
    {
        const int r = e / kCholNB, c = e % kCholNB;
        if (r < bs && c < bs)
        {
            chol_cp_async<sizeof(T)>(&blk[r][c], A + (int64_t)(k + r) * n + k + c, true);
        }
    }
    chol_cp_commit();
    if (tid == 0)
    {
        fail = -1;
    }
    chol_cp_wait<0>();
    __syncthreads();
    for (int e = tid; e < bs * bs; e += kCholNB)
    {
        const int r = e / bs, c = e - (e / bs) * bs;
        orig[r][c]  = blk[r][c];
    }
    T s[kCholNB];
#pragma unroll
    for (int j = 0; j < kCholNB; ++j)
    {
        s[j] = T(0);
    }
    __syncthreads();
#pragma unroll
    for (int c = 0; c < kCholNB; ++c)
    {
        if (c >= bs)
        {
            break;
        }
        if (tid == c)
        {
            const T d = rn_sub(blk[c][c], s[c]);
            if (d <= T(0))
            {
                fail = c;
            }
            else
            {
                blk[c][c] = chol_sqrt(d);
            }
        }
        __syncthreads();
        if (fail >= 0)
        {
            break;
        }
        const bool below = tid > c && tid < bs;
        if (below)
        {
            blk[tid][c] = rn_sub(blk[tid][c], s[c]) / blk[c][c];
        }
        __syncthreads();
        if (below)
        {
            const T v = blk[tid][c];
#pragma unroll
            for (int j = c + 1; j < kCholNB; ++j)
            {
                if (j <= tid)
                {
                    s[j] = chol_term_blk(s[j], v, blk[j][c], c, j, j == tid);
                }
            }
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

// Failure gate of the block that ends at row `limit`: a device error, or a
// non-positive pivot found before `limit`.  A later block's diagonal kernel
// may run concurrently (look-ahead) and set a later pivot; that one does not
// stop this block's work, as in the reference, which finished this block
// before it reached the failing one.
__device__ __forceinline__ bool chol_gated(const DeviceStatus* st, int64_t limit)
{
    if (ld_volatile_i32(&st->error) != 0)
    {
        return true;
    }
    const int64_t f = *reinterpret_cast<const volatile int64_t*>(&st->first_zero);
    return f >= 0 && f < limit;
}

// A21 = A21 L11^-T for a full block (bs = kCholNB): rows [k+64, n), a
// thread per row, kCholTrsmRows rows per CTA staged in shared memory with
// L11.  Row r, column c: l_rc = (a_rc - s_rc) / l_cc, then the row's later
// partial sums s_rj (j > c, registers) get the term l_rc l_jc: the
// reference's dot products term by term, in its order and rounding.  The
// CTAs also clear the block's rows right of it (A[k..k+64)[k+64..n)),
// kCholTrsmRows columns each, as the reference does once the block is
// factored.
template <typename T>
__global__ void __launch_bounds__(kCholTrsmRows) k_chol_trsm(T* __restrict__ A, int n, int k, const DeviceStatus* st)
{
    extern __shared__ __align__(16) unsigned char chol_smem[];
    T(*l11)[kCholNB + 1]  = reinterpret_cast<T(*)[kCholNB + 1]>(chol_smem);
    T(*rows)[kCholNB + 1] = l11 + kCholNB;
    if (chol_gated(st, (int64_t)k + kCholNB))
    {
        return;
    }
    const int tid = threadIdx.x;
    const int r0  = k + kCholNB + blockIdx.x * kCholTrsmRows;
    const int nr  = min(kCholTrsmRows, n - r0);
    for (int e = tid; e < kCholNB * kCholNB; e += kCholTrsmRows)
    {
        const int r = e / kCholNB, c = e % kCholNB;
        chol_cp_async<sizeof(T)>(&l11[r][c], A + (int64_t)(k + r) * n + k + c, true);
    }
    for (int e = tid; e < nr * kCholNB; e += kCholTrsmRows)
    {
        const int r = e / kCholNB, c = e % kCholNB;
        chol_cp_async<sizeof(T)>(&rows[r][c], A + (int64_t)(r0 + r) * n + k + c, true);
    }
    chol_cp_commit();
    for (int e = tid; e < kCholNB * nr; e += kCholTrsmRows)
    {
        const int r = e / nr, c = e - (e / nr) * nr;
        A[(int64_t)(k + r) * n + r0 + c] = T(0);
    }
    chol_cp_wait<0>();
    __syncthreads();
    if (tid < nr)
    {
        T* row = &rows[tid][0];
        T  s[kCholNB];
#pragma unroll
        for (int j = 0; j < kCholNB; ++j)
        {
            s[j] = T(0);
        }
#pragma unroll
        for (int c = 0; c < kCholNB; ++c)
        {
            const T v = rn_sub(row[c], s[c]) / l11[c][c];
            row[c]    = v;
#pragma unroll
            for (int j = c + 1; j < kCholNB; ++j)
            {
                s[j] = chol_term(s[j], v, l11[j][c], c, j);
            }
        }
    }
    __syncthreads();
    for (int e = tid; e < nr * kCholNB; e += kCholTrsmRows)
    {
        const int r = e / kCholNB, c = e % kCholNB;
        A[(int64_t)(r0 + r) * n + k + c] = rows[r][c];
    }
}

// Trailing lower triangle t_ij -= dot(a21_i, a21_j, 64), i >= j, over
// [k+64, n)^2 for a full block.  With 64 terms every product is rounded and
// added in order (chol_dot's whole-vector part covers them all).  CTA tile
// 64 x 64 of 256 threads with 4 x 4 entries each.  The tiles on or below the
// diagonal are launched in one of three sets: all of them (blockIdx.x
// enumerates the triangle row by row), the first tile column only (the
// columns the next block factors), or the rest.  The two A21 slices arrive
// in shared memory by cp.async in two halves of 32 columns, the second
// landing while the first is multiplied; the C tile is prefetched into L2.
constexpr int kSyrkTile = 64;
enum Chol_syrk_set
{
    kSyrkAll   = 0,
    kSyrkFirst = 1,
    kSyrkRest  = 2
};
static_assert(chol_rend<double>(kCholNB) == kCholNB && chol_rend<float>(kCholNB) == kCholNB,
    "a full block's trailing dot products round every product");

__device__ __forceinline__ void chol_tri_tile(int b, int& I, int& J)
{
    int i = (int)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
    while ((int64_t)i * (i + 1) / 2 > b)
    {
        --i;
    }
    while ((int64_t)(i + 1) * (i + 2) / 2 <= b)
    {
        ++i;
    }
    I = i;
    J = b - i * (i + 1) / 2;
}

template <typename T>
__global__ void __launch_bounds__(256) k_chol_syrk(T* __restrict__ A, int n, int k, int set, const DeviceStatus* st)
{
    extern __shared__ __align__(16) unsigned char chol_smem[];
    T(*ai)[kCholNB + 1] = reinterpret_cast<T(*)[kCholNB + 1]>(chol_smem);
    T(*aj)[kCholNB + 1] = ai + kSyrkTile;
    if (chol_gated(st, (int64_t)k + kCholNB))
    {
        return;
    }
    int I, J;
    if (set == kSyrkFirst)
    {
        I = blockIdx.x;
        J = 0;
    }
    else
    {
        chol_tri_tile(blockIdx.x, I, J);
        if (set == kSyrkRest)
        {
            ++I;
            ++J;
        }
    }
    const int base = k + kCholNB;
    const int i0 = base + I * kSyrkTile, j0 = base + J * kSyrkTile;
    const int tid = threadIdx.x;
    // C tile into L2: 64 rows of 64 entries, 128-byte lines
    constexpr int lines = kSyrkTile * (int)sizeof(T) / 128;
    if (tid < kSyrkTile * lines)
    {
        const int r = tid / lines, l = tid - (tid / lines) * lines;
        if (i0 + r < n)
        {
            const T* p = A + (int64_t)(i0 + r) * n + j0 + l * (128 / (int)sizeof(T));
            asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
        }
    }
    // the A21 slices, two halves of 32 columns (8 elements per thread per
    // slice and half); rows past n read as zeros
#pragma unroll
    for (int h = 0; h < 2; ++h)
    {
#pragma unroll
        for (int q = 0; q < 8; ++q)
        {
            const int  e  = tid + 256 * q;
            const int  r  = e >> 5, c = (e & 31) + 32 * h;
            const bool vi = i0 + r < n, vj = j0 + r < n;
            chol_cp_async<sizeof(T)>(&ai[r][c], A + (int64_t)(vi ? i0 + r : base) * n + k + c, vi);
            chol_cp_async<sizeof(T)>(&aj[r][c], A + (int64_t)(vj ? j0 + r : base) * n + k + c, vj);
        }
        chol_cp_commit();
    }
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
#pragma unroll
    for (int h = 0; h < 2; ++h)
    {
        if (h == 0)
        {
            chol_cp_wait<1>();
        }
        else
        {
            chol_cp_wait<0>();
        }
        __syncthreads();
#pragma unroll 8
        for (int p = 32 * h; p < 32 * h + 32; ++p)
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
                    acc[a][b] = rn_add(acc[a][b], rn_mul(x[a], y[b]));
                }
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
            if (j <= i)
            {
                T* p = A + (int64_t)i * n + j;
                *p   = rn_sub(*p, acc[a][b]);
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
