// One-launch triangular solve for a single right-hand side, op(A) x = b
// with op = identity (lower or upper, unit or not), x overwritten in place.
//
// Row blocks of kTvRows rows are claimed by CTAs through an atomic ticket in
// solve order, so a CTA only ever waits for blocks claimed before its own
// (those CTAs are already running): no deadlock, whatever the residency.
// A CTA accumulates A[block, j] x_j for every solved block j as soon as
// block j's flag is set (bounded wait, 2 s), then solves its diagonal block
// with one warp and publishes x_block with a release store of its flag.
//
// TA is the matrix type (the factors: double or float), TX the vector and
// arithmetic type (double), so the same kernel solves with FP32 LU factors
// in FP64 for iterative refinement.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <chrono>
#include <random>

#include "common.cuh"

namespace b200la
{

constexpr int kTvRows    = 64;
constexpr int kTvThreads = 256;

// Epoch of one k_trsv_blocks launch: the value its flagged words carry.  One
// counter for every caller in the process, never 0 (the value of cleared
// memory), started at a random point so that words left in reused device
// memory by an earlier process do not carry the epochs this one issues.
inline uint32_t tv_next_epoch()
{
    static std::atomic<uint32_t> e{[] {
        std::random_device rd;
        return (uint32_t)rd() ^ (uint32_t)std::chrono::steady_clock::now().time_since_epoch().count();
    }()};
    uint32_t v = e.fetch_add(1) + 1;
    if (v == 0)
    {
        v = e.fetch_add(1) + 1;
    }
    return v;
}

struct TrsvSync
{
    int32_t  ticket;
    int32_t  pad[31];
    uint32_t flags[1];  // [nblocks], cleared per call
};

// Inverses of the kTvRows x kTvRows diagonal blocks of the unit-lower (L)
// and upper (U) triangles of an LU factor, FP64, row-major per block:
// dinv[(2*b + 0)] = L_bb^-1, dinv[(2*b + 1)] = U_bb^-1.  grid (nblocks, 2),
// one thread per column of the inverse (forward/back substitution on e_j).
// A partial last block is padded with the identity.
template <typename TA>
__global__ void __launch_bounds__(kTvRows) k_invert_diag_blocks(const TA* __restrict__ a, int64_t lda, int n,
    double* __restrict__ dinv)
{
    __shared__ double tri[kTvRows][kTvRows + 1];
    const int  blk   = blockIdx.x;
    const bool upper = blockIdx.y == 1;
    const int  r0    = blk * kTvRows;
    const int  br    = min(kTvRows, n - r0);
    const int  j     = threadIdx.x;
    for (int e = j; e < kTvRows * kTvRows; e += kTvRows)
    {
        const int i = e / kTvRows, c = e % kTvRows;
        double    v = (i == c) ? 1.0 : 0.0;
        if (i < br && c < br && (upper ? c >= i : c < i))
        {
            v = (double)a[(int64_t)(r0 + i) * lda + r0 + c];
        }
        tri[i][c] = v;
    }
    __syncthreads();
    // column j of the inverse, built in place in the output block (each
    // thread reads back only its own column)
    double* out = dinv + ((size_t)blk * 2 + (upper ? 1 : 0)) * kTvRows * kTvRows;
    if (!upper)
    {
        for (int i = 0; i < kTvRows; ++i)
        {
            double s = (i == j) ? 1.0 : 0.0;
            for (int p = j; p < i; ++p)
            {
                s = fma(-tri[i][p], out[p * kTvRows + j], s);
            }
            out[i * kTvRows + j] = i < j ? 0.0 : s;
        }
    }
    else
    {
        for (int i = kTvRows - 1; i >= 0; --i)
        {
            double s = (i == j) ? 1.0 : 0.0;
            for (int p = i + 1; p <= j; ++p)
            {
                s = fma(-tri[i][p], out[p * kTvRows + j], s);
            }
            out[i * kTvRows + j] = i > j ? 0.0 : s / tri[i][i];
        }
    }
}

// Flagged publication of a solved block: value i of block b is two 8-byte
// words (low/high halves of the double, each with the call's epoch in the
// high 32 bits), so a reader that sees the epoch in both words has the value.
__device__ __forceinline__ void tv_publish(uint64_t* xll, int blk, int i, double v, uint32_t epoch)
{
    const uint64_t bits = (uint64_t)__double_as_longlong(v);
    const uint64_t w0   = ((uint64_t)epoch << 32) | (bits & 0xffffffffull);
    const uint64_t w1   = ((uint64_t)epoch << 32) | (bits >> 32);
    asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(xll + ((size_t)blk * kTvRows + i) * 2),
        "l"(w0), "l"(w1)
        : "memory");
}
__device__ __forceinline__ bool tv_read(const uint64_t* xll, int blk, int i, uint32_t epoch, double& v)
{
    uint64_t w0, w1;
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(w0), "=l"(w1)
                 : "l"(xll + ((size_t)blk * kTvRows + i) * 2)
                 : "memory");
    if ((uint32_t)(w0 >> 32) != epoch || (uint32_t)(w1 >> 32) != epoch)
    {
        return false;
    }
    v = __longlong_as_double((long long)(((w1 & 0xffffffffull) << 32) | (w0 & 0xffffffffull)));
    return true;
}

// x <- T^-1 x for T the unit-lower (upper = 0) or upper (upper = 1) triangle
// of the factor `a`; with CHOL, of a Cholesky factor L (lower triangle of
// `a`): T = L (upper = 0, non-unit) or T = L^T (upper = 1, read from L's
// rows: a block's off-diagonal tile is the transpose of a 64-column slice of
// the solved rows, loaded row by row, coalesced).  CTA = one 64-row block, claimed by ticket in solve
// order; xll receives the flagged copies of the solved blocks (epoch: a value
// this call's flags carry, never reused).  The diagonal block is applied as
// its inverse from dinv (k_invert_diag_blocks; SUBST = false, the refinement
// solves, whose rounding the refinement corrects) or solved by substitution
// from the block's own triangle (SUBST = true, dinv unused: backward stable,
// for the plain FP64 solve).  wait_ns bounds each wait for another block
// (kWaitLimitNs in the library's own launches).
template <typename TA, bool SUBST = false, bool CHOL = false>
__global__ void __launch_bounds__(kTvThreads) k_trsv_blocks(const TA* __restrict__ a, int64_t lda,
    double* __restrict__ x, int n, int upper, const double* __restrict__ dinv, uint64_t* __restrict__ xll,
    uint32_t epoch, int32_t* __restrict__ ticket, DeviceStatus* st, uint64_t wait_ns)
{
    constexpr int Q = kTvRows / (kTvThreads / kTvRows);  // columns per thread per tile (16)
    __shared__ double inv[kTvRows][kTvRows + 1];
    __shared__ double part[kTvRows][kTvThreads / kTvRows + 1];
    __shared__ double xs[2][kTvRows];
    __shared__ double vb[kTvRows];
    __shared__ int    s_t, s_abort;
    const int nb  = (n + kTvRows - 1) / kTvRows;
    const int tid = threadIdx.x;
    if (tid == 0)
    {
        s_t     = atomicAdd(ticket, 1);
        s_abort = 0;
    }
    __syncthreads();
    const int t = s_t;
    if (t >= nb)
    {
        return;
    }
    const int blk = upper ? nb - 1 - t : t;
    const int r0  = blk * kTvRows;
    const int br  = min(kTvRows, n - r0);
    if (SUBST)
    {
        // the diagonal block's triangle (unit diagonal not stored for L)
        for (int e = tid; e < kTvRows * kTvRows; e += kTvThreads)
        {
            const int  i = e / kTvRows, c = e % kTvRows;
            const bool in = i < br && c < br && (upper ? c >= i : (CHOL ? c <= i : c < i));
            const int  ri = CHOL && upper ? c : i, ci = CHOL && upper ? i : c;
            inv[i][c]     = in ? (double)a[(int64_t)(r0 + ri) * lda + r0 + ci] : 0.0;
        }
    }
    else
    {
        const double* src = dinv + ((size_t)blk * 2 + (upper ? 1 : 0)) * kTvRows * kTvRows;
        for (int e = tid; e < kTvRows * kTvRows; e += kTvThreads)
        {
            inv[e / kTvRows][e % kTvRows] = src[e];
        }
    }
    const int r = tid % kTvRows;
    const int q = tid / kTvRows;
    double    acc = 0.0;
    // software pipeline: A tile of the next block in registers, and (threads
    // < 64) the flagged x value of the next block
    TA     an[Q];
    double xn     = 0.0;
    bool   xn_ok  = false;
    auto   load_a = [&](int s, TA (&dst)[Q]) {
        const int jb = upper ? nb - 1 - s : s;
        const int c0 = jb * kTvRows + q * Q;
#pragma unroll
        for (int j = 0; j < Q; ++j)
        {
            const int64_t at = CHOL && upper ? (int64_t)(c0 + j) * lda + r0 + r : (int64_t)(r0 + r) * lda + c0 + j;
            dst[j]           = (r < br && c0 + j < n) ? a[at] : TA(0);
        }
    };
    if (t > 0)
    {
        load_a(0, an);
        if (tid < kTvRows)
        {
            xn_ok = tv_read(xll, upper ? nb - 1 : 0, tid, epoch, xn);
        }
    }
    for (int s = 0; s < t; ++s)
    {
        const int jb = upper ? nb - 1 - s : s;
        TA        ac[Q];
#pragma unroll
        for (int j = 0; j < Q; ++j)
        {
            ac[j] = an[j];
        }
        if (tid < kTvRows)
        {
            const int cw = min(kTvRows, n - jb * kTvRows);
            if (tid < cw && !xn_ok)
            {
                const uint64_t t0    = global_ns();
                uint32_t       polls = 0;
                while (!tv_read(xll, jb, tid, epoch, xn))
                {
                    if ((++polls & 255u) == 0 && global_ns() - t0 > wait_ns)
                    {
                        raise_error(st, DEV_WAIT_TIMEOUT, 20);
                        s_abort = 1;
                        break;
                    }
                }
            }
            xs[s & 1][tid] = tid < cw ? xn : 0.0;
        }
        __syncthreads();
        if (s_abort)
        {
            return;
        }
        if (s + 1 < t)
        {
            load_a(s + 1, an);
            if (tid < kTvRows)
            {
                xn_ok = tv_read(xll, upper ? nb - 2 - s : s + 1, tid, epoch, xn);
            }
        }
        // this block's products summed on their own, then added: blocked
        // summation keeps each row's dependent chain at one add per block
        double bp = 0.0;
#pragma unroll
        for (int j = 0; j < Q; ++j)
        {
            bp = fma((double)ac[j], xs[s & 1][q * Q + j], bp);
        }
        acc += bp;
    }
    part[r][q] = acc;
    __syncthreads();
    if (tid < kTvRows)
    {
        double sum = 0.0;
#pragma unroll
        for (int g = 0; g < kTvThreads / kTvRows; ++g)
        {
            sum += part[tid][g];
        }
        vb[tid] = tid < br ? x[r0 + tid] - sum : 0.0;
    }
    __syncthreads();
    if (SUBST)
    {
        // warp 0: lane l holds rows l and l + 32; at step p the owner of row
        // p finishes it (divides by the diagonal when upper) and broadcasts
        // it, and every lane updates its rows still to be solved
        if (tid < 32)
        {
            double v0 = vb[tid], v1 = vb[tid + 32];
            for (int qq = 0; qq < kTvRows; ++qq)
            {
                const int p = upper ? kTvRows - 1 - qq : qq;
                if (p >= br)
                {
                    continue;  // uniform across the warp
                }
                double vp = p < 32 ? v0 : v1;
                if (upper || CHOL)
                {
                    vp = vp / inv[p][p];
                }
                vp = __shfl_sync(0xffffffffu, vp, p & 31);
                if (tid == (p & 31))
                {
                    if (p < 32)
                        v0 = vp;
                    else
                        v1 = vp;
                }
                const int i0 = tid, i1 = tid + 32;
                if (upper ? i0 < p : (i0 > p && i0 < br))
                {
                    v0 = fma(-inv[i0][p], vp, v0);
                }
                if (upper ? i1 < p : (i1 > p && i1 < br))
                {
                    v1 = fma(-inv[i1][p], vp, v1);
                }
            }
            if (tid < br)
            {
                x[r0 + tid] = v0;
                tv_publish(xll, blk, tid, v0, epoch);
            }
            if (tid + 32 < br)
            {
                x[r0 + tid + 32] = v1;
                tv_publish(xll, blk, tid + 32, v1, epoch);
            }
        }
        return;
    }
    if (tid < br)
    {
        double v = 0.0;
#pragma unroll 8
        for (int c = 0; c < kTvRows; ++c)
        {
            v = fma(inv[tid][c], vb[c], v);
        }
        x[r0 + tid] = v;
        tv_publish(xll, blk, tid, v, epoch);
    }
}

// ---------------------------------------------------------------------------
// Refinement solves: the same one-launch scheme with 128-row blocks and the
// diagonal block applied as its inverse by every thread.
// ---------------------------------------------------------------------------
constexpr int    kTrRows    = 128;
constexpr int    kTrThreads = 512;  // 16 warps x 8 rows
constexpr size_t kTrInvSmem = sizeof(double) * kTrRows * (kTrRows + 1);

// Inverses of the 128 x 128 diagonal blocks of the unit-lower (blockIdx.y 0)
// and upper (1) triangles of an LU factor, FP64, row-major per block:
// dinv[2 b + 0] = L_bb^-1, dinv[2 b + 1] = U_bb^-1.  One thread per column of
// the inverse (substitution on e_j), the triangle in shared memory; a partial
// last block is padded with the identity.
template <typename TA>
__global__ void __launch_bounds__(kTrRows) k_invert_diag_blocks128(const TA* __restrict__ a, int64_t lda, int n,
    double* __restrict__ dinv)
{
    extern __shared__ double tri[];  // [kTrRows][kTrRows + 1]
    constexpr int LD    = kTrRows + 1;
    const int     blk   = blockIdx.x;
    const bool    upper = blockIdx.y == 1;
    const int     r0    = blk * kTrRows;
    const int     br    = min(kTrRows, n - r0);
    const int     j     = threadIdx.x;
    for (int e = j; e < kTrRows * kTrRows; e += kTrRows)
    {
        const int i = e / kTrRows, c = e % kTrRows;
        double    v = (i == c) ? 1.0 : 0.0;
        if (i < br && c < br && (upper ? c >= i : c < i))
        {
            v = (double)a[(int64_t)(r0 + i) * lda + r0 + c];
        }
        tri[i * LD + c] = v;
    }
    __syncthreads();
    double* out = dinv + ((size_t)blk * 2 + (upper ? 1 : 0)) * kTrRows * kTrRows;
    if (!upper)
    {
        for (int i = 0; i < kTrRows; ++i)
        {
            double s = (i == j) ? 1.0 : 0.0;
            for (int p = j; p < i; ++p)
            {
                s = fma(-tri[i * LD + p], out[p * kTrRows + j], s);
            }
            out[i * kTrRows + j] = i < j ? 0.0 : s;
        }
    }
    else
    {
        for (int i = kTrRows - 1; i >= 0; --i)
        {
            double s = (i == j) ? 1.0 : 0.0;
            for (int p = i + 1; p <= j; ++p)
            {
                s = fma(-tri[i * LD + p], out[p * kTrRows + j], s);
            }
            out[i * kTrRows + j] = i > j ? 0.0 : s / tri[i * LD + i];
        }
    }
}

// Sums, over the 32 lanes, eight per-lane values v[0..7] (one per row of a
// warp's 8 rows) in 9 shuffles: the halves exchanged at distance 16, 8, 4
// carry a row index bit each (4, 2, 1), the last two steps are plain sums.
// Lane l with (l & 3) == 0 ends with the sum for row
// 4 ((l >> 4) & 1) + 2 ((l >> 3) & 1) + ((l >> 2) & 1); tr_row gives it.
__device__ __forceinline__ double tr_reduce8(double (&v)[8], int lane)
{
    double h[4];
    const bool b4 = lane & 16;
#pragma unroll
    for (int j = 0; j < 4; ++j)
    {
        const double send = b4 ? v[j] : v[j + 4];
        const double keep = b4 ? v[j + 4] : v[j];
        h[j]              = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
    double    g[2];
    const bool b3 = lane & 8;
#pragma unroll
    for (int j = 0; j < 2; ++j)
    {
        const double send = b3 ? h[j] : h[j + 2];
        const double keep = b3 ? h[j + 2] : h[j];
        g[j]              = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
    const bool   b2   = lane & 4;
    const double send = b2 ? g[0] : g[1];
    double       r    = (b2 ? g[1] : g[0]) + __shfl_xor_sync(0xffffffffu, send, 4);
    r += __shfl_xor_sync(0xffffffffu, r, 2);
    r += __shfl_xor_sync(0xffffffffu, r, 1);
    return r;
}

__device__ __forceinline__ int tr_row(int lane)
{
    return 4 * ((lane >> 4) & 1) + 2 * ((lane >> 3) & 1) + ((lane >> 2) & 1);
}

// x <- T^-1 x for the unit-lower (upper = 0) or upper triangle of the factor
// `a` (FP32 or FP64 values, FP64 arithmetic), one right-hand side, for the
// refinement's corrections.  CTA = one 128-row block, claimed by ticket in
// solve order.  Warp w owns rows 8 w .. 8 w + 7 of the block and reads them
// row by row, coalesced: lane l multiplies columns 4 l .. 4 l + 3 of each
// solved block's tile by that block's values and keeps one partial sum per
// row; the partial sums are reduced across the warp once, after the last
// tile.  The tile of the block being waited for is already loaded (FP32: the
// next one too) when the block's publication is polled (bounded by wait_ns).
// The block's own values are the inverse diagonal block
// (k_invert_diag_blocks128, staged in shared memory at the start) applied in
// the same warp-per-row layout.  Solved values are published as flagged words
// (tv_publish layout, indexed by row) with the call's epoch.
template <typename TA>
__global__ void __launch_bounds__(kTrThreads, 1) k_trsv_refine(const TA* __restrict__ a, int64_t lda,
    double* __restrict__ x, int n, int upper, const double* __restrict__ dinv, uint64_t* __restrict__ xll,
    uint32_t epoch, int32_t* __restrict__ ticket, DeviceStatus* st, uint64_t wait_ns)
{
    extern __shared__ __align__(16) double inv[];  // [kTrRows][kTrRows]
    constexpr int  NW   = kTrThreads / 32;
    constexpr int  RPW  = kTrRows / NW;  // 8 rows per warp
    constexpr int  CPL  = kTrRows / 32;  // 4 columns per lane
    constexpr bool PREF = sizeof(TA) == 4;
    static_assert(RPW == 8 && CPL == 4, "warp-per-row layout");
    __shared__ __align__(16) double xs[2][kTrRows];
    __shared__ __align__(16) double vb[kTrRows];
    __shared__ int                  s_t, s_abort;
    const int nb   = (n + kTrRows - 1) / kTrRows;
    const int tid  = threadIdx.x;
    const int lane = tid & 31;
    const int w    = tid >> 5;
    if (tid == 0)
    {
        s_t     = atomicAdd(ticket, 1);
        s_abort = 0;
    }
    __syncthreads();
    const int t = s_t;
    if (t >= nb)
    {
        return;
    }
    const int blk = upper ? nb - 1 - t : t;
    const int r0  = blk * kTrRows;
    const int br  = min(kTrRows, n - r0);
    {
        const double2* src =
            reinterpret_cast<const double2*>(dinv + ((size_t)blk * 2 + (upper ? 1 : 0)) * kTrRows * kTrRows);
        double2* dst = reinterpret_cast<double2*>(inv);
        for (int e = tid; e < kTrRows * kTrRows / 2; e += kTrThreads)
        {
            dst[e] = src[e];
        }
    }
    // vector loads need every row start aligned to CPL elements
    const bool vec = (lda % CPL) == 0 && (reinterpret_cast<uintptr_t>(a) % (CPL * sizeof(TA))) == 0;
    auto load_tile = [&](int s, TA (&dst)[RPW][CPL]) {
        const int jb = upper ? nb - 1 - s : s;
        const int c  = jb * kTrRows + lane * CPL;
#pragma unroll
        for (int i = 0; i < RPW; ++i)
        {
            const int row = w * RPW + i;
            const TA* src = a + (int64_t)(r0 + (row < br ? row : 0)) * lda + c;
            if (row < br && vec && c + CPL <= n)
            {
                if constexpr (sizeof(TA) == 4)
                {
                    const float4 q = __ldg(reinterpret_cast<const float4*>(src));
                    dst[i][0] = q.x, dst[i][1] = q.y, dst[i][2] = q.z, dst[i][3] = q.w;
                }
                else
                {
                    const double2 q0 = __ldg(reinterpret_cast<const double2*>(src));
                    const double2 q1 = __ldg(reinterpret_cast<const double2*>(src) + 1);
                    dst[i][0] = q0.x, dst[i][1] = q0.y, dst[i][2] = q1.x, dst[i][3] = q1.y;
                }
            }
            else
            {
#pragma unroll
                for (int j = 0; j < CPL; ++j)
                {
                    dst[i][j] = (row < br && c + j < n) ? src[j] : TA(0);
                }
            }
        }
    };
    double acc[RPW];
#pragma unroll
    for (int i = 0; i < RPW; ++i)
    {
        acc[i] = 0.0;
    }
    TA cur[RPW][CPL];
    TA nxt[RPW][CPL];
    if (PREF && t > 0)
    {
        load_tile(0, nxt);
    }
    for (int s = 0; s < t; ++s)
    {
        const int jb = upper ? nb - 1 - s : s;
        if constexpr (PREF)
        {
#pragma unroll
            for (int i = 0; i < RPW; ++i)
            {
#pragma unroll
                for (int j = 0; j < CPL; ++j)
                {
                    cur[i][j] = nxt[i][j];
                }
            }
            if (s + 1 < t)
            {
                load_tile(s + 1, nxt);
            }
        }
        else
        {
            load_tile(s, cur);
        }
        if (tid < kTrRows)
        {
            const int cw = min(kTrRows, n - jb * kTrRows);
            double    xv = 0.0;
            if (tid < cw)
            {
                const uint64_t t0    = global_ns();
                uint32_t       polls = 0;
                while (!tv_read(xll, 0, jb * kTrRows + tid, epoch, xv))
                {
                    if ((++polls & 255u) == 0 && global_ns() - t0 > wait_ns)
                    {
                        raise_error(st, DEV_WAIT_TIMEOUT, 21);
                        s_abort = 1;
                        break;
                    }
                }
            }
            xs[s & 1][tid] = tid < cw ? xv : 0.0;  // double-buffered: read below until the next barrier
        }
        __syncthreads();
        if (s_abort)
        {
            return;
        }
        const double2 x01 = reinterpret_cast<const double2*>(xs[s & 1])[lane * 2];
        const double2 x23 = reinterpret_cast<const double2*>(xs[s & 1])[lane * 2 + 1];
#pragma unroll
        for (int i = 0; i < RPW; ++i)
        {
            acc[i] = fma((double)cur[i][0], x01.x, acc[i]);
            acc[i] = fma((double)cur[i][1], x01.y, acc[i]);
            acc[i] = fma((double)cur[i][2], x23.x, acc[i]);
            acc[i] = fma((double)cur[i][3], x23.y, acc[i]);
        }
    }
    const int my = w * RPW + tr_row(lane);  // the row whose sums this lane ends with (lane % 4 == 0)
    {
        const double sum = tr_reduce8(acc, lane);
        if ((lane & 3) == 0)
        {
            vb[my] = my < br ? x[r0 + my] - sum : 0.0;
        }
    }
    __syncthreads();
    const double2 v01 = reinterpret_cast<const double2*>(vb)[lane * 2];
    const double2 v23 = reinterpret_cast<const double2*>(vb)[lane * 2 + 1];
#pragma unroll
    for (int i = 0; i < RPW; ++i)
    {
        const double2 m01 = reinterpret_cast<const double2*>(inv + (w * RPW + i) * kTrRows)[lane * 2];
        const double2 m23 = reinterpret_cast<const double2*>(inv + (w * RPW + i) * kTrRows)[lane * 2 + 1];
        double        v   = m01.x * v01.x;
        v                 = fma(m01.y, v01.y, v);
        v                 = fma(m23.x, v23.x, v);
        acc[i]            = fma(m23.y, v23.y, v);
    }
    const double sum = tr_reduce8(acc, lane);
    if ((lane & 3) == 0 && my < br)
    {
        x[r0 + my] = sum;
        tv_publish(xll, 0, r0 + my, sum, epoch);
    }
}

// X <- T^-1 X for the unit-lower (upper = 0) or upper triangle of the factor
// `a` (FP32 or FP64 values, FP64 arithmetic), nrhs <= 64 right-hand sides
// stored row-major (n x nrhs, row stride nrhs), for the refinement's
// corrections of several right-hand sides.  One launch per triangle: CTA =
// one 128-row block, claimed by ticket in solve order; thread (i, j) keeps
// the 8 x 4 products of rows 8i..8i+7 and right-hand sides j, j+16, j+32,
// j+48 (so a warp's reads of a solved row are one broadcast wavefront).  For
// each solved block the CTA stages its 128 x 128 tile of the factor in
// shared memory as FP64 (converted once, not per product), then waits
// (thread 0, bounded by wait_ns) for that block's flag, reads the block's
// solved rows (L2, not L1: other SMs wrote them) and multiplies; the block's
// own rows are the inverse diagonal block (k_invert_diag_blocks128) times
// (B - products), applied in two 64-column halves.  A solved block is stored
// to x, fenced, and published by a release store of the call's epoch into
// flags[block].  Row strides of the staged tiles are odd (129, 65 doubles)
// so the two rows a warp reads fall in different banks.
constexpr int    kTmRhs     = 64;
constexpr int    kTmThreads = 256;
constexpr int    kTmLd      = kTrRows + 1;  // staged factor tile row stride (doubles)
constexpr int    kTmDLd     = 65;           // staged inverse half-tile row stride (doubles)
constexpr size_t kTmSmem    = sizeof(double) * kTrRows * kTmRhs + sizeof(double) * kTrRows * kTmLd;

template <typename TA>
__global__ void __launch_bounds__(kTmThreads, 1) k_trsm_refine(const TA* __restrict__ a, int64_t lda,
    double* __restrict__ x, int n, int nrhs, int upper, const double* __restrict__ dinv,
    uint32_t* __restrict__ flags, uint32_t epoch, int32_t* __restrict__ ticket, DeviceStatus* st, uint64_t wait_ns)
{
    extern __shared__ __align__(16) double tm_smem[];
    double*        Xs = tm_smem;                      // [128][64]
    double*        Ls = tm_smem + kTrRows * kTmRhs;   // [128][kTmLd]; also the inverse halves [128][kTmDLd]
    __shared__ int s_t, s_abort;
    const int      nb  = (n + kTrRows - 1) / kTrRows;
    const int      tid = threadIdx.x;
    const int      ti  = tid >> 4;  // rows 8 ti .. 8 ti + 7
    const int      tj  = tid & 15;  // right-hand sides tj + 16 q
    if (tid == 0)
    {
        s_t     = atomicAdd(ticket, 1);
        s_abort = 0;
    }
    __syncthreads();
    const int t = s_t;
    if (t >= nb)
    {
        return;
    }
    const int     blk = upper ? nb - 1 - t : t;
    const int     r0  = blk * kTrRows;
    const int     br  = min(kTrRows, n - r0);
    constexpr int V   = 16 / (int)sizeof(TA);
    const bool    vec = (lda % V) == 0 && (reinterpret_cast<uintptr_t>(a) % 16) == 0;
    double        acc[8][4];
#pragma unroll
    for (int m = 0; m < 8; ++m)
#pragma unroll
        for (int q = 0; q < 4; ++q)
            acc[m][q] = 0.0;
    auto product = [&](const double* S, int lds, int kcount, int xrow0) {
#pragma unroll 2
        for (int kk = 0; kk < kcount; ++kk)
        {
            double av[8], xv[4];
#pragma unroll
            for (int m = 0; m < 8; ++m)
                av[m] = S[(8 * ti + m) * lds + kk];
#pragma unroll
            for (int q = 0; q < 4; ++q)
                xv[q] = Xs[(xrow0 + kk) * kTmRhs + tj + 16 * q];
#pragma unroll
            for (int m = 0; m < 8; ++m)
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    acc[m][q] = fma(av[m], xv[q], acc[m][q]);
        }
    };
    for (int s = 0; s < t; ++s)
    {
        const int jb = upper ? nb - 1 - s : s;
        const int c0 = jb * kTrRows;
        const int cw = min(kTrRows, n - c0);
        __syncthreads();  // the previous tile's reads are done
        // the factor tile: rows r0.., columns c0.. (zeros outside), as FP64
        for (int e = tid; e < kTrRows * (kTrRows / V); e += kTmThreads)
        {
            const int row = e / (kTrRows / V);
            const int col = (e - row * (kTrRows / V)) * V;
            TA        v[V];
            const TA* src = a + (int64_t)(r0 + (row < br ? row : 0)) * lda + c0 + col;
            if (row < br && vec && col + V <= cw)
            {
                if constexpr (sizeof(TA) == 4)
                {
                    const float4 q = __ldg(reinterpret_cast<const float4*>(src));
                    v[0] = q.x, v[1] = q.y, v[2] = q.z, v[3] = q.w;
                }
                else
                {
                    const double2 q = __ldg(reinterpret_cast<const double2*>(src));
                    v[0] = q.x, v[1] = q.y;
                }
            }
            else
            {
#pragma unroll
                for (int u = 0; u < V; ++u)
                    v[u] = (row < br && col + u < cw) ? src[u] : TA(0);
            }
#pragma unroll
            for (int u = 0; u < V; ++u)
                Ls[row * kTmLd + col + u] = (double)v[u];
        }
        if (tid == 0)
        {
            const uint64_t t0    = global_ns();
            uint32_t       polls = 0;
            for (;;)
            {
                uint32_t f;
                asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(f) : "l"(flags + jb) : "memory");
                if (f == epoch)
                {
                    break;
                }
                if ((++polls & 255u) == 0 && global_ns() - t0 > wait_ns)
                {
                    raise_error(st, DEV_WAIT_TIMEOUT, 22);
                    s_abort = 1;
                    break;
                }
            }
        }
        __syncthreads();
        if (s_abort)
        {
            return;
        }
        for (int e = tid; e < kTrRows * kTmRhs; e += kTmThreads)
        {
            const int row = e / kTmRhs, q = e - row * kTmRhs;
            Xs[e]         = (row < cw && q < nrhs) ? __ldcg(x + (size_t)(c0 + row) * nrhs + q) : 0.0;
        }
        __syncthreads();
        product(Ls, kTmLd, kTrRows, 0);
    }
    __syncthreads();
    // V = B - products, in Xs
#pragma unroll
    for (int m = 0; m < 8; ++m)
    {
        const int row = 8 * ti + m;
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            const int c = tj + 16 * q;
            Xs[row * kTmRhs + c] =
                (row < br && c < nrhs) ? __ldcg(x + (size_t)(r0 + row) * nrhs + c) - acc[m][q] : 0.0;
            acc[m][q] = 0.0;
        }
    }
    // X = Dinv V, the inverse in two 64-column halves
    const double* D = dinv + ((size_t)blk * 2 + (upper ? 1 : 0)) * kTrRows * kTrRows;
    for (int h = 0; h < 2; ++h)
    {
        __syncthreads();
        for (int e = tid; e < kTrRows * 32; e += kTmThreads)
        {
            const int     row = e >> 5, c2 = (e & 31) * 2;
            const double2 v   = __ldg(reinterpret_cast<const double2*>(D + (size_t)row * kTrRows + h * 64 + c2));
            Ls[row * kTmDLd + c2]     = v.x;
            Ls[row * kTmDLd + c2 + 1] = v.y;
        }
        __syncthreads();
        product(Ls, kTmDLd, 64, h * 64);
    }
#pragma unroll
    for (int m = 0; m < 8; ++m)
    {
        const int row = 8 * ti + m;
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            const int c = tj + 16 * q;
            if (row < br && c < nrhs)
            {
                x[(size_t)(r0 + row) * nrhs + c] = acc[m][q];
            }
        }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0)
    {
        asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(flags + blk), "r"(epoch) : "memory");
    }
}

}  // namespace b200la
