// FP64 matrix update on the tensor cores: C[M x N] -= A[M x K] B[K x N]
// (row-major, row strides lda, ldb, ldc) with mma.sync m8n8k4 f64 (DMMA).
//
// One m8n8k4 DMMA computes, for every element of its 8 x 8 tile,
// d = c + a0 b0 + a1 b1 + a2 b2 + a3 b3 as four fused multiply-adds in k
// order, each rounded: on the B200 a chain of them along k gives the same
// bits as the scalar loop d = fma(a_k, b_k, d) for k = 0, 1, ... (measured
// on normal, subnormal, underflowing, overflowing, NaN/Inf and signed-zero
// operands).  That is what lets the blocked LU's trailing update run here
// and still reproduce the reference's factors bit for bit.
//
// Two modes:
//   FROM_ZERO = true   delta = sum_k a_ik b_kj accumulated from zero in k
//                      order, then C = C - delta: the LU trailing update of
//                      lu_decomposition_native.cpp:400-422 (delta from the
//                      GEMM, then subtracted), bit-identical to it;
//   FROM_ZERO = false  the accumulators start at -C and end at -(C - A B),
//                      stored negated (inversion: no bit-parity requirement,
//                      and C is loaded while the first stages are in flight).
//
// CTA tile kDmTile x kDmTile, 16 warps of 32 x 32 (4 x 4 DMMA tiles, 32
// accumulators per thread, 4 warps per scheduler), K streamed in kDmKC-deep
// stages through a kDmStages cp.async ring.  Fragments (g = lane/4,
// t = lane%4): A[8 rows][4 k] -> a = A[g][t]; B[4 k][8 cols] -> b = B[t][g];
// C[8][8] -> c0, c1 = C[g][2t], C[g][2t+1].  The padded smem rows (A: kDmKC
// + 4 doubles, B: kDmTile + 4) place the rows one fragment load touches 8
// banks apart, so every fragment load is the minimal two wavefronts.
// Zero-filled padding (k >= K, rows >= M, columns >= N) adds +0 products,
// which leave a from-zero sum unchanged (it is never -0).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "lu_kernels.cuh"
#include "solve_kernels.cuh"

namespace b200la
{

constexpr int    kDmTile    = 128;
constexpr int    kDmThreads = 512;
constexpr int    kDmKC      = 32;
constexpr int    kDmLDA     = kDmKC + 4;
constexpr int    kDmLDB     = kDmTile + 4;
constexpr int    kDmStages  = 3;
constexpr int    kDmAElems  = kDmTile * kDmLDA;
constexpr int    kDmStage   = kDmAElems + kDmKC * kDmLDB;
constexpr size_t kDmSmem    = sizeof(double) * (size_t)kDmStages * kDmStage;

__device__ __forceinline__ void dmma_884(double& c0, double& c1, double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(c0), "+d"(c1)
        : "d"(a), "d"(b));
}

// One 16-byte piece (two doubles) global -> shared; `valid` leading elements
// copied, the rest zero-filled.  Whole pieces as one 16-byte cp.async when
// the rows are 16-byte aligned, else element by element.
__device__ __forceinline__ void dm_piece(double* s, const double* g, const double* safe, int valid, bool vec16)
{
    if (vec16 && (valid >= 2 || valid <= 0))
    {
        cp_async16(s, valid > 0 ? g : safe, valid > 0);
        return;
    }
    cp_async8(s, valid > 0 ? g : safe, valid > 0);
    cp_async8(s + 1, valid > 1 ? g + 1 : safe, valid > 1);
}

// A thread's share of one stage: pieces i < 4 of the A tile (row tid/16 +
// 32 i, columns 2 (tid%16) .. +1 of the stage) and of the B tile (row
// tid/64 + 8 i, columns 2 (tid%64) .. +1).  Addresses are formed once per
// tile; a stage only advances them by its depth.
struct DmLoader
{
    const double* a;     // A row tid/16 of the tile, column 2 (tid%16)
    const double* b;     // B row tid/64, column n0 + 2 (tid%64)
    int           acol;  // 2 (tid%16)
    int           arows; // bit i: A row tid/16 + 32 i is inside M
    int           bcols; // valid columns of the B piece (0..2)
    int           brow;  // tid/64
};

__device__ __forceinline__ DmLoader dm_loader(const double* A, int64_t lda, const double* B, int64_t ldb, int M,
    int N, int m0, int n0)
{
    DmLoader  L;
    const int ra = threadIdx.x >> 4, qa = threadIdx.x & 15;
    const int rb = threadIdx.x >> 6, qb = threadIdx.x & 63;
    L.acol  = 2 * qa;
    L.a     = A + (int64_t)(m0 + ra) * lda + L.acol;
    L.arows = 0;
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        L.arows |= (m0 + ra + 32 * i < M) ? (1 << i) : 0;
    }
    L.brow  = rb;
    L.bcols = max(0, min(2, N - (n0 + 2 * qb)));
    L.b     = B + (int64_t)rb * ldb + n0 + 2 * qb;
    return L;
}

// Issue piece `i` (0..3: A, 4..7: B) of the stage at depth k0 into slot `st`.
__device__ __forceinline__ void dm_issue(const DmLoader& L, double* st, int i, const double* A, int64_t lda,
    const double* B, int64_t ldb, int K, int k0, bool vec16)
{
    if (i < 4)
    {
        const int  valid = (L.arows >> i) & 1 ? min(2, K - (k0 + L.acol)) : 0;
        const int  r     = (threadIdx.x >> 4) + 32 * i;
        dm_piece(st + r * kDmLDA + L.acol, L.a + (int64_t)(32 * i) * lda + k0, A, valid, vec16);
    }
    else
    {
        const int i4    = i - 4;
        const int p     = L.brow + 8 * i4;
        const int valid = k0 + p < K ? L.bcols : 0;
        dm_piece(st + kDmAElems + p * kDmLDB + 2 * (threadIdx.x & 63), L.b + (int64_t)(k0 + 8 * i4) * ldb, B,
            valid, vec16);
    }
}

template <bool FROM_ZERO>
__global__ void __launch_bounds__(kDmThreads, 1) k_dmma_update(int M, int N, int K, const double* __restrict__ A,
    int64_t lda, const double* __restrict__ B, int64_t ldb, double* __restrict__ C, int64_t ldc, int vec16,
    const DeviceStatus* gate)
{
    extern __shared__ __align__(16) unsigned char dm_smem[];
    if (gated(gate))
    {
        return;
    }
    double*    smem    = reinterpret_cast<double*>(dm_smem);
    const int  m0      = blockIdx.y * kDmTile;
    const int  n0      = blockIdx.x * kDmTile;
    const int  warp    = threadIdx.x >> 5;
    const int  lane    = threadIdx.x & 31;
    const int  g       = lane >> 2;
    const int  t       = lane & 3;
    const int  wm      = (warp >> 2) * 32;
    const int  wn      = (warp & 3) * 32;
    const int  nchunks = (K + kDmKC - 1) / kDmKC;
    const bool v16     = vec16 != 0;

    double acc[4][4][2];
    if (FROM_ZERO)
    {
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                acc[i][j][0] = 0.0;
                acc[i][j][1] = 0.0;
            }
        }
        // pull the C tile into L2 while the products accumulate
        const int r = threadIdx.x >> 2, q = threadIdx.x & 3;
        if (m0 + r < M)
        {
            const double* crow = C + (int64_t)(m0 + r) * ldc + n0;
#pragma unroll
            for (int h = 0; h < 2; ++h)
            {
                const int c = (q + 4 * h) * 16;
                if (n0 + c < N)
                {
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(crow + c));
                }
            }
        }
    }
    else
    {
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
            const int     row  = m0 + wm + 8 * i + g;
            const double* crow = C + (int64_t)row * ldc;
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                const int col = n0 + wn + 8 * j + 2 * t;
                double2   v   = make_double2(0.0, 0.0);
                if (row < M)
                {
                    if (v16 && col + 1 < N)
                    {
                        v = *reinterpret_cast<const double2*>(crow + col);
                    }
                    else
                    {
                        v.x = col < N ? crow[col] : 0.0;
                        v.y = col + 1 < N ? crow[col + 1] : 0.0;
                    }
                }
                acc[i][j][0] = -v.x;
                acc[i][j][1] = -v.y;
            }
        }
    }

    const DmLoader L = dm_loader(A, lda, B, ldb, M, N, m0, n0);
#pragma unroll
    for (int s = 0; s < kDmStages - 1; ++s)
    {
        if (s < nchunks)
        {
#pragma unroll
            for (int i = 0; i < 8; ++i)
            {
                dm_issue(L, smem + s * kDmStage, i, A, lda, B, ldb, K, s * kDmKC, v16);
            }
        }
        cp_async_commit();
    }
    for (int c = 0; c < nchunks; ++c)
    {
        cp_async_wait<kDmStages - 2>();
        __syncthreads();  // stage c landed for every thread; stage c-1 is free
        const int     pf   = c + kDmStages - 1;
        double*       dst  = smem + (pf % kDmStages) * kDmStage;
        const double* sa   = smem + (c % kDmStages) * kDmStage + (wm + g) * kDmLDA + t;
        const double* sb   = smem + (c % kDmStages) * kDmStage + kDmAElems + t * kDmLDB + wn + g;
#pragma unroll
        for (int ks = 0; ks < kDmKC / 4; ++ks)
        {
            // one piece of stage pf per depth step, spread over the chunk
            if (pf < nchunks)
            {
                dm_issue(L, dst, ks, A, lda, B, ldb, K, pf * kDmKC, v16);
            }
            double af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
            {
                af[i] = sa[8 * i * kDmLDA + 4 * ks];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                bf[j] = sb[4 * ks * kDmLDB + 8 * j];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
            {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                    dmma_884(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
                }
            }
        }
        cp_async_commit();
    }
    cp_async_wait<0>();

#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        const int row = m0 + wm + 8 * i + g;
        if (row >= M)
        {
            continue;
        }
        double* crow = C + (int64_t)row * ldc;
        if (FROM_ZERO)
        {
            double2 cv[4];
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                const int col = n0 + wn + 8 * j + 2 * t;
                if (v16 && col + 1 < N)
                {
                    cv[j] = *reinterpret_cast<const double2*>(crow + col);
                }
                else
                {
                    cv[j].x = col < N ? crow[col] : 0.0;
                    cv[j].y = col + 1 < N ? crow[col + 1] : 0.0;
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                cv[j].x = cv[j].x - acc[i][j][0];
                cv[j].y = cv[j].y - acc[i][j][1];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                const int col = n0 + wn + 8 * j + 2 * t;
                if (v16 && col + 1 < N)
                {
                    *reinterpret_cast<double2*>(crow + col) = cv[j];
                }
                else
                {
                    if (col < N)
                    {
                        crow[col] = cv[j].x;
                    }
                    if (col + 1 < N)
                    {
                        crow[col + 1] = cv[j].y;
                    }
                }
            }
        }
        else
        {
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                const int col = n0 + wn + 8 * j + 2 * t;
                if (v16 && col + 1 < N)
                {
                    *reinterpret_cast<double2*>(crow + col) = make_double2(-acc[i][j][0], -acc[i][j][1]);
                }
                else
                {
                    if (col < N)
                    {
                        crow[col] = -acc[i][j][0];
                    }
                    if (col + 1 < N)
                    {
                        crow[col + 1] = -acc[i][j][1];
                    }
                }
            }
        }
    }
}

// The LU trailing update A22 -= L21 U12 (panel depth K <= kBandK) as a
// band kernel, bit-identical to k_dmma_update<true>.  The kDmTile x kDmTile
// output tiles (units) are numbered row band by row band; CTA b of G takes
// units [b*T/G, (b+1)*T/G), and G is a whole number of waves of SMs, so every
// CTA gets the same count within one and no wave runs nearly empty, while
// CTAs stay short (a few units) and an SM frees up for a concurrent
// higher-priority kernel every few tens of microseconds.  It keeps its band's kDmTile x K
// slice of L21 resident in shared memory, computes tile u while tile u+1's
// U12 slice lands in the other buffer and its A22 rows are pulled into L2,
// and reloads the L21 slice only when its run of units enters the next band.
// Per tile: delta from zero over k in order, then A22 - delta.
constexpr int    kBandK      = 64;
constexpr int    kBandLDA    = kBandK + 4;
constexpr int    kBandAElems = kDmTile * kBandLDA;
constexpr int    kBandBElems = kBandK * kDmLDB;
constexpr size_t kBandSmem   = sizeof(double) * ((size_t)kBandAElems + 2 * (size_t)kBandBElems);

__device__ __forceinline__ void band_load_b(double* sb, const double* B, int64_t ldb, int N, int K, int n0, bool vec16)
{
    constexpr int BPR = kDmTile / 2;
#pragma unroll
    for (int e = threadIdx.x; e < kBandK * BPR; e += kDmThreads)
    {
        const int p = e / BPR, q = e - (e / BPR) * BPR;
        const int col = n0 + 2 * q;
        const int valid = p < K ? min(2, N - col) : 0;
        dm_piece(sb + p * kDmLDB + 2 * q, valid > 0 ? B + (int64_t)p * ldb + col : B, B, valid, vec16);
    }
}

__device__ __forceinline__ void band_prefetch_c(const double* C, int64_t ldc, int M, int N, int m0, int n0)
{
    const int r = threadIdx.x >> 2, q = threadIdx.x & 3;
    if (m0 + r < M)
    {
        const double* crow = C + (int64_t)(m0 + r) * ldc + n0;
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            const int c = (q + 4 * h) * 16;
            if (n0 + c < N)
            {
                asm volatile("prefetch.global.L2 [%0];" ::"l"(crow + c));
            }
        }
    }
}

__device__ __forceinline__ void band_load_a(double* sa, const double* A, int64_t lda, int M, int K, int m0,
    bool vec16)
{
    constexpr int APR = kBandK / 2;
#pragma unroll
    for (int e = threadIdx.x; e < kDmTile * APR; e += kDmThreads)
    {
        const int r = e / APR, q = e - (e / APR) * APR;
        const int row = m0 + r, col = 2 * q;
        const int valid = row < M ? min(2, K - col) : 0;
        dm_piece(sa + r * kBandLDA + col, valid > 0 ? A + (int64_t)row * lda + col : A, A, valid, vec16);
    }
}

template <int Unused = 0>
__global__ void __launch_bounds__(kDmThreads, 1) k_dmma_band(int M, int N, int K, const double* __restrict__ A,
    int64_t lda, const double* __restrict__ B, int64_t ldb, double* __restrict__ C, int64_t ldc, int vec16,
    const DeviceStatus* gate)
{
    extern __shared__ __align__(16) unsigned char dm_smem[];
    if (gated(gate))
    {
        return;
    }
    double*    sa    = reinterpret_cast<double*>(dm_smem);
    double*    sbuf  = sa + kBandAElems;
    const int  ct    = (N + kDmTile - 1) / kDmTile;
    const int  total = ct * ((M + kDmTile - 1) / kDmTile);
    const int  u0    = (int)(((int64_t)blockIdx.x * total) / gridDim.x);
    const int  u1    = (int)(((int64_t)(blockIdx.x + 1) * total) / gridDim.x);
    const int  warp  = threadIdx.x >> 5;
    const int  lane  = threadIdx.x & 31;
    const int  g     = lane >> 2;
    const int  t     = lane & 3;
    const int  wm    = (warp >> 2) * 32;
    const int  wn    = (warp & 3) * 32;
    const bool v16   = vec16 != 0;
    if (u0 >= u1)
    {
        return;
    }

    // the first unit's L21 slice (zero-filled past M and K) and U12 tile
    band_load_a(sa, A, lda, M, K, (u0 / ct) * kDmTile, v16);
    band_load_b(sbuf, B, ldb, N, K, (u0 % ct) * kDmTile, v16);
    cp_async_commit();
    band_prefetch_c(C, ldc, M, N, (u0 / ct) * kDmTile, (u0 % ct) * kDmTile);

    for (int u = u0; u < u1; ++u)
    {
        const int  m0   = (u / ct) * kDmTile;
        const int  n0   = (u % ct) * kDmTile;
        const int  cur  = (u - u0) & 1;
        const bool next = u + 1 < u1;
        const bool same = next && (u + 1) / ct == u / ct;
        cp_async_wait<0>();
        __syncthreads();  // this unit's operands landed; the other buffer is free
        if (same)
        {
            band_load_b(sbuf + (cur ^ 1) * kBandBElems, B, ldb, N, K, ((u + 1) % ct) * kDmTile, v16);
            band_prefetch_c(C, ldc, M, N, m0, ((u + 1) % ct) * kDmTile);
        }
        cp_async_commit();

        double acc[4][4][2];
#pragma unroll
        for (int i = 0; i < 4; ++i)
        {
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                acc[i][j][0] = 0.0;
                acc[i][j][1] = 0.0;
            }
        }
        const double* fa = sa + (wm + g) * kBandLDA + t;
        const double* fb = sbuf + cur * kBandBElems + t * kDmLDB + wn + g;
#pragma unroll 4
        for (int ks = 0; ks < kBandK / 4; ++ks)
        {
            double af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
            {
                af[i] = fa[8 * i * kBandLDA + 4 * ks];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                bf[j] = fb[4 * ks * kDmLDB + 8 * j];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
            {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                    dmma_884(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
                }
            }
        }

        // this thread's A22 values two fragment rows at a time: the loads of
        // a half are independent (mostly L2 hits after the prefetch) and
        // issue together, then the subtractions and stores
#pragma unroll
        for (int h = 0; h < 2; ++h)
        {
            double2 cv[2][4];
#pragma unroll
            for (int ii = 0; ii < 2; ++ii)
            {
                const int     row  = m0 + wm + 8 * (2 * h + ii) + g;
                const double* crow = C + (int64_t)row * ldc;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                    const int col = n0 + wn + 8 * j + 2 * t;
                    if (row < M && v16 && col + 1 < N)
                    {
                        cv[ii][j] = *reinterpret_cast<const double2*>(crow + col);
                    }
                    else
                    {
                        cv[ii][j].x = row < M && col < N ? crow[col] : 0.0;
                        cv[ii][j].y = row < M && col + 1 < N ? crow[col + 1] : 0.0;
                    }
                }
            }
#pragma unroll
            for (int ii = 0; ii < 2; ++ii)
            {
                const int i   = 2 * h + ii;
                const int row = m0 + wm + 8 * i + g;
                if (row >= M)
                {
                    continue;
                }
                double* crow = C + (int64_t)row * ldc;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                    const int col = n0 + wn + 8 * j + 2 * t;
                    cv[ii][j].x   = cv[ii][j].x - acc[i][j][0];
                    cv[ii][j].y   = cv[ii][j].y - acc[i][j][1];
                    if (v16 && col + 1 < N)
                    {
                        *reinterpret_cast<double2*>(crow + col) = cv[ii][j];
                    }
                    else
                    {
                        if (col < N)
                        {
                            crow[col] = cv[ii][j].x;
                        }
                        if (col + 1 < N)
                        {
                            crow[col + 1] = cv[ii][j].y;
                        }
                    }
                }
            }
        }

        if (next && !same)
        {
            // the run enters the next band: every warp is done with this
            // band's L21 slice before it is replaced
            __syncthreads();
            band_load_a(sa, A, lda, M, K, ((u + 1) / ct) * kDmTile, v16);
            band_load_b(sbuf + (cur ^ 1) * kBandBElems, B, ldb, N, K, ((u + 1) % ct) * kDmTile, v16);
            cp_async_commit();
            band_prefetch_c(C, ldc, M, N, ((u + 1) / ct) * kDmTile, ((u + 1) % ct) * kDmTile);
        }
    }
    cp_async_wait<0>();
}

// Grid size for k_dmma_band: whole waves of one CTA per SM, about
// kBandUnits units per CTA (fewer CTAs only when there are fewer units).
constexpr int kBandUnits = 4;
inline int band_grid(int rows, int cols, int sms)
{
    const int total = ((rows + kDmTile - 1) / kDmTile) * ((cols + kDmTile - 1) / kDmTile);
    const int sm    = sms > 0 ? sms : 148;
    const int waves = (total + sm * kBandUnits - 1) / (sm * kBandUnits);
    const int g     = waves * sm;
    return total < g ? total : g;
}

// General FP64 multiplication on the tensor cores, bit-identical to the
// reference's loops where they are fma chains:
//   c = beta c (beta == 0: c = 0, c not read), then for k in order
//   c = fma(alpha a_ik, b_kj, c)  with alpha a_ik rounded first
// (multiplication_native.cpp, op(b) = b; alpha == 1 leaves a exact), which
// is also the reference's batched kernel (sum += a b from zero,
// multiplication_batched_cublas.cu:15-40) with alpha = 1, beta = 0.  A
// chain of m8n8k4 DMMAs along k is that fma chain.  TRANS_A: op(a) = a^T
// (a stored depth x rows).  Tiles, warps and the cp.async ring as
// k_dmma_update; blockIdx.z selects the matrix of a batch (element strides
// sa, sb, sc).
template <bool TRANS_A>
__global__ void __launch_bounds__(kDmThreads, 1) k_dmma_gemm(int M, int N, int K, double alpha,
    const double* __restrict__ A, int64_t lda, int64_t sa, const double* __restrict__ B, int64_t ldb, int64_t sb,
    double beta, double* __restrict__ C, int64_t ldc, int64_t sc, int vec16)
{
    extern __shared__ __align__(16) unsigned char dm_smem[];
    double*    smem    = reinterpret_cast<double*>(dm_smem);
    A += (int64_t)blockIdx.z * sa;
    B += (int64_t)blockIdx.z * sb;
    C += (int64_t)blockIdx.z * sc;
    const int  m0      = blockIdx.y * kDmTile;
    const int  n0      = blockIdx.x * kDmTile;
    const int  warp    = threadIdx.x >> 5;
    const int  lane    = threadIdx.x & 31;
    const int  g       = lane >> 2;
    const int  t       = lane & 3;
    const int  wm      = (warp >> 2) * 32;
    const int  wn      = (warp & 3) * 32;
    const int  nchunks = (K + kDmKC - 1) / kDmKC;
    const bool v16     = vec16 != 0;

    // stage loader: A as [m][k] (row stride kDmLDA) or, transposed, [k][m]
    // (row stride kDmLDB); B as [k][n] (kDmLDB)
    auto load_stage = [&](double* st, int k0) {
        if (!TRANS_A)
        {
            constexpr int APR = kDmKC / 2;
            for (int e = threadIdx.x; e < kDmTile * APR; e += kDmThreads)
            {
                const int r = e / APR, q = e - (e / APR) * APR;
                const int row = m0 + r, col = k0 + 2 * q;
                const int valid = row < M ? min(2, K - col) : 0;
                dm_piece(st + r * kDmLDA + 2 * q, valid > 0 ? A + (int64_t)row * lda + col : A, A, valid, v16);
            }
        }
        else
        {
            constexpr int APR = kDmTile / 2;
            for (int e = threadIdx.x; e < kDmKC * APR; e += kDmThreads)
            {
                const int p = e / APR, q = e - (e / APR) * APR;
                const int kk = k0 + p, col = m0 + 2 * q;
                const int valid = kk < K ? min(2, M - col) : 0;
                dm_piece(st + p * kDmLDB + 2 * q, valid > 0 ? A + (int64_t)kk * lda + col : A, A, valid, v16);
            }
        }
        constexpr int BPR = kDmTile / 2;
        for (int e = threadIdx.x; e < kDmKC * BPR; e += kDmThreads)
        {
            const int p = e / BPR, q = e - (e / BPR) * BPR;
            const int kk = k0 + p, col = n0 + 2 * q;
            const int valid = kk < K ? min(2, N - col) : 0;
            dm_piece(st + kDmAElems + p * kDmLDB + 2 * q, valid > 0 ? B + (int64_t)kk * ldb + col : B, B, valid,
                v16);
        }
    };

    // accumulators: beta c (c not read when beta == 0)
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        const int     row  = m0 + wm + 8 * i + g;
        const double* crow = C + (int64_t)row * ldc;
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const int col = n0 + wn + 8 * j + 2 * t;
            double2   v   = make_double2(0.0, 0.0);
            if (beta != 0.0 && row < M)
            {
                if (v16 && col + 1 < N)
                {
                    v = *reinterpret_cast<const double2*>(crow + col);
                }
                else
                {
                    v.x = col < N ? crow[col] : 0.0;
                    v.y = col + 1 < N ? crow[col + 1] : 0.0;
                }
                if (beta != 1.0)
                {
                    v.x = v.x * beta;
                    v.y = v.y * beta;
                }
            }
            acc[i][j][0] = v.x;
            acc[i][j][1] = v.y;
        }
    }

#pragma unroll
    for (int s = 0; s < kDmStages - 1; ++s)
    {
        if (s < nchunks)
        {
            load_stage(smem + s * kDmStage, s * kDmKC);
        }
        cp_async_commit();
    }
    const bool scale = alpha != 1.0;
    for (int c = 0; c < nchunks; ++c)
    {
        cp_async_wait<kDmStages - 2>();
        __syncthreads();  // stage c landed for every thread; stage c-1 is free
        const int pf = c + kDmStages - 1;
        if (pf < nchunks)
        {
            load_stage(smem + (pf % kDmStages) * kDmStage, pf * kDmKC);
        }
        cp_async_commit();
        const double* st = smem + (c % kDmStages) * kDmStage;
        const double* sb_ = st + kDmAElems + t * kDmLDB + wn + g;
#pragma unroll
        for (int ks = 0; ks < kDmKC / 4; ++ks)
        {
            double af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; ++i)
            {
                af[i] = TRANS_A ? st[(4 * ks + t) * kDmLDB + wm + g + 8 * i]
                                : st[(wm + g + 8 * i) * kDmLDA + 4 * ks + t];
                if (scale)
                {
                    af[i] = alpha * af[i];
                }
            }
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                bf[j] = sb_[4 * ks * kDmLDB + 8 * j];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
            {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                    dmma_884(acc[i][j][0], acc[i][j][1], af[i], bf[j]);
                }
            }
        }
    }
    cp_async_wait<0>();

#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        const int row = m0 + wm + 8 * i + g;
        if (row >= M)
        {
            continue;
        }
        double* crow = C + (int64_t)row * ldc;
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const int col = n0 + wn + 8 * j + 2 * t;
            if (v16 && col + 1 < N)
            {
                *reinterpret_cast<double2*>(crow + col) = make_double2(acc[i][j][0], acc[i][j][1]);
            }
            else
            {
                if (col < N)
                {
                    crow[col] = acc[i][j][0];
                }
                if (col + 1 < N)
                {
                    crow[col + 1] = acc[i][j][1];
                }
            }
        }
    }
}

inline bool dm_aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// 1 when every operand's rows start 16-byte aligned (the 16-byte copy path).
inline int dm_vec16(const double* a, int64_t lda, const double* b, int64_t ldb, const double* c, int64_t ldc)
{
    return dm_aligned16(a) && dm_aligned16(b) && dm_aligned16(c) && (lda * 8) % 16 == 0 && (ldb * 8) % 16 == 0 &&
           (ldc * 8) % 16 == 0;
}

}  // namespace b200la
