// Mixed-precision LU solve with FP64 iterative refinement (LU-IR) and
// GMRES-IR, on the B200 tensor cores.
//
//   1. A (FP64) -> A32 (FP32 copy), ||A||_inf on the way.
//   2. Blocked LU with partial pivoting of A32 in 256-column outer blocks:
//      inside a block, 64-column panels (the FP32 panel kernels), their row
//      interchanges, and in-block updates (SIMT FP32); then the block's
//      U12 = L11^-1 A12 (FP32, k_outer_u12), the operand copies of L21 and
//      U12^T in the factorization precision, and the trailing update
//      A22 -= L21 U12 on tcgen05 with FP32 accumulation (k_tc_update).
//      Precisions: FP32 (three-term TF32 split), TF32, BF16, FP16, and
//      FP8-E4M3 with power-of-two scales per row of L21 and per column of
//      U12 (each spanning the block's 256-deep reduction).
//   3. x0 = U^-1 L^-1 P b with the FP32 factors applied in FP64; then
//      r = b - A x in FP64, eta = ||r|| / (||A|| ||x|| + ||b||) (inf norms),
//      stop at eta <= tolerance; else d = U^-1 L^-1 P r, x += d.  When plain
//      refinement stalls, GMRES-IR: restarted GMRES in FP64 on A d = r, left
//      preconditioned by the low-precision factors (Carson & Higham, SISC
//      40(2), 2018).  If that fails too, the next precision up is tried, down
//      to plain FP64 LU.
// FP64 stays on the GPU for the residual, the update and the test.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_fp8.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "lu_driver.cuh"
#include "tc_api.cuh"
#include "trsv.cuh"

namespace b200la
{
namespace
{
constexpr int kOuterNB = 256;
constexpr int kMaxBlockPanels = kOuterNB / 32;  // panels of an outer block (32 or 64 columns wide)

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ void atomic_max_nonneg(unsigned long long* p, double v)
{
    atomicMax(p, (unsigned long long)__double_as_longlong(v));
}

// A32 = (float)A, and ||A||_inf = max row sum of |A|.  A warp per row.
__global__ void k_convert_a(const double* __restrict__ a, int64_t lda, float* __restrict__ a32, int n,
    unsigned long long* anorm)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= n)
    {
        return;
    }
    const double* row = a + (int64_t)warp * lda;
    float*        out = a32 + (int64_t)warp * n;
    double        s   = 0.0;
    for (int j = lane; j < n; j += 32)
    {
        const double v = row[j];
        out[j]         = (float)v;
        s += fabs(v);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        s += __shfl_down_sync(0xffffffffu, s, off);
    }
    if (lane == 0)
    {
        atomic_max_nonneg(anorm, s);
    }
}

__device__ __forceinline__ float tf32_trunc(float x) { return __uint_as_float(__float_as_uint(x) & ~0x1FFFu); }

template <int KIND> struct OpStore;
template <> struct OpStore<TC_TF32>
{
    using type = float;
    __device__ static float conv(float x) { return x; }
};
template <> struct OpStore<TC_BF16>
{
    using type = __nv_bfloat16;
    __device__ static __nv_bfloat16 conv(float x) { return __float2bfloat16_rn(x); }
};
template <> struct OpStore<TC_FP16>
{
    using type = __half;
    __device__ static __half conv(float x) { return __float2half_rn(x); }
};
template <> struct OpStore<TC_FP8>
{
    using type = __nv_fp8_storage_t;
    __device__ static __nv_fp8_storage_t conv(float x) { return __nv_cvt_float_to_fp8(x, __NV_SATFINITE, __NV_E4M3); }
};

// Power-of-two scale s with amax * s in [128, 256) (E4M3's largest finite
// value is 448), exponent clamped to the normal float range; 1 for amax 0.
// Returns s and stores 1/s (exact) in *inv.
__device__ __forceinline__ float fp8_scale(float amax, float* inv)
{
    if (!(amax > 0.f) || !isfinite(amax))
    {
        *inv = 1.f;
        return 1.f;
    }
    int e = 0;
    frexpf(amax, &e);  // amax = f 2^e, f in [0.5, 1)
    int se = 8 - e;
    se     = se > 126 ? 126 : (se < -126 ? -126 : se);
    *inv   = ldexpf(1.f, -se);
    return ldexpf(1.f, se);
}

// FP8 L21 operand: a warp per row of rows [r_begin, n) x columns [K, K+256)
// of A32; the row's scale brings its largest entry into [128, 256).
__global__ void k_make_l21_fp8(const float* __restrict__ a32, int n, int K, int r_begin,
    __nv_fp8_storage_t* __restrict__ op, float* __restrict__ inv_scale)
{
    const int     lane = threadIdx.x & 31;
    const int64_t rows = n - r_begin;
    for (int64_t r = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; r < rows;
         r += ((int64_t)gridDim.x * blockDim.x) >> 5)
    {
        const float* src = a32 + (r_begin + r) * (int64_t)n + K;
        float        v[kOuterNB / 32];
        float        amax = 0.f;
#pragma unroll
        for (int q = 0; q < kOuterNB / 32; ++q)
        {
            v[q] = src[q * 32 + lane];
            amax = fmaxf(amax, fabsf(v[q]));
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, off));
        }
        float       inv;
        const float sc = fp8_scale(amax, &inv);
#pragma unroll
        for (int q = 0; q < kOuterNB / 32; ++q)
        {
            op[r * kOuterNB + q * 32 + lane] = OpStore<TC_FP8>::conv(v[q] * sc);
        }
        if (lane == 0)
        {
            inv_scale[r] = inv;
        }
    }
}

// L21 operand: rows [r_begin, n) x columns [K, K+256) of A32 -> K-major copy.
template <int KIND, bool SPLIT>
__global__ void k_make_l21(const float* __restrict__ a32, int n, int K, int r_begin,
    typename OpStore<KIND>::type* __restrict__ op, float* __restrict__ op_small)
{
    const int64_t total = (int64_t)(n - r_begin) * kOuterNB;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t r  = e / kOuterNB;
        const int     kk = (int)(e - r * kOuterNB);
        const float   v  = a32[(r_begin + r) * (int64_t)n + K + kk];
        op[e]            = OpStore<KIND>::conv(v);
        if constexpr (SPLIT)
        {
            op_small[e] = v - tf32_trunc(v);
        }
    }
}

// U12 = L11^-1 A12 for the outer block rows [K, K+256), columns [K+256, n)
// (strips of 64 columns), written back in FP32 and as the transposed operand
// copy U12^T (rows = columns of A22, K-major).
constexpr int kOuStrip = 64;

// Lb = the 64 x 64 block of A32 at (r0, c0) (strictly lower part only when
// `unit_lower`), by 256 threads with all 16 loads of a thread in flight
// before any store.
constexpr int kLbLd = kNB + 4;  // 16-byte aligned rows for float4 reads

__device__ __forceinline__ void load_lblock(float (*Lb)[kLbLd], const float* __restrict__ a32, int n, int r0,
    int c0, bool unit_lower)
{
    float v[kNB * kNB / 256];
#pragma unroll
    for (int t = 0; t < kNB * kNB / 256; ++t)
    {
        const int e = threadIdx.x + 256 * t;
        const int i = e / kNB, p = e % kNB;
        v[t]        = (!unit_lower || p < i) ? a32[(int64_t)(r0 + i) * n + c0 + p] : 0.f;
    }
#pragma unroll
    for (int t = 0; t < kNB * kNB / 256; ++t)
    {
        const int e = threadIdx.x + 256 * t;
        Lb[e / kNB][e % kNB] = v[t];
    }
}

template <int KIND, bool SPLIT>
__global__ void __launch_bounds__(256) k_outer_u12(float* __restrict__ a32, int n, int K,
    typename OpStore<KIND>::type* __restrict__ opT, float* __restrict__ opT_small, float* __restrict__ inv_scale,
    int strip0)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float(*S)[kOuStrip + 1]  = reinterpret_cast<float(*)[kOuStrip + 1]>(smem_raw);  // [256]
    float(*Lb)[kLbLd]        = reinterpret_cast<float(*)[kLbLd]>(smem_raw + sizeof(float) * kOuterNB * (kOuStrip + 1));
    const int tid = threadIdx.x;
    const int cl  = tid % kOuStrip;
    const int rg  = tid / kOuStrip;  // 4 row groups
    const int Kend = K + kOuterNB;
    const int c0  = Kend + (strip0 + (int)blockIdx.x) * kOuStrip;
    const int col = c0 + cl;
    const bool valid = col < n;

    // the strip, 16 independent loads per thread in flight
    for (int i0 = rg; i0 < kOuterNB; i0 += 4 * 16)
    {
        float v[16];
#pragma unroll
        for (int t = 0; t < 16; ++t)
        {
            const int i = i0 + 4 * t;
            v[t]        = (valid && i < kOuterNB) ? a32[(int64_t)(K + i) * n + col] : 0.f;
        }
#pragma unroll
        for (int t = 0; t < 16; ++t)
        {
            const int i = i0 + 4 * t;
            if (i < kOuterNB)
            {
                S[i][cl] = v[t];
            }
        }
    }
    for (int jb = 0; jb < kOuterNB / kNB; ++jb)
    {
        __syncthreads();
        load_lblock(Lb, a32, n, K + jb * kNB, K + jb * kNB, true);
        // unit-lower diagonal block, column-oriented substitution
        for (int p = 0; p + 1 < kNB; ++p)
        {
            __syncthreads();
            const float xp = S[jb * kNB + p][cl];
            for (int i = p + 1 + rg; i < kNB; i += 4)
            {
                S[jb * kNB + i][cl] = fmaf(-Lb[i][p], xp, S[jb * kNB + i][cl]);
            }
        }
        for (int jb2 = jb + 1; jb2 < kOuterNB / kNB; ++jb2)
        {
            __syncthreads();
            load_lblock(Lb, a32, n, K + jb2 * kNB, K + jb * kNB, false);
            __syncthreads();
            // rows rg, rg+4, ... : each S value read once, L read as float4
            // broadcasts; per element the sum runs over p in order
            float acc[kNB / 4];
#pragma unroll
            for (int t = 0; t < kNB / 4; ++t)
            {
                acc[t] = 0.f;
            }
            for (int p = 0; p < kNB; p += 4)
            {
                const float s0 = S[jb * kNB + p][cl], s1 = S[jb * kNB + p + 1][cl];
                const float s2 = S[jb * kNB + p + 2][cl], s3 = S[jb * kNB + p + 3][cl];
#pragma unroll
                for (int t = 0; t < kNB / 4; ++t)
                {
                    const float4 l = *reinterpret_cast<const float4*>(&Lb[rg + 4 * t][p]);
                    acc[t]         = fmaf(l.x, s0, acc[t]);
                    acc[t]         = fmaf(l.y, s1, acc[t]);
                    acc[t]         = fmaf(l.z, s2, acc[t]);
                    acc[t]         = fmaf(l.w, s3, acc[t]);
                }
            }
#pragma unroll
            for (int t = 0; t < kNB / 4; ++t)
            {
                S[jb2 * kNB + rg + 4 * t][cl] -= acc[t];
            }
        }
    }
    __syncthreads();
    for (int i = rg; i < kOuterNB; i += 4)
    {
        if (valid)
        {
            a32[(int64_t)(K + i) * n + col] = S[i][cl];
        }
    }
    // FP8: power-of-two scale per column (per row of the transposed copy)
    __shared__ float colsc[kOuStrip];
    if constexpr (KIND == TC_FP8)
    {
        __shared__ float part[4][kOuStrip];
        float            amax = 0.f;
        for (int i = rg; i < kOuterNB; i += 4)
        {
            amax = fmaxf(amax, fabsf(S[i][cl]));
        }
        part[rg][cl] = amax;
        __syncthreads();
        if (rg == 0)
        {
            amax = fmaxf(fmaxf(part[0][cl], part[1][cl]), fmaxf(part[2][cl], part[3][cl]));
            float inv;
            colsc[cl] = fp8_scale(amax, &inv);
            if (valid)
            {
                inv_scale[col - Kend] = inv;
            }
        }
        __syncthreads();
    }
    // transposed operand copy: row (col - Kend), K index kk
    for (int e = tid; e < kOuStrip * kOuterNB; e += 256)
    {
        const int c  = e / kOuterNB;
        const int kk = e % kOuterNB;
        if (c0 + c < n)
        {
            float v = S[kk][c];
            if constexpr (KIND == TC_FP8)
            {
                v *= colsc[c];
            }
            const int64_t idx = (int64_t)(c0 + c - Kend) * kOuterNB + kk;
            opT[idx]          = OpStore<KIND>::conv(v);
            if constexpr (SPLIT)
            {
                opT_small[idx] = v - tf32_trunc(v);
            }
        }
    }
}

constexpr size_t outer_u12_smem() { return sizeof(float) * ((size_t)kOuterNB * (kOuStrip + 1) + kNB * kLbLd); }

// r = b - A x (one right-hand side), FP64; b == nullptr means b = 0.  A CTA
// handles 32 rows; x is staged through shared memory in chunks.  Also max|r|
// (atomic).
constexpr int kResRows  = 32;
constexpr int kResChunk = 2048;
__global__ void __launch_bounds__(256) k_residual(const double* __restrict__ a, int64_t lda,
    const double* __restrict__ x, const double* __restrict__ b, double* __restrict__ r, int n,
    unsigned long long* rmax)
{
    __shared__ double xs[kResChunk];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row0 = blockIdx.x * kResRows + warp * 4;
    double    acc[4] = {0, 0, 0, 0};
    for (int c0 = 0; c0 < n; c0 += kResChunk)
    {
        const int cw = min(kResChunk, n - c0);
        __syncthreads();
        for (int j = threadIdx.x; j < cw; j += 256)
        {
            xs[j] = x[c0 + j];
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 4; ++q)
        {
            const int row = row0 + q;
            if (row < n)
            {
                const double* ar = a + (int64_t)row * lda + c0;
                double        s  = 0.0;
                for (int j = lane; j < cw; j += 32)
                {
                    s = fma(ar[j], xs[j], s);
                }
                acc[q] += s;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
    {
        double s = acc[q];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            s += __shfl_down_sync(0xffffffffu, s, off);
        }
        const int row = row0 + q;
        if (lane == 0 && row < n)
        {
            const double v = (b != nullptr ? b[row] : 0.0) - s;
            r[row]         = v;
            atomic_max_nonneg(rmax, fabs(v));
        }
    }
}

// Per-column max |v| of an n x m row-major block (ld), into out[m].
__global__ void k_colmax(const double* __restrict__ v, int64_t ld, int n, int m, unsigned long long* out)
{
    const int64_t total = (int64_t)n * m;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t r = e / m;
        const int     c = (int)(e - r * m);
        atomic_max_nonneg(out + c, fabs(v[r * ld + c]));
    }
}

// x += d (n x m, row strides ldx / ldd)
__global__ void k_axpy2d(double* __restrict__ x, int64_t ldx, const double* __restrict__ d, int64_t ldd, int n, int m)
{
    const int64_t total = (int64_t)n * m;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    {
        const int64_t r = e / m;
        const int     c = (int)(e - r * m);
        x[r * ldx + c] += d[r * ldd + c];
    }
}

// ---- GMRES helpers (one right-hand side) ----------------------------------
// h[i] += sum_r V[i][r] w[r] for i < m (V: m vectors of n, contiguous)
__global__ void k_dots(const double* __restrict__ V, const double* __restrict__ w, int n, int m, double* h)
{
    const int i = blockIdx.y;
    double    s = 0.0;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    {
        s = fma(V[(int64_t)i * n + r], w[r], s);
    }
    __shared__ double red[8];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        s += __shfl_down_sync(0xffffffffu, s, off);
    }
    if ((threadIdx.x & 31) == 0)
    {
        red[threadIdx.x >> 5] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double t = 0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q)
        {
            t += red[q];
        }
        atomicAdd(h + i, t);
    }
}

// w[r] -= sum_{i<m} h[i] V[i][r]   (or, with sign +1 and w = 0, w = V h)
__global__ void k_comb(const double* __restrict__ V, const double* __restrict__ h, int n, int m, double sign,
    double* __restrict__ w)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    {
        double s = 0.0;
        for (int i = 0; i < m; ++i)
        {
            s = fma(h[i], V[(int64_t)i * n + r], s);
        }
        w[r] += sign * s;
    }
}

__global__ void k_scale_copy(const double* __restrict__ src, double alpha, double* __restrict__ dst, int n)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x)
    {
        dst[r] = alpha * src[r];
    }
}

// ---------------------------------------------------------------------------
// host
// ---------------------------------------------------------------------------
inline int grid_for(int64_t total, int threads = 256)
{
    int64_t g = (total + threads - 1) / threads;
    if (g < 1)
        g = 1;
    if (g > 148 * 8)
        g = 148 * 8;
    return (int)g;
}

struct MixedPlan
{
    GetrfPlan<float>   gp;
    float*             a32;
    int64_t*           piv;
    void*              l21op;
    float*             l21small;
    void*              u12op;
    float*             u12small;
    int32_t*           perm;
    double*            r;       // n x nrhs residual / correction
    double*            y;       // n x nrhs scratch for the solves
    unsigned long long* norms;  // [0] ||A||, [1..] per-column maxima (3 x 64)
    TrsvSync*          tsync;
    double*            dinv;    // inverses of the 128 x 128 diagonal blocks of L and U
    uint64_t*          xll;     // flagged copies of solved blocks (k_trsv_blocks)
    double*            V;       // GMRES basis (m+1) x n
    double*            h;       // GMRES dot products (m+1)
    PermList*          perms;   // interchange lists of the panels of two outer blocks (by block parity)
    float*             sel;     // selector network input (12) and output (4)
    float*             l21inv;  // FP8: inverse row scales of L21
    float*             u12inv;  // FP8: inverse row scales of U12^T
    double*            a64;     // FP64 copy of A for the FP64 fallback
    GetrfPlan<double>  gp64;
    int64_t*           piv64;
};

constexpr int kMaxNrhsMixed = 64;

constexpr int kGmresMaxRestart = 50;

MixedPlan plan_mixed(Arena& a, int64_t n, int64_t nrhs, int restart, bool fp64_fallback)
{
    MixedPlan p{};
    p.gp       = plan_getrf<float>(a);
    p.a32      = a.next<float>((size_t)n * n);
    p.piv      = a.next<int64_t>((size_t)n);
    p.l21op    = a.next<float>((size_t)n * kOuterNB);
    p.l21small = a.next<float>((size_t)n * kOuterNB);
    p.u12op    = a.next<float>((size_t)n * kOuterNB);
    p.u12small = a.next<float>((size_t)n * kOuterNB);
    p.perm     = a.next<int32_t>((size_t)n);
    p.perms    = a.next<PermList>(2 * kMaxBlockPanels);
    p.sel      = a.next<float>(64);
    p.l21inv   = a.next<float>((size_t)n);
    p.u12inv   = a.next<float>((size_t)n);
    p.r        = a.next<double>((size_t)n * nrhs);
    p.y        = a.next<double>((size_t)n * nrhs);
    p.norms    = a.next<unsigned long long>(4 + 3 * kMaxNrhsMixed + 16);
    p.tsync    = reinterpret_cast<TrsvSync*>(a.next<int32_t>(32 + (size_t)(n + kTvRows - 1) / kTvRows + 32));
    p.dinv     = a.next<double>((size_t)((n + kTrRows - 1) / kTrRows) * 2 * kTrRows * kTrRows);
    p.xll      = a.next<uint64_t>((size_t)((n + kTvRows - 1) / kTvRows) * kTvRows * 2);
    const int m = restart > 0 ? restart : 0;
    p.V        = a.next<double>((size_t)(m + 1) * n);
    p.h        = a.next<double>((size_t)m + 2);
    if (fp64_fallback)
    {
        p.a64   = a.next<double>((size_t)n * n);
        p.gp64  = plan_getrf<double>(a);
        p.piv64 = a.next<int64_t>((size_t)n);
    }
    return p;
}

// rowid[i] = i: the row permutation of the factorization, tracked as it
// happens (row i of P A is row rowid[i] of A).
__global__ void k_iota(int32_t* __restrict__ rowid, int n)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
        rowid[i] = (int32_t)i;
    }
}

// Applies the interchange lists of an outer block's panels, in order, to
// rowid (the same gather/scatter the interchanges do to a column).  One CTA.
__global__ void k_rowid_apply(int32_t* __restrict__ rowid, const PermList* __restrict__ perms, int npanels)
{
    for (int j = 0; j < npanels; ++j)
    {
        const PermList* pl  = perms + j;
        const int       cnt = pl->count;
        int32_t         v   = 0;
        if ((int)threadIdx.x < cnt)
        {
            v = rowid[pl->src[threadIdx.x]];
        }
        __syncthreads();
        if ((int)threadIdx.x < cnt)
        {
            rowid[pl->dst[threadIdx.x]] = v;
        }
        __syncthreads();
    }
}

// An outer block's row interchanges on columns [c_begin, c_end): CTA = 64
// columns; the panels' interchange lists are applied in order, each as one
// gather of the rows it touches and one scatter.
constexpr int kBlockSwapThreads = 256;
constexpr int kBlockSwapGroups  = kBlockSwapThreads / kSwapCols;
__global__ void __launch_bounds__(kBlockSwapThreads) k_laswp_block(float* __restrict__ a32, int n,
    const PermList* __restrict__ perms, int npanels, int c_begin, int c_end)
{
    __shared__ float staged[2 * kNB][kSwapCols];
    const int  tid   = threadIdx.x;
    const int  cl    = tid % kSwapCols;
    const int  rg    = tid / kSwapCols;
    const int  col   = c_begin + (int)blockIdx.x * kSwapCols + cl;
    const bool valid = col < c_end;
    constexpr int PT = 2 * kNB / kBlockSwapGroups;
    for (int j = 0; j < npanels; ++j)
    {
        const PermList* pl  = perms + j;
        const int       cnt = pl->count;
        float           v[PT];
#pragma unroll
        for (int t = 0; t < PT; ++t)
        {
            const int q = rg + kBlockSwapGroups * t;
            v[t]        = (valid && q < cnt) ? a32[(size_t)pl->src[q] * n + col] : 0.f;
        }
#pragma unroll
        for (int t = 0; t < PT; ++t)
        {
            staged[rg + kBlockSwapGroups * t][cl] = v[t];
        }
        __syncthreads();
        if (valid)
        {
            for (int q = rg; q < cnt; q += kBlockSwapGroups)
            {
                if (pl->dst[q] != pl->src[q])
                {
                    a32[(size_t)pl->dst[q] * n + col] = staged[q][cl];
                }
            }
        }
        __syncthreads();
    }
}

// The interchange lists of outer block K's panels (two sets, by the block's
// parity, so a block's lists stay valid while the next block's panels run).
inline PermList* block_perms(MixedPlan& p, int K) { return p.perms + ((K / kOuterNB) & 1) * kMaxBlockPanels; }

// Panel width of the outer blocks: 32 columns whenever a 32-column panel of
// the block fits one cluster's shared memory (every order up to about
// 25,000), else 64 on the grid-wide kernel.  32-column panels hold twice the
// rows of 64-column ones in a cluster, cost a little less per column, and
// one width for the whole factorization keeps its rounding the same from
// block to block (measured at n = 16384: 5 refinement corrections, against 7
// when the blocks whose 64-column panels fit used those).
// B200LA_MIXED_PANEL_WIDTH=64 keeps 64-column panels where they fit.
int block_panel_width(int n, int K)
{
    int cl = 0, gmax = 0;
    if (panel_config<float>(cl, gmax) != B200LA_SUCCESS || cl == 0)
        return 64;
    const char* e = getenv("B200LA_MIXED_PANEL_WIDTH");
    if (e != nullptr && e[0] == '6' && cluster_panel_fits<float>(n - K, 64, cl))
        return 64;
    return cluster_panel_fits<float>(n - K, 32, cl) ? 32 : 64;
}

inline int block_panel_count(int n, int K, int Kend)
{
    const int pw = block_panel_width(n, K);
    return (Kend - K + pw - 1) / pw;
}

// Nested look-ahead inside a block (B200LA_MIXED_NESTED=0: off).
bool nested_enabled()
{
    const char* e = getenv("B200LA_MIXED_NESTED");
    return !(e != nullptr && e[0] == '0');
}

// Inner panels of the outer block [K, Kend): panels of block_panel_width
// columns, their row interchanges on columns [K, Kend) (left of the block
// they are applied later by enqueue_block_left_swaps, right of it after the
// block by enqueue_block_swaps), U12 inside the block and the SIMT updates
// inside the block.  Panel j's interchange list goes to block_perms(p, K)[j].
//
// With a second stream `rs` and the events ev_p, ev_r[2] (nested
// look-ahead), the work after panel j is split: the next panel's columns
// (interchanges, U12, update) are applied by the next panel kernel itself
// when it is the FP32 32-column cluster kernel (else by the two kernels
// right before it on `s`), and the block's other columns (the interchanges
// left of the panel, the columns after the next panel) go to `rs`, so panel
// j + 1 starts as soon as panel j is done and the rest of panel j - 1 has
// reached its columns.  The streams touch disjoint columns; `s` waits for
// the block's last rest before it returns.
int enqueue_block_panels(MixedPlan& p, int n, int K, int Kend, int cl, int gmax, cudaStream_t s,
    cudaStream_t rs = nullptr, cudaEvent_t ev_p = nullptr, cudaEvent_t* ev_r = nullptr)
{
    float*     a32  = p.a32;
    int        rc   = B200LA_SUCCESS;
    const int  pw   = block_panel_width(n, K);
    const bool nest = rs != nullptr && rs != s && ev_p != nullptr && ev_r != nullptr && nested_enabled();
    auto swaps = [&](const PermList* perm, int k, int w, int left_cols, int rb, int re, cudaStream_t st) {
        const int nl = (left_cols + kSwapCols - 1) / kSwapCols;
        const int nr = re > rb ? (re - rb + kSwapCols - 1) / kSwapCols : 0;
        if (nl + nr > 0)
        {
            prof_begin(KC_SWAP, st);
            k_laswp_trsm<float><<<nl + nr, kSwapThreads, laswp_smem_bytes<float>(), st>>>(a32, n, k, w, perm, nl,
                Kend, K, K + left_cols, re, rb);
            prof_end(KC_SWAP, st);
        }
    };
    auto update = [&](int k, int w, int c_off, int ncols, cudaStream_t st) {
        const int rest = n - k - w;
        if (rest > 0 && ncols > 0)
        {
            dim3 grid((ncols + kChunkN - 1) / kChunkN, (rest + kBandM - 1) / kBandM);
            prof_begin(KC_TRAILING, st);
            k_trailing<float><<<grid, 128, trailing_smem_bytes<float>(), st>>>(a32, n, k, w, ncols, c_off);
            prof_end(KC_TRAILING, st);
        }
    };
    int last = -1;
    for (int k = K, j = 0; k < Kend; k += pw, ++j)
    {
        const int        w  = Kend - k < pw ? Kend - k : pw;
        GetrfPlan<float> gp = p.gp;
        gp.perm             = block_perms(p, K) + j;
        const int kn        = k + w;  // the next panel's columns [kn, kn2)
        const int kn2       = kn + pw < Kend ? kn + pw : Kend;
        if (!nest)
        {
            if ((rc = launch_panel<float>(a32, n, k, w, p.piv, gp, cl, gmax, s)) != B200LA_SUCCESS)
                return rc;
            swaps(gp.perm, k, w, k - K, kn, Kend, s);
            B200LA_LAUNCH_CHECK();
            update(k, w, 0, Kend - kn, s);
            B200LA_LAUNCH_CHECK();
            continue;
        }
        if (j >= 2)
        {
            B200LA_CUDA(cudaStreamWaitEvent(s, ev_r[j & 1], 0));  // the rest of panel j - 2
        }
        const PermList* prev = j >= 1 ? block_perms(p, K) + (j - 1) : nullptr;
        const bool      fuse = prev != nullptr && panel_can_fuse<float>(n - k, w, pw, cl);
        if (prev != nullptr && !fuse)
        {
            // panel j - 1's work on this panel's columns, before it
            swaps(prev, k - pw, pw, 0, k, kn, s);
            B200LA_LAUNCH_CHECK();
            update(k - pw, pw, 0, w, s);
            B200LA_LAUNCH_CHECK();
        }
        if ((rc = launch_panel<float>(a32, n, k, w, p.piv, gp, cl, gmax, s, false, fuse ? prev : nullptr,
                 fuse ? k - pw : -1)) != B200LA_SUCCESS)
            return rc;
        B200LA_CUDA(cudaEventRecord(ev_p, s));
        B200LA_CUDA(cudaStreamWaitEvent(rs, ev_p, 0));
        swaps(gp.perm, k, w, k - K, kn2, Kend, rs);
        B200LA_LAUNCH_CHECK();
        update(k, w, kn2 - kn, Kend - kn2, rs);
        B200LA_LAUNCH_CHECK();
        B200LA_CUDA(cudaEventRecord(ev_r[j & 1], rs));
        last = j;
    }
    if (nest && last >= 0)
    {
        B200LA_CUDA(cudaStreamWaitEvent(s, ev_r[last & 1], 0));
    }
    return B200LA_SUCCESS;
}

// The outer block's row interchanges on columns [c_begin, c_end) (right of
// the block), all its panels in one launch.
int enqueue_block_swaps(MixedPlan& p, int n, int K, int Kend, int c_begin, int c_end, cudaStream_t s)
{
    const int cols = c_end - c_begin;
    if (cols <= 0)
        return B200LA_SUCCESS;
    prof_begin(KC_SWAP, s);
    k_laswp_block<<<(cols + kSwapCols - 1) / kSwapCols, kBlockSwapThreads, 0, s>>>(p.a32, n, block_perms(p, K),
        block_panel_count(n, K, Kend), c_begin, c_end);
    prof_end(KC_SWAP, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

// The outer block's interchanges on the columns left of it, [0, K).
int enqueue_block_left_swaps(MixedPlan& p, int n, int K, int Kend, cudaStream_t s)
{
    return enqueue_block_swaps(p, n, K, Kend, 0, K, s);
}

// The outer block's interchanges applied to the row permutation.
int enqueue_block_rowid(MixedPlan& p, int n, int K, int Kend, cudaStream_t s)
{
    k_rowid_apply<<<1, 2 * kNB, 0, s>>>(p.perm, block_perms(p, K), block_panel_count(n, K, Kend));
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

// A stream per device and slot (high priority for the look-ahead panels and,
// slot 1, the rest of each panel's block work; low for the interchanges left
// of a block, which nothing reads before the solve).
cudaStream_t lookahead_stream(int* rc, bool high = true, int slot = 0)
{
    static std::mutex   m;
    static cudaStream_t all_streams[3][64] = {};
    cudaStream_t*       streams            = all_streams[high ? (slot != 0 ? 2 : 0) : 1];
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
    std::lock_guard<std::mutex> lock(m);
    if (streams[dev] == nullptr)
    {
        int least = 0, greatest = 0;
        cudaDeviceGetStreamPriorityRange(&least, &greatest);
        e = cudaStreamCreateWithPriority(&streams[dev], cudaStreamNonBlocking, high ? greatest : least);
        if (e != cudaSuccess)
        {
            streams[dev] = nullptr;
            *rc          = cuda_check(e, "cudaStreamCreateWithPriority");
            return nullptr;
        }
    }
    return streams[dev];
}

bool lookahead_enabled()
{
    const char* e = getenv("B200LA_MIXED_LOOKAHEAD");
    return !(e != nullptr && e[0] == '0');
}

// The outer block's operand copies for strips [strip0, strip0 + count) of
// U12 (64 columns each) and, with `l21`, the L21 copy (all rows).
void enqueue_block_operands(MixedPlan& p, int n, int K, int Kend, int rest, int kind, bool split, int strip0,
    int count, bool l21, cudaStream_t s)
{
    float*        a32   = p.a32;
    const int64_t elems = (int64_t)rest * kOuterNB;
    if (kind == TC_TF32 && split)
    {
        if (l21)
            k_make_l21<TC_TF32, true><<<grid_for(elems), 256, 0, s>>>(a32, n, K, Kend, (float*)p.l21op, p.l21small);
        if (count > 0)
            k_outer_u12<TC_TF32, true><<<count, 256, outer_u12_smem(), s>>>(a32, n, K, (float*)p.u12op, p.u12small, nullptr, strip0);
    }
    else if (kind == TC_TF32)
    {
        if (l21)
            k_make_l21<TC_TF32, false><<<grid_for(elems), 256, 0, s>>>(a32, n, K, Kend, (float*)p.l21op, nullptr);
        if (count > 0)
            k_outer_u12<TC_TF32, false><<<count, 256, outer_u12_smem(), s>>>(a32, n, K, (float*)p.u12op, nullptr, nullptr, strip0);
    }
    else if (kind == TC_BF16)
    {
        if (l21)
            k_make_l21<TC_BF16, false><<<grid_for(elems), 256, 0, s>>>(a32, n, K, Kend, (__nv_bfloat16*)p.l21op, nullptr);
        if (count > 0)
            k_outer_u12<TC_BF16, false><<<count, 256, outer_u12_smem(), s>>>(a32, n, K, (__nv_bfloat16*)p.u12op, nullptr, nullptr, strip0);
    }
    else if (kind == TC_FP16)
    {
        if (l21)
            k_make_l21<TC_FP16, false><<<grid_for(elems), 256, 0, s>>>(a32, n, K, Kend, (__half*)p.l21op, nullptr);
        if (count > 0)
            k_outer_u12<TC_FP16, false><<<count, 256, outer_u12_smem(), s>>>(a32, n, K, (__half*)p.u12op, nullptr, nullptr, strip0);
    }
    else
    {
        if (l21)
            k_make_l21_fp8<<<grid_for((int64_t)rest * 32), 256, 0, s>>>(a32, n, K, Kend, (__nv_fp8_storage_t*)p.l21op, p.l21inv);
        if (count > 0)
            k_outer_u12<TC_FP8, false><<<count, 256, outer_u12_smem(), s>>>(a32, n, K, (__nv_fp8_storage_t*)p.u12op, nullptr, p.u12inv, strip0);
    }
}

// The tensor-core trailing update of the outer block (columns [c0, n) of
// A22 = rows and columns from Kend), operands from the block's copies.
int enqueue_block_update(MixedPlan& p, int n, int Kend, int c0, int kind, bool split, const CUtensorMap& ma,
    const CUtensorMap& mb, const CUtensorMap& mas, const CUtensorMap& mbs, int ncols, cudaStream_t s,
    int max_ctas = 0, int place_cluster = 0)
{
    const int rest = n - Kend;
    return enqueue_tc_update(kind, split, ma, mb, mas, mbs, p.a32 + (int64_t)Kend * n + c0, n, rest, ncols, kOuterNB,
        p.gp.st, s, p.l21inv, p.u12inv + (c0 - Kend), max_ctas, place_cluster);
}

// CTAs of the persistent tensor-core update that runs beside the next
// block's panels: the SMs less those the panel cluster and the panels'
// in-block kernels use (B200LA_MIXED_UPDATE_CTAS overrides).
// The update beside the panels is launched as clusters of this many CTAs
// (whole GPCs, one left free for the panel's cluster); 0 (variable
// B200LA_MIXED_UPDATE_CLUSTER=0) launches it without placement.
int beside_panel_cluster()
{
    const char* e = getenv("B200LA_MIXED_UPDATE_CLUSTER");
    if (e != nullptr)
        return atoi(e) > 1 && atoi(e) <= 16 ? atoi(e) : 0;
    return 16;
}

int beside_panel_ctas()
{
    const char* e = getenv("B200LA_MIXED_UPDATE_CTAS");
    if (e != nullptr && atoi(e) > 0)
        return atoi(e);
    const int sms = device_sm_count();
    return sms > 40 ? sms - 24 : sms;
}

// Mixed-precision factorization of p.a32 in place; pivots in p.piv.
//
// Look-ahead: outer block K first gets only what the next block's panels
// need (its interchanges, U12 strips and operand copies for the next block's
// 256 columns, and those columns' tensor-core update); the next block's
// panels then run on a high-priority stream while the rest of block K's
// interchanges, U12 strips and update run on `s`.  The next block's
// interchanges right of it wait until that update is done, so both streams
// touch disjoint columns; every per-element operation is the same as
// without look-ahead.
int enqueue_getrf_mixed(MixedPlan& p, int n, int kind, bool split, cudaStream_t s)
{
    int rc = clear_panel_exchange<float>(p.gp, s);
    if (rc != B200LA_SUCCESS)
        return rc;
    k_status_init<<<1, 32, 0, s>>>(p.gp.st, p.gp.perm);
    k_iota<<<grid_for(n), 256, 0, s>>>(p.perm, n);
    B200LA_LAUNCH_CHECK();
    int cl = 0, gmax = 0;
    if ((rc = panel_config<float>(cl, gmax)) != B200LA_SUCCESS)
        return rc;
    const int  elem = tc_elem_bytes(kind);
    const bool la   = lookahead_enabled() && n > 2 * kOuterNB;
    CUtensorMap ma, mb, mas, mbs, mb2, mbs2;
    if ((rc = make_kmajor_map(&ma, p.l21op, kind, n, kOuterNB, kOuterNB, kTcBM)) != B200LA_SUCCESS ||
        (rc = make_kmajor_map(&mb, p.u12op, kind, n, kOuterNB, kOuterNB, kTcBN)) != B200LA_SUCCESS)
        return rc;
    mas = ma;
    mbs = mb;
    if (split && ((rc = make_kmajor_map(&mas, p.l21small, TC_TF32, n, kOuterNB, kOuterNB, kTcBM)) != B200LA_SUCCESS ||
                     (rc = make_kmajor_map(&mbs, p.u12small, TC_TF32, n, kOuterNB, kOuterNB, kTcBN)) != B200LA_SUCCESS))
        return rc;
    mb2  = mb;
    mbs2 = mbs;
    if (la)
    {
        // B operand rows from the second 256 on (the columns right of the next block)
        const size_t off = (size_t)kOuterNB * kOuterNB;
        if ((rc = make_kmajor_map(&mb2, static_cast<unsigned char*>(p.u12op) + off * elem, kind, n - kOuterNB,
                 kOuterNB, kOuterNB, kTcBN)) != B200LA_SUCCESS)
            return rc;
        if (split && (rc = make_kmajor_map(&mbs2, p.u12small + off, TC_TF32, n - kOuterNB, kOuterNB, kOuterNB,
                          kTcBN)) != B200LA_SUCCESS)
            return rc;
    }
    cudaStream_t side = s, left = s, rest_s = nullptr;
    cudaEvent_t  ev_update = nullptr, ev_panels = nullptr, ev_left[2] = {nullptr, nullptr};
    cudaEvent_t  ev_np = nullptr, ev_nr[2] = {nullptr, nullptr};  // nested look-ahead inside a block
    if (la)
    {
        side = lookahead_stream(&rc);
        if (rc != B200LA_SUCCESS)
            return rc;
        left = lookahead_stream(&rc, false);
        if (rc != B200LA_SUCCESS)
            return rc;
        rest_s = lookahead_stream(&rc, true, 1);
        if (rc != B200LA_SUCCESS)
            return rc;
        B200LA_CUDA(cudaEventCreateWithFlags(&ev_update, cudaEventDisableTiming));
        B200LA_CUDA(cudaEventCreateWithFlags(&ev_panels, cudaEventDisableTiming));
        B200LA_CUDA(cudaEventCreateWithFlags(&ev_left[0], cudaEventDisableTiming));
        B200LA_CUDA(cudaEventCreateWithFlags(&ev_left[1], cudaEventDisableTiming));
        B200LA_CUDA(cudaEventCreateWithFlags(&ev_np, cudaEventDisableTiming));
        B200LA_CUDA(cudaEventCreateWithFlags(&ev_nr[0], cudaEventDisableTiming));
        B200LA_CUDA(cudaEventCreateWithFlags(&ev_nr[1], cudaEventDisableTiming));
    }
    struct EventGuard
    {
        cudaEvent_t e[7];
        ~EventGuard()
        {
            for (cudaEvent_t x : e)
                if (x)
                    cudaEventDestroy(x);
        }
    } guard{{ev_update, ev_panels, ev_left[0], ev_left[1], ev_np, ev_nr[0], ev_nr[1]}};
    // interchanges left of block K once its panels are done (`done_on`:
    // where they ran); the event guards the interchange lists' slot
    auto left_swaps = [&](int K, int Kend, cudaStream_t done_on) -> int {
        if (K <= 0)
            return B200LA_SUCCESS;
        if (la)
        {
            B200LA_CUDA(cudaStreamWaitEvent(left, done_on == s ? ev_update : ev_panels, 0));
        }
        int r = enqueue_block_left_swaps(p, n, K, Kend, left);
        if (r == B200LA_SUCCESS && la)
        {
            B200LA_CUDA(cudaEventRecord(ev_left[(K / kOuterNB) & 1], left));
        }
        return r;
    };

    float* a32 = p.a32;
    if ((rc = enqueue_block_panels(p, n, 0, n < kOuterNB ? n : kOuterNB, cl, gmax, s, rest_s, ev_np, ev_nr)) !=
        B200LA_SUCCESS)
        return rc;
    bool panels_on_side = false;
    for (int K = 0; K < n; K += kOuterNB)
    {
        const int Kend = K + kOuterNB < n ? K + kOuterNB : n;
        if (panels_on_side)
        {
            B200LA_CUDA(cudaStreamWaitEvent(s, ev_panels, 0));
            panels_on_side = false;
        }
        if ((rc = enqueue_block_rowid(p, n, K, Kend, s)) != B200LA_SUCCESS)
            return rc;
        const int rest = n - Kend;
        if (rest <= 0)
        {
            continue;
        }
        const int  Kend2 = Kend + kOuterNB < n ? Kend + kOuterNB : n;
        const bool ahead = la && Kend2 < n;
        // with look-ahead, first only what the next block's panels need: its
        // columns' interchanges and U12 strips, then its columns' update
        const int  c_first = ahead ? Kend2 : n;
        if ((rc = enqueue_block_swaps(p, n, K, Kend, Kend, c_first, s)) != B200LA_SUCCESS)
            return rc;
        const int nstrips = (rest + kOuStrip - 1) / kOuStrip;
        const int first   = ahead ? (Kend2 - Kend) / kOuStrip : nstrips;
        prof_begin(KC_PREP, s);
        enqueue_block_operands(p, n, K, Kend, rest, kind, split, 0, first, true, s);
        prof_end(KC_PREP, s);
        B200LA_LAUNCH_CHECK();
        if (ahead)
        {
            if ((rc = enqueue_block_update(p, n, Kend, Kend, kind, split, ma, mb, mas, mbs, Kend2 - Kend, s)) !=
                B200LA_SUCCESS)
                return rc;
            B200LA_CUDA(cudaEventRecord(ev_update, s));
            B200LA_CUDA(cudaStreamWaitEvent(side, ev_update, 0));
            // the lists' slot of block K+1 was last used by block K-1's
            // left-of-block interchanges
            if (K > 0)
            {
                B200LA_CUDA(cudaStreamWaitEvent(side, ev_left[((K / kOuterNB) + 1) & 1], 0));
            }
            if ((rc = enqueue_block_panels(p, n, Kend, Kend2, cl, gmax, side, rest_s, ev_np, ev_nr)) != B200LA_SUCCESS)
                return rc;
            B200LA_CUDA(cudaEventRecord(ev_panels, side));
            panels_on_side = true;
            if ((rc = left_swaps(Kend, Kend2, side)) != B200LA_SUCCESS)
                return rc;
            // the rest, beside the next block's panels
            if ((rc = enqueue_block_swaps(p, n, K, Kend, Kend2, n, s)) != B200LA_SUCCESS)
                return rc;
            prof_begin(KC_PREP, s);
            enqueue_block_operands(p, n, K, Kend, rest, kind, split, first, nstrips - first, false, s);
            prof_end(KC_PREP, s);
            B200LA_LAUNCH_CHECK();
            if ((rc = enqueue_block_update(p, n, Kend, Kend2, kind, split, ma, mb2, mas, mbs2, n - Kend2, s,
                     beside_panel_ctas(), beside_panel_cluster())) !=
                B200LA_SUCCESS)
                return rc;
        }
        else
        {
            if ((rc = enqueue_block_update(p, n, Kend, Kend, kind, split, ma, mb, mas, mbs, rest, s)) != B200LA_SUCCESS)
                return rc;
            if (la && K > 0)
            {
                B200LA_CUDA(cudaStreamWaitEvent(s, ev_left[((K / kOuterNB) + 1) & 1], 0));
            }
            if ((rc = enqueue_block_panels(p, n, Kend, Kend2, cl, gmax, s, rest_s, ev_np, ev_nr)) != B200LA_SUCCESS)
                return rc;
            if (la)
            {
                B200LA_CUDA(cudaEventRecord(ev_update, s));
            }
            if ((rc = left_swaps(Kend, Kend2, s)) != B200LA_SUCCESS)
                return rc;
        }
    }
    if (la)
    {
        // the solve needs every interchange applied
        B200LA_CUDA(cudaEventRecord(ev_left[0], left));
        B200LA_CUDA(cudaStreamWaitEvent(s, ev_left[0], 0));
    }
    k_status_finish<<<1, 32, 0, s>>>(p.gp.st);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

int set_mixed_attributes()
{
    static std::mutex m;
    static bool       done[64] = {};
    int               dev      = 0;
    B200LA_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(m);
    if (dev >= 0 && dev < 64 && done[dev])
        return B200LA_SUCCESS;
    B200LA_CUDA(cudaFuncSetAttribute(k_outer_u12<TC_TF32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)outer_u12_smem()));
    B200LA_CUDA(cudaFuncSetAttribute(k_outer_u12<TC_TF32, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)outer_u12_smem()));
    B200LA_CUDA(cudaFuncSetAttribute(k_outer_u12<TC_BF16, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)outer_u12_smem()));
    B200LA_CUDA(cudaFuncSetAttribute(k_outer_u12<TC_FP16, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)outer_u12_smem()));
    B200LA_CUDA(cudaFuncSetAttribute(k_outer_u12<TC_FP8, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)outer_u12_smem()));
    B200LA_CUDA(cudaFuncSetAttribute(k_trsv_refine<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrInvSmem));
    B200LA_CUDA(cudaFuncSetAttribute(k_trsv_refine<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrInvSmem));
    B200LA_CUDA(cudaFuncSetAttribute(k_trsm_refine<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTmSmem));
    B200LA_CUDA(cudaFuncSetAttribute(k_trsm_refine<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTmSmem));
    B200LA_CUDA(cudaFuncSetAttribute(k_invert_diag_blocks128<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrInvSmem));
    B200LA_CUDA(cudaFuncSetAttribute(k_invert_diag_blocks128<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrInvSmem));
    if (dev >= 0 && dev < 64)
        done[dev] = true;
    return B200LA_SUCCESS;
}

// v (n x nrhs, row stride ldv) <- U^-1 L^-1 P v with the factors `lu`
// (float or double) applied in FP64.  Uses p.y as scratch.
template <typename TA>
int enqueue_lu_apply(const TA* lu, const int32_t* perm, int n, int nrhs, double* v, int64_t ldv, MixedPlan& p,
    DeviceStatus* st, cudaStream_t s)
{
    const int64_t total = (int64_t)n * nrhs;
    prof_begin(KC_SOLVE, s);
    k_gather_rows<double><<<grid_for(total), 256, 0, s>>>(v, ldv, perm, p.y, nrhs, n, nrhs, nullptr);
    prof_end(KC_SOLVE, s);
    B200LA_LAUNCH_CHECK();
    if (nrhs == 1)
    {
        const int nb = (n + kTrRows - 1) / kTrRows;
        for (int pass = 0; pass < 2; ++pass)
        {
            B200LA_CUDA(cudaMemsetAsync(p.tsync, 0, sizeof(int32_t), s));
            const uint32_t epoch = tv_next_epoch();
            prof_begin(KC_SOLVE, s);
            k_trsv_refine<TA><<<nb, kTrThreads, kTrInvSmem, s>>>(lu, n, p.y, n, pass, p.dinv, p.xll, epoch,
                reinterpret_cast<int32_t*>(p.tsync), st, kWaitLimitNs);
            prof_end(KC_SOLVE, s);
            B200LA_LAUNCH_CHECK();
        }
    }
    else if (nrhs <= kTmRhs)
    {
        // one launch per triangle, all right-hand sides per 128-row block;
        // flags[] (one word per block) live in the flagged-word buffer
        const int nb = (n + kTrRows - 1) / kTrRows;
        for (int pass = 0; pass < 2; ++pass)
        {
            B200LA_CUDA(cudaMemsetAsync(p.tsync, 0, sizeof(int32_t), s));
            const uint32_t epoch = tv_next_epoch();
            prof_begin(KC_SOLVE, s);
            k_trsm_refine<TA><<<nb, kTmThreads, kTmSmem, s>>>(lu, n, p.y, n, nrhs, pass, p.dinv,
                reinterpret_cast<uint32_t*>(p.xll), epoch, reinterpret_cast<int32_t*>(p.tsync), st, kWaitLimitNs);
            prof_end(KC_SOLVE, s);
            B200LA_LAUNCH_CHECK();
        }
    }
    else
    {
        int rc = enqueue_trsm_inplace<TA, double>(false, false, true, n, nrhs, lu, n, p.y, nrhs, nullptr, s);
        if (rc != B200LA_SUCCESS)
            return rc;
        rc = enqueue_trsm_inplace<TA, double>(true, false, false, n, nrhs, lu, n, p.y, nrhs, nullptr, s);
        if (rc != B200LA_SUCCESS)
            return rc;
    }
    prof_begin(KC_SOLVE, s);
    k_copy2d<double><<<grid_for(total), 256, 0, s>>>(p.y, nrhs, v, ldv, n, nrhs, nullptr);
    prof_end(KC_SOLVE, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

// r = b - A x and eta_j = ||r_j|| / (||A|| ||x_j|| + ||b_j||); returns max_j eta_j.
int residual_eta(const double* a, int64_t lda, int n, int nrhs, const double* b, int64_t ldb, const double* x,
    int64_t ldx, MixedPlan& p, double anorm, const std::vector<double>& bnorm, double* eta, cudaStream_t s)
{
    B200LA_CUDA(cudaMemsetAsync(p.norms + 4, 0, sizeof(unsigned long long) * 3 * kMaxNrhsMixed, s));
    if (nrhs == 1)
    {
        prof_begin(KC_RESIDUAL, s);
        k_residual<<<(n + kResRows - 1) / kResRows, 256, 0, s>>>(a, lda, x, b, p.r, n, p.norms + 4);
        prof_end(KC_RESIDUAL, s);
        B200LA_LAUNCH_CHECK();
        prof_begin(KC_RESIDUAL, s);
        k_colmax<<<grid_for(n), 256, 0, s>>>(x, ldx, n, 1, p.norms + 4 + kMaxNrhsMixed);
        prof_end(KC_RESIDUAL, s);
    }
    else
    {
        // R = B - A X on the FP64 GEMM
        prof_begin(KC_RESIDUAL, s);
        k_copy2d<double><<<grid_for((int64_t)n * nrhs), 256, 0, s>>>(b, ldb, p.r, nrhs, n, nrhs, nullptr);
        prof_end(KC_RESIDUAL, s);
        // the FP64 tensor-core GEMM of the multiplication row (its launches
        // count in the gemm class)
        const int grc = gemm<double>(0, 0, n, nrhs, n, -1.0, a, lda, x, ldx, 1.0, p.r, nrhs, s);
        if (grc != B200LA_SUCCESS)
            return grc;
        prof_begin(KC_RESIDUAL, s);
        k_colmax<<<grid_for((int64_t)n * nrhs), 256, 0, s>>>(p.r, nrhs, n, nrhs, p.norms + 4);
        k_colmax<<<grid_for((int64_t)n * nrhs), 256, 0, s>>>(x, ldx, n, nrhs, p.norms + 4 + kMaxNrhsMixed);
        prof_end(KC_RESIDUAL, s);
    }
    B200LA_LAUNCH_CHECK();
    std::vector<unsigned long long> h(2 * kMaxNrhsMixed);
    B200LA_CUDA(cudaMemcpyAsync(h.data(), p.norms + 4, sizeof(unsigned long long) * 2 * kMaxNrhsMixed,
        cudaMemcpyDeviceToHost, s));
    B200LA_CUDA(cudaStreamSynchronize(s));
    double worst = 0.0;
    for (int j = 0; j < nrhs; ++j)
    {
        double rn, xn;
        memcpy(&rn, &h[j], 8);
        memcpy(&xn, &h[kMaxNrhsMixed + j], 8);
        const double den = anorm * xn + bnorm[j];
        const double e   = den > 0 ? rn / den : (rn > 0 ? INFINITY : 0.0);
        if (!(e <= worst))
            worst = e;  // NaN propagates
    }
    *eta = worst;
    return B200LA_SUCCESS;
}

double dot_host(const double* a, const double* b, int n, double* h, cudaStream_t s)
{
    cudaMemsetAsync(h, 0, sizeof(double), s);
    dim3 grid(grid_for(n), 1);
    k_dots<<<grid, 256, 0, s>>>(a, b, n, 1, h);
    double v = 0;
    cudaMemcpyAsync(&v, h, sizeof(double), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    return v;
}

// One restarted-GMRES solve of A d = r (r in p.r), left preconditioned by the
// factors; d accumulated into x.  Returns the iterations used.
template <typename TA>
int gmres_correction(const double* a, int64_t lda, const TA* lu, int n, int restart, double rtol, double* x,
    MixedPlan& p, DeviceStatus* st, cudaStream_t s, int* iters)
{
    const int m = restart;
    double*   V = p.V;
    // z0 = M^-1 r  -> V[0]
    B200LA_CUDA(cudaMemcpyAsync(V, p.r, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    int rc = enqueue_lu_apply<TA>(lu, p.perm, n, 1, V, 1, p, st, s);
    if (rc != B200LA_SUCCESS)
        return rc;
    const double beta = std::sqrt(dot_host(V, V, n, p.h, s));
    if (!(beta > 0) || !std::isfinite(beta))
    {
        *iters = 0;
        return B200LA_SUCCESS;
    }
    k_scale_copy<<<grid_for(n), 256, 0, s>>>(V, 1.0 / beta, V, n);
    std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1, 0.0);
    g[0] = beta;
    int j = 0;
    for (; j < m; ++j)
    {
        double* w = V + (size_t)(j + 1) * n;
        // w = M^-1 A v_j
        k_residual<<<(n + kResRows - 1) / kResRows, 256, 0, s>>>(a, lda, V + (size_t)j * n, nullptr, w, n, p.norms + 2);
        B200LA_LAUNCH_CHECK();
        rc = enqueue_lu_apply<TA>(lu, p.perm, n, 1, w, 1, p, st, s);
        if (rc != B200LA_SUCCESS)
            return rc;
        // w currently holds -M^-1 A v_j (b = 0); flip sign while orthogonalizing
        k_scale_copy<<<grid_for(n), 256, 0, s>>>(w, -1.0, w, n);
        // classical Gram-Schmidt, twice
        std::vector<double> hcol(j + 1, 0.0);
        for (int pass = 0; pass < 2; ++pass)
        {
            B200LA_CUDA(cudaMemsetAsync(p.h, 0, sizeof(double) * (j + 1), s));
            k_dots<<<dim3(grid_for(n) / 4 + 1, j + 1), 256, 0, s>>>(V, w, n, j + 1, p.h);
            k_comb<<<grid_for(n), 256, 0, s>>>(V, p.h, n, j + 1, -1.0, w);
            std::vector<double> hh(j + 1);
            B200LA_CUDA(cudaMemcpyAsync(hh.data(), p.h, sizeof(double) * (j + 1), cudaMemcpyDeviceToHost, s));
            B200LA_CUDA(cudaStreamSynchronize(s));
            for (int i = 0; i <= j; ++i)
                hcol[i] += hh[i];
        }
        const double hn = std::sqrt(dot_host(w, w, n, p.h, s));
        for (int i = 0; i <= j; ++i)
            H[(size_t)i * m + j] = hcol[i];
        H[(size_t)(j + 1) * m + j] = hn;
        if (hn > 0)
            k_scale_copy<<<grid_for(n), 256, 0, s>>>(w, 1.0 / hn, w, n);
        // Givens rotations on column j
        for (int i = 0; i < j; ++i)
        {
            const double t0 = H[(size_t)i * m + j], t1 = H[(size_t)(i + 1) * m + j];
            H[(size_t)i * m + j]       = cs[i] * t0 + sn[i] * t1;
            H[(size_t)(i + 1) * m + j] = -sn[i] * t0 + cs[i] * t1;
        }
        const double a0 = H[(size_t)j * m + j], a1 = H[(size_t)(j + 1) * m + j];
        const double rr = std::hypot(a0, a1);
        cs[j]           = rr > 0 ? a0 / rr : 1.0;
        sn[j]           = rr > 0 ? a1 / rr : 0.0;
        H[(size_t)j * m + j]       = rr;
        H[(size_t)(j + 1) * m + j] = 0.0;
        g[j + 1]        = -sn[j] * g[j];
        g[j]            = cs[j] * g[j];
        if (std::fabs(g[j + 1]) <= rtol * beta || hn == 0)
        {
            ++j;
            break;
        }
    }
    // y = H^-1 g (upper triangular j x j), d = V y, x += d
    std::vector<double> yv(j, 0.0);
    for (int i = j - 1; i >= 0; --i)
    {
        double t = g[i];
        for (int q = i + 1; q < j; ++q)
            t -= H[(size_t)i * m + q] * yv[q];
        yv[i] = H[(size_t)i * m + i] != 0 ? t / H[(size_t)i * m + i] : 0.0;
    }
    B200LA_CUDA(cudaMemcpyAsync(p.h, yv.data(), sizeof(double) * j, cudaMemcpyHostToDevice, s));
    k_comb<<<grid_for(n), 256, 0, s>>>(V, p.h, n, j, 1.0, x);
    B200LA_LAUNCH_CHECK();
    *iters = j;
    return B200LA_SUCCESS;
}


// ---------------------------------------------------------------------------
// factor / refine steps shared by the mixed and the selected solves
// ---------------------------------------------------------------------------
// The FP32 Cholesky factor in LU form for the Cholesky-IR: with L lower
// (l_ij, i >= j) and D = diag(l_ii), L_u = L D^-1 (unit lower) and
// U = D L^T satisfy L_u U = L L^T, so the LU refinement applies it with the
// identity permutation.  One thread per strictly lower (i, j) writes
// u_ji = l_jj l_ij and l_ij / l_jj; the diagonal is only read here.
__global__ void k_chol_lu_pairs(float* __restrict__ a, int n, const DeviceStatus* gate)
{
    if (gated(gate))
        return;
    const int64_t total = (int64_t)n * n;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x)
    {
        const int i = (int)(e / n), j = (int)(e - (e / n) * n);
        if (j < i)
        {
            const float l         = a[e];
            const float d         = a[(int64_t)j * n + j];
            a[(int64_t)j * n + i] = d * l;
            a[e]                  = l / d;
        }
    }
}

// Then u_ii = l_ii^2, and the identity permutation.
__global__ void k_chol_lu_diag(float* __restrict__ a, int n, int32_t* __restrict__ perm, const DeviceStatus* gate)
{
    if (gated(gate))
        return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const float d        = a[(int64_t)i * n + i];
        a[(int64_t)i * n + i] = d * d;
        perm[i]              = i;
    }
}

struct SolveState
{
    double              anorm      = 0.0;
    bool                have_anorm = false;
    std::vector<double> bnorm;
};

// Factor A in `precision` into p.a32 (or p.a64 for FP64), with p.perm and the
// inverted diagonal blocks; *info = LAPACK info.  Adds the device time to
// out.factor_ms.  Reads ||A|| and ||b_j|| the first time.  spd: the FP32
// factorization is the Cholesky of A's lower triangle, stored in LU form
// (info = the first non-positive pivot's row); FP64 stays the plain LU.
int mixed_factor(const double* a, int nn, int nr, int precision, MixedPlan& p, SolveState& ss, int* info,
    b200la_refine_result& out, cudaEvent_t e0, cudaEvent_t e1, cudaStream_t s, bool spd = false)
{
    const int64_t n     = nn;
    const bool    use64 = precision == B200LA_PREC_FP64;
    const int     kind  = precision == B200LA_PREC_BF16   ? TC_BF16
                          : precision == B200LA_PREC_FP16 ? TC_FP16
                          : precision == B200LA_PREC_FP8  ? TC_FP8
                                                          : TC_TF32;
    const bool    split = precision == B200LA_PREC_FP32;
    int           rc    = B200LA_SUCCESS;
    cudaEventRecord(e0, s);
    DeviceStatus* st = use64 ? p.gp64.st : p.gp.st;
    if (!use64)
    {
        k_convert_a<<<(nn * 32 + 255) / 256, 256, 0, s>>>(a, n, p.a32, nn, p.norms);
        B200LA_LAUNCH_CHECK();
        if (spd)
        {
            if ((rc = enqueue_potrf<float>(p.a32, nn, false, st, s)) != B200LA_SUCCESS)
                return rc;
            prof_begin(KC_CHOL_AUX, s);
            k_chol_lu_pairs<<<grid_for(n * n), 256, 0, s>>>(p.a32, nn, st);
            prof_end(KC_CHOL_AUX, s);
            B200LA_LAUNCH_CHECK();
            prof_begin(KC_CHOL_AUX, s);
            k_chol_lu_diag<<<grid_for(n), 256, 0, s>>>(p.a32, nn, p.perm, st);
            prof_end(KC_CHOL_AUX, s);
        }
        // the factorization leaves its row permutation in p.perm
        else if ((rc = enqueue_getrf_mixed(p, nn, kind, split, s)) != B200LA_SUCCESS)
            return rc;
    }
    else
    {
        B200LA_CUDA(cudaMemcpy2DAsync(p.a64, sizeof(double) * n, a, sizeof(double) * n, sizeof(double) * n, n,
            cudaMemcpyDeviceToDevice, s));
        if (!ss.have_anorm)
        {
            k_convert_a<<<(nn * 32 + 255) / 256, 256, 0, s>>>(a, n, p.a32, nn, p.norms);
            B200LA_LAUNCH_CHECK();
        }
        if ((rc = enqueue_getrf<double>(p.a64, nn, p.piv64, p.gp64, s)) != B200LA_SUCCESS)
            return rc;
        k_perm_from_pivots<0><<<1, 256, perm_smem_bytes(nn), s>>>(p.piv64, nn, p.perm, perm_smem_bytes(nn) > 0 ? 1 : 0, st, nullptr);
    }
    B200LA_LAUNCH_CHECK();
    {
        const int nbk = (nn + kTrRows - 1) / kTrRows;
        prof_begin(KC_SOLVE, s);
        if (use64)
            k_invert_diag_blocks128<double><<<dim3(nbk, 2), kTrRows, kTrInvSmem, s>>>(p.a64, n, nn, p.dinv);
        else
            k_invert_diag_blocks128<float><<<dim3(nbk, 2), kTrRows, kTrInvSmem, s>>>(p.a32, n, nn, p.dinv);
        prof_end(KC_SOLVE, s);
        B200LA_LAUNCH_CHECK();
    }
    *info = 0;
    if ((rc = read_status(st, info, s)) < 0)
        return rc;
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float fms = 0;
    cudaEventElapsedTime(&fms, e0, e1);
    out.factor_ms += fms;
    out.info = *info;
    if (!ss.have_anorm)
    {
        unsigned long long hb[1 + kMaxNrhsMixed];
        B200LA_CUDA(cudaMemcpy(hb, p.norms, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        memcpy(&ss.anorm, &hb[0], 8);
        B200LA_CUDA(cudaMemcpy(hb + 1, p.norms + 4 + 2 * kMaxNrhsMixed, sizeof(unsigned long long) * nr,
            cudaMemcpyDeviceToHost));
        ss.bnorm.assign(nr, 0.0);
        for (int j = 0; j < nr; ++j)
            memcpy(&ss.bnorm[j], &hb[1 + j], 8);
        ss.have_anorm = true;
    }
    return B200LA_SUCCESS;
}

// x0 = M^-1 b with the factors of `precision`, then refinement (LU-IR,
// switching to GMRES-IR when it stalls) until eta <= tolerance or
// max_iterations corrections.  *converged on exit.
int mixed_refine(const double* a, int nn, int nr, const double* b, int64_t ldb, double* x, int64_t ldx,
    int precision, const b200la_refine_options* o, int restart, MixedPlan& p, SolveState& ss, bool* converged,
    b200la_refine_result& out, cudaEvent_t e0, cudaEvent_t e1, cudaStream_t s)
{
    const int64_t n     = nn;
    const int64_t nrhs  = nr;
    const bool    use64 = precision == B200LA_PREC_FP64;
    DeviceStatus* st    = use64 ? p.gp64.st : p.gp.st;
    int           rc    = B200LA_SUCCESS;
    *converged          = false;
    cudaEventRecord(e0, s);
    k_copy2d<double><<<grid_for((int64_t)n * nrhs), 256, 0, s>>>(b, ldb, x, ldx, nn, nr, nullptr);
    B200LA_LAUNCH_CHECK();
    rc = use64 ? enqueue_lu_apply<double>(p.a64, p.perm, nn, nr, x, ldx, p, st, s)
               : enqueue_lu_apply<float>(p.a32, p.perm, nn, nr, x, ldx, p, st, s);
    if (rc != B200LA_SUCCESS)
        return rc;
    double eta_prev = INFINITY;
    bool   gmres_on = false;
    for (int it = 0; it < o->max_iterations; ++it)
    {
        double eta = INFINITY;
        if ((rc = residual_eta(a, n, nn, nr, b, ldb, x, ldx, p, ss.anorm, ss.bnorm, &eta, s)) != B200LA_SUCCESS)
            return rc;
        out.backward_error = eta;
        if (eta <= o->tolerance)
        {
            *converged = true;
            break;
        }
        const bool stalled = !std::isfinite(eta) || (it > 0 && eta > 0.5 * eta_prev);
        if (stalled && (!gmres_on && restart > 0))
        {
            gmres_on = true;  // switch to GMRES-IR for the remaining iterations
        }
        else if (stalled && it > 1)
        {
            break;  // give up on this precision
        }
        eta_prev = eta;
        out.iterations++;
        if (gmres_on)
        {
            int gi = 0;
            rc = use64 ? gmres_correction<double>(a, n, p.a64, nn, restart, 1e-6, x, p, st, s, &gi)
                       : gmres_correction<float>(a, n, p.a32, nn, restart, 1e-6, x, p, st, s, &gi);
            if (rc != B200LA_SUCCESS)
                return rc;
            out.gmres_iterations += gi;
        }
        else
        {
            rc = use64 ? enqueue_lu_apply<double>(p.a64, p.perm, nn, nr, p.r, nr, p, st, s)
                       : enqueue_lu_apply<float>(p.a32, p.perm, nn, nr, p.r, nr, p, st, s);
            if (rc != B200LA_SUCCESS)
                return rc;
            k_axpy2d<<<grid_for((int64_t)n * nrhs), 256, 0, s>>>(x, ldx, p.r, nr, nn, nr);
            B200LA_LAUNCH_CHECK();
        }
    }
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float rms = 0;
    cudaEventElapsedTime(&rms, e0, e1);
    out.refine_ms += rms;
    return B200LA_SUCCESS;
}

// Next precision up after a failed attempt: FP8 -> BF16; BF16, FP16, TF32 ->
// FP32 (three-term TF32); FP32 -> FP64.
int next_precision(int precision)
{
    return precision == B200LA_PREC_FP8    ? B200LA_PREC_BF16
           : precision == B200LA_PREC_FP32 ? B200LA_PREC_FP64
                                           : B200LA_PREC_FP32;
}

// Factor-refine-escalate loop from `precision`.  With `prefactored` the FP32
// factors (three-term TF32) are already in p (info `pre_info`) and the first
// attempt reuses them.  spd: FP32 is the Cholesky (see mixed_factor).
int mixed_loop(const double* a, int nn, int nr, const double* b, int64_t ldb, double* x, int64_t ldx,
    int precision, bool prefactored, int pre_info, const b200la_refine_options* o, int restart, MixedPlan& p,
    SolveState& ss, b200la_refine_result& out, cudaEvent_t e0, cudaEvent_t e1, cudaStream_t s, bool spd = false)
{
    int escalations = 0;
    for (;;)
    {
        int info = 0, rc;
        if (prefactored)
        {
            info     = pre_info;
            out.info = info;
            prefactored = false;
        }
        else if ((rc = mixed_factor(a, nn, nr, precision, p, ss, &info, out, e0, e1, s, spd)) != B200LA_SUCCESS &&
                 rc != B200LA_SINGULAR)
        {
            return rc;
        }
        bool converged = false;
        if (info == 0)
        {
            if ((rc = mixed_refine(a, nn, nr, b, ldb, x, ldx, precision, o, restart, p, ss, &converged, out, e0,
                     e1, s)) != B200LA_SUCCESS)
                return rc;
        }
        out.precision_used = precision;
        out.converged      = converged ? 1 : 0;
        if (converged || !o->escalate || precision == B200LA_PREC_FP64)
            break;
        precision = next_precision(precision);
        ++escalations;
    }
    out.escalations += escalations;
    return B200LA_SUCCESS;
}

// ---------------------------------------------------------------------------
// selector features
// ---------------------------------------------------------------------------
// out[] words: see k_row_features / k_col_features / k_lu_features
// (selector.cu); the FP32 factors are in p.a32 / p.perm.

// z = A^-T v with the FP32 factors (P A = L U => A^T = U^T L^T P):
// U^T w = v, L^T u = w, z = P^T u.  v is overwritten; z must not alias v.
__global__ void k_scatter_perm(const double* __restrict__ u, const int32_t* __restrict__ perm, int n,
    double* __restrict__ z)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    {
        z[perm[i]] = u[i];
    }
}

int apply_inverse_transpose(MixedPlan& p, int n, double* v, double* z, cudaStream_t s)
{
    int rc = enqueue_trsm_inplace<float, double>(true, true, false, n, 1, p.a32, n, v, 1, nullptr, s);
    if (rc != B200LA_SUCCESS)
        return rc;
    rc = enqueue_trsm_inplace<float, double>(false, true, true, n, 1, p.a32, n, v, 1, nullptr, s);
    if (rc != B200LA_SUCCESS)
        return rc;
    k_scatter_perm<<<grid_for(n), 256, 0, s>>>(v, p.perm, n, z);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

// Hager's estimate of ||A^-1||_1 (Hager, SIAM J. Sci. Stat. Comput. 5, 1984)
// with Higham's extra test vector and stopping rules (Higham, ACM TOMS 14,
// 1988), using the FP32 LU factors in p applied in FP64.  Vectors are reduced
// on the host (n doubles per step, at most five steps).
int hager_inverse_norm1(MixedPlan& p, int n, double* est, cudaStream_t s)
{
    std::vector<double> hx(n, 1.0 / n), hy(n), hz(n);
    double*             dv = p.r;   // n doubles
    double*             dz = p.V != nullptr ? p.V : p.y;
    double              e  = 0.0;
    int                 rc;
    int                 jlast = -1;
    for (int iter = 0; iter < 5; ++iter)
    {
        B200LA_CUDA(cudaMemcpyAsync(dv, hx.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
        if ((rc = enqueue_lu_apply<float>(p.a32, p.perm, n, 1, dv, 1, p, p.gp.st, s)) != B200LA_SUCCESS)
            return rc;
        B200LA_CUDA(cudaMemcpyAsync(hy.data(), dv, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        B200LA_CUDA(cudaStreamSynchronize(s));
        double e_new = 0.0;
        for (int i = 0; i < n; ++i)
            e_new += std::fabs(hy[i]);
        if (!std::isfinite(e_new))
        {
            *est = INFINITY;
            return B200LA_SUCCESS;
        }
        if (iter > 0 && e_new <= e)
            break;
        e = e_new;
        for (int i = 0; i < n; ++i)
            hy[i] = hy[i] >= 0 ? 1.0 : -1.0;
        B200LA_CUDA(cudaMemcpyAsync(dv, hy.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
        if ((rc = apply_inverse_transpose(p, n, dv, dz, s)) != B200LA_SUCCESS)
            return rc;
        B200LA_CUDA(cudaMemcpyAsync(hz.data(), dz, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
        B200LA_CUDA(cudaStreamSynchronize(s));
        int    j  = 0;
        double zx = 0.0;
        for (int i = 0; i < n; ++i)
        {
            if (std::fabs(hz[i]) > std::fabs(hz[j]))
                j = i;
            zx += hz[i] * hx[i];
        }
        if (iter > 0 && (std::fabs(hz[j]) <= zx || j == jlast))
            break;
        jlast = j;
        std::fill(hx.begin(), hx.end(), 0.0);
        hx[j] = 1.0;
    }
    // Higham's alternating test vector
    for (int i = 0; i < n; ++i)
        hx[i] = (i % 2 == 0 ? 1.0 : -1.0) * (1.0 + (n > 1 ? (double)i / (n - 1) : 0.0));
    B200LA_CUDA(cudaMemcpyAsync(dv, hx.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s));
    if ((rc = enqueue_lu_apply<float>(p.a32, p.perm, n, 1, dv, 1, p, p.gp.st, s)) != B200LA_SUCCESS)
        return rc;
    B200LA_CUDA(cudaMemcpyAsync(hy.data(), dv, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    B200LA_CUDA(cudaStreamSynchronize(s));
    double alt = 0.0;
    for (int i = 0; i < n; ++i)
        alt += std::fabs(hy[i]);
    alt = 2.0 * alt / (3.0 * n);
    *est = alt > e ? alt : e;
    return B200LA_SUCCESS;
}

}  // namespace

// The selector's statistics kernels and network (selector.cu).
int enqueue_matrix_stats(const double* a, int n, unsigned long long* out, cudaStream_t s);
int enqueue_mlp_forward(const float* params, const float* x, int batch, float* probs, cudaStream_t s);
constexpr int kSelFeatures = 12, kSelClasses = 4, kSelParams = 5252;

namespace
{
inline double word_to_double(unsigned long long w)
{
    double d;
    memcpy(&d, &w, 8);
    return d;
}
inline float safe_log10(double v) { return (float)std::log10(v > 1e-300 ? v : 1e-300); }

// The 12 selector features of A (host floats) from its O(n^2) statistics
// (enqueue_matrix_stats into `stats`, 16 device words).  Synchronizes `s`.
int selector_features(const double* a, int nn, unsigned long long* stats, float* f, cudaStream_t s)
{
    int rc = enqueue_matrix_stats(a, nn, stats, s);
    if (rc != B200LA_SUCCESS)
        return rc;
    unsigned long long h[16];
    B200LA_CUDA(cudaMemcpyAsync(h, stats, sizeof(h), cudaMemcpyDeviceToHost, s));
    B200LA_CUDA(cudaStreamSynchronize(s));
    const double n         = nn;
    const double norm_inf  = word_to_double(h[0]);
    const double amax      = word_to_double(h[1]);
    const double fro       = std::sqrt(word_to_double(h[2]));
    const double dd_inv    = word_to_double(h[3]);  // max over rows of 1 / (1 + r_i)
    const double dd_rows   = (double)h[4];
    const double norm_1    = word_to_double(h[5]);
    const double row_min   = word_to_double(h[6]);
    const double dmin      = word_to_double(h[7]);
    const double dmax      = word_to_double(h[8]);
    const double abs_sum   = word_to_double(h[9]);
    const double col_min   = word_to_double(h[10]);
    const double diag_sum  = word_to_double(h[11]);
    const double min_ratio = dd_inv > 0 ? 1.0 / dd_inv - 1.0 : 1e30;
    f[0]  = (float)(std::log2(n) / 12.0);
    f[1]  = safe_log10(norm_inf / amax);
    f[2]  = safe_log10(norm_1 / amax);
    f[3]  = safe_log10(fro / (amax * n));
    f[4]  = safe_log10(abs_sum / (amax * n * n));
    f[5]  = safe_log10(min_ratio) / 4.0f;
    f[6]  = (float)(dd_rows / n);
    f[7]  = safe_log10(dmin / amax) / 4.0f;
    f[8]  = safe_log10(dmax / amax);
    f[9]  = safe_log10(row_min / norm_inf) / 4.0f;
    f[10] = safe_log10(col_min / norm_1) / 4.0f;
    f[11] = safe_log10(diag_sum / (amax * n));
    return B200LA_SUCCESS;
}
}  // namespace
}  // namespace b200la

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
using namespace b200la;

extern "C" {

B200LA_API void b200la_refine_default_options(b200la_refine_options* o)
{
    if (o == nullptr)
        return;
    o->precision      = B200LA_PREC_FP32;
    o->max_iterations = 50;
    o->tolerance      = 1e-14;
    o->gmres_restart  = 30;
    o->escalate       = 1;
}

B200LA_API size_t b200la_dsolve_mixed_workspace_size(int64_t n, int64_t nrhs, const b200la_refine_options* o)
{
    if (n <= 0 || nrhs <= 0 || nrhs > kMaxNrhsMixed)
        return 0;
    b200la_refine_options d;
    b200la_refine_default_options(&d);
    if (o == nullptr)
        o = &d;
    const int restart = nrhs == 1 ? (o->gmres_restart > kGmresMaxRestart ? kGmresMaxRestart : (o->gmres_restart < 0 ? 0 : o->gmres_restart)) : 0;
    Arena a;
    plan_mixed(a, n, nrhs, restart, o->escalate != 0 || o->precision == B200LA_PREC_FP64);
    return a.size();
}

static int check_mixed_call(const double* a, int64_t n, int64_t nrhs, const double* b, int64_t ldb,
    const double* x, int64_t ldx, const b200la_refine_options* o, void* ws, size_t ws_bytes)
{
    if (a == nullptr || b == nullptr || x == nullptr)
        return set_error(B200LA_INVALID_ARGUMENT, "a, b and x must not be null");
    if (n <= 0 || nrhs <= 0 || nrhs > kMaxNrhsMixed || ldb < nrhs || ldx < nrhs || n > 65536)
        return set_error(B200LA_INVALID_ARGUMENT, "invalid sizes (n %lld, nrhs %lld; nrhs <= %d)",
            (long long)n, (long long)nrhs, kMaxNrhsMixed);
    if (o->precision < B200LA_PREC_FP64 || o->precision > B200LA_PREC_FP8 || o->max_iterations < 1 ||
        !(o->tolerance > 0))
        return set_error(B200LA_INVALID_ARGUMENT, "invalid refinement options");
    const size_t need = b200la_dsolve_mixed_workspace_size(n, nrhs, o);
    if (ws == nullptr || ws_bytes < need)
        return set_error(B200LA_WORKSPACE_TOO_SMALL, "workspace too small (%zu < %zu)", ws_bytes, need);
    int rc = prepare<float>();
    if (rc != B200LA_SUCCESS)
        return rc;
    if ((rc = prepare<double>()) != B200LA_SUCCESS)
        return rc;
    return set_mixed_attributes();
}

static int restart_of(const b200la_refine_options* o, int64_t nrhs)
{
    return nrhs == 1 ? (o->gmres_restart > kGmresMaxRestart ? kGmresMaxRestart : (o->gmres_restart < 0 ? 0 : o->gmres_restart)) : 0;
}

struct MixedEvents
{
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    MixedEvents()
    {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
    }
    ~MixedEvents()
    {
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
};

static int finish_result(b200la_refine_result& out, b200la_refine_result* res)
{
    if (res)
        *res = out;
    if (out.info != 0)
        return B200LA_SINGULAR;
    return out.converged ? B200LA_SUCCESS : B200LA_NOT_CONVERGED;
}

static int solve_mixed(const double* a, int64_t n, int64_t nrhs, const double* b, int64_t ldb, double* x,
    int64_t ldx, const b200la_refine_options* o, b200la_refine_result* res, void* ws, size_t ws_bytes,
    void* stream, bool spd)
{
    int rc = check_mixed_call(a, n, nrhs, b, ldb, x, ldx, o, ws, ws_bytes);
    if (rc != B200LA_SUCCESS)
        return rc;
    cudaStream_t s        = static_cast<cudaStream_t>(stream);
    const int    restart  = restart_of(o, nrhs);
    const bool   fallback = o->escalate != 0 || o->precision == B200LA_PREC_FP64;
    Arena        ar(ws, ws_bytes);
    MixedPlan    p  = plan_mixed(ar, n, nrhs, restart, fallback);
    const int    nn = (int)n, nr = (int)nrhs;

    b200la_refine_result out{};
    out.backward_error = INFINITY;
    MixedEvents ev;
    // ||b_j||_inf (read with ||A|| after the first factorization)
    B200LA_CUDA(cudaMemsetAsync(p.norms, 0, sizeof(unsigned long long) * (4 + 3 * kMaxNrhsMixed), s));
    k_colmax<<<grid_for((int64_t)n * nrhs), 256, 0, s>>>(b, ldb, nn, nr, p.norms + 4 + 2 * kMaxNrhsMixed);
    B200LA_LAUNCH_CHECK();
    SolveState ss;
    if ((rc = mixed_loop(a, nn, nr, b, ldb, x, ldx, o->precision, false, 0, o, restart, p, ss, out, ev.e0, ev.e1,
             s, spd)) != B200LA_SUCCESS)
        return rc;
    return finish_result(out, res);
}

B200LA_API int b200la_dsolve_mixed(const double* a, int64_t n, int64_t nrhs, const double* b, int64_t ldb,
    double* x, int64_t ldx, const b200la_refine_options* opts, b200la_refine_result* res, void* ws,
    size_t ws_bytes, void* stream)
{
    b200la_refine_options d;
    b200la_refine_default_options(&d);
    return solve_mixed(a, n, nrhs, b, ldb, x, ldx, opts ? opts : &d, res, ws, ws_bytes, stream, false);
}

B200LA_API int b200la_dsolve_mixed_spd(const double* a, int64_t n, int64_t nrhs, const double* b, int64_t ldb,
    double* x, int64_t ldx, const b200la_refine_options* opts, b200la_refine_result* res, void* ws,
    size_t ws_bytes, void* stream)
{
    b200la_refine_options d;
    b200la_refine_default_options(&d);
    const b200la_refine_options* o = opts ? opts : &d;
    if (o->precision != B200LA_PREC_FP32 && o->precision != B200LA_PREC_FP64)
        return set_error(B200LA_INVALID_ARGUMENT, "Cholesky-IR: the factorization precision is FP32 or FP64");
    return solve_mixed(a, n, nrhs, b, ldb, x, ldx, o, res, ws, ws_bytes, stream, true);
}

B200LA_API int b200la_selector_features(const double* a, int64_t n, float* features, void* ws, size_t ws_bytes,
    void* stream)
{
    if (a == nullptr || features == nullptr || n <= 0 || n > 65536)
        return set_error(B200LA_INVALID_ARGUMENT, "selector_features: invalid arguments");
    if (ws == nullptr || ws_bytes < 16 * sizeof(unsigned long long) || (reinterpret_cast<uintptr_t>(ws) & 7) != 0)
        return set_error(B200LA_WORKSPACE_TOO_SMALL, "selector_features: needs 128 bytes of 8-byte aligned workspace");
    int rc = require_sm100();
    if (rc != B200LA_SUCCESS)
        return rc;
    return selector_features(a, (int)n, static_cast<unsigned long long*>(ws), features,
        static_cast<cudaStream_t>(stream));
}

B200LA_API int b200la_dcondition_estimate(const double* a, int64_t n, double* kappa1, int* info, void* ws,
    size_t ws_bytes, void* stream)
{
    b200la_refine_options o;
    b200la_refine_default_options(&o);
    if (kappa1 == nullptr)
        return set_error(B200LA_INVALID_ARGUMENT, "condition_estimate: kappa1 must not be null");
    int rc = check_mixed_call(a, n, 1, a, 1, a, 1, &o, ws, ws_bytes);
    if (rc != B200LA_SUCCESS)
        return rc;
    cudaStream_t s  = static_cast<cudaStream_t>(stream);
    const int    nn = (int)n;
    Arena        ar(ws, ws_bytes);
    MixedPlan    p = plan_mixed(ar, n, 1, restart_of(&o, 1), true);
    B200LA_CUDA(cudaMemsetAsync(p.norms, 0, sizeof(unsigned long long) * (4 + 3 * kMaxNrhsMixed), s));
    b200la_refine_result out{};
    MixedEvents          ev;
    SolveState           ss;
    int                  inf = 0;
    // ||A||_1 from the statistics, then one FP32 LU (three-term TF32 updates)
    unsigned long long* stats = p.norms + 4 + 3 * kMaxNrhsMixed;
    if ((rc = enqueue_matrix_stats(a, nn, stats, s)) != B200LA_SUCCESS)
        return rc;
    unsigned long long h[16];
    B200LA_CUDA(cudaMemcpyAsync(h, stats, sizeof(h), cudaMemcpyDeviceToHost, s));
    if ((rc = mixed_factor(a, nn, 1, B200LA_PREC_FP32, p, ss, &inf, out, ev.e0, ev.e1, s)) != B200LA_SUCCESS &&
        rc != B200LA_SINGULAR)
        return rc;
    if (info)
        *info = inf;
    if (inf != 0)
    {
        *kappa1 = INFINITY;
        return B200LA_SINGULAR;
    }
    double ainv1 = INFINITY;
    if ((rc = hager_inverse_norm1(p, nn, &ainv1, s)) != B200LA_SUCCESS)
        return rc;
    *kappa1 = word_to_double(h[5]) * ainv1;
    return B200LA_SUCCESS;
}

B200LA_API int b200la_dsolve_selected(const double* a, int64_t n, const double* b, double* x,
    const float* params, const b200la_refine_options* opts, b200la_refine_result* res, int* predicted,
    float* features, void* ws, size_t ws_bytes, void* stream)
{
    b200la_refine_options d;
    b200la_refine_default_options(&d);
    b200la_refine_options o = opts ? *opts : d;
    o.precision             = B200LA_PREC_FP32;
    o.escalate              = 1;
    if (params == nullptr)
        return set_error(B200LA_INVALID_ARGUMENT, "dsolve_selected: params must not be null");
    int rc = check_mixed_call(a, n, 1, b, 1, x, 1, &o, ws, ws_bytes);
    if (rc != B200LA_SUCCESS)
        return rc;
    cudaStream_t s       = static_cast<cudaStream_t>(stream);
    const int    restart = restart_of(&o, 1);
    Arena        ar(ws, ws_bytes);
    MixedPlan    p  = plan_mixed(ar, n, 1, restart, true);
    const int    nn = (int)n;

    b200la_refine_result out{};
    out.backward_error = INFINITY;
    MixedEvents ev;
    B200LA_CUDA(cudaMemsetAsync(p.norms, 0, sizeof(unsigned long long) * (4 + 3 * kMaxNrhsMixed), s));
    k_colmax<<<grid_for(n), 256, 0, s>>>(b, 1, nn, 1, p.norms + 4 + 2 * kMaxNrhsMixed);
    B200LA_LAUNCH_CHECK();
    float f[kSelFeatures];
    if ((rc = selector_features(a, nn, p.norms + 4 + 3 * kMaxNrhsMixed, f, s)) != B200LA_SUCCESS)
        return rc;
    if (features)
        memcpy(features, f, sizeof(f));
    // standardize with the network's stored mean / inverse std, then infer
    float norm[2 * kSelFeatures];
    B200LA_CUDA(cudaMemcpyAsync(norm, params + kSelParams, sizeof(norm), cudaMemcpyDeviceToHost, s));
    B200LA_CUDA(cudaStreamSynchronize(s));
    float xin[kSelFeatures];
    for (int i = 0; i < kSelFeatures; ++i)
        xin[i] = (f[i] - norm[i]) * norm[kSelFeatures + i];
    B200LA_CUDA(cudaMemcpyAsync(p.sel, xin, sizeof(xin), cudaMemcpyHostToDevice, s));
    if ((rc = enqueue_mlp_forward(params, p.sel, 1, p.sel + kSelFeatures, s)) != B200LA_SUCCESS)
        return rc;
    float probs[kSelClasses];
    B200LA_CUDA(cudaMemcpyAsync(probs, p.sel + kSelFeatures, sizeof(probs), cudaMemcpyDeviceToHost, s));
    B200LA_CUDA(cudaStreamSynchronize(s));
    int cls = 0;
    for (int c = 1; c < kSelClasses; ++c)
        if (probs[c] > probs[cls])
            cls = c;
    static const int kClassPrec[kSelClasses] = {B200LA_PREC_FP8, B200LA_PREC_BF16, B200LA_PREC_FP32,
        B200LA_PREC_FP64};
    if (predicted)
        *predicted = kClassPrec[cls];
    // the predicted precision first; refinement failure escalates
    SolveState ss;
    if ((rc = mixed_loop(a, nn, 1, b, 1, x, 1, kClassPrec[cls], false, 0, &o, restart, p, ss, out, ev.e0, ev.e1,
             s)) != B200LA_SUCCESS)
        return rc;
    return finish_result(out, res);
}
}
