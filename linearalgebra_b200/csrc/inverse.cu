// inversion and determinant on the B200.
//
// Replaces inversion<T, Backend>::apply / ::workspace_size
// (include/matrix_operation/inversion.h:15-53) and determinant<T, Backend>::
// apply / ::workspace_size (include/matrix_operation/determinant.h) in all
// four modes.  The LU modes reuse the LU factors: LU mode factors m in place
// with the bit-exact blocked LU of lu_driver.cuh (the reference's NATIVE
// lu_decomposition), LU_UPFRONT takes m and pivot as the caller's factors.
//
// Inversion, A^-1 = U^-1 L^-1 P:
//   1. W = I (the n x n workspace);
//   2. W = L^-1 W, forward substitution in row blocks of kNB (512: deeper
//      GEMM updates run closer to the tensor pipe's rate): the block row
//      is solved against L's unit diagonal block (block_solve),
//      then every row below it is updated by one GEMM, C -= A B with
//      A = L[below, block], B = W[block, :], restricted to the columns left
//      of the block's end (L^-1 is lower triangular, the rest stays zero);
//   3. W = U^-1 W, back substitution in the same blocks from the bottom: the
//      block row is solved against U's diagonal block, then every row above
//      it is updated by one GEMM over all n columns;
//   4. m[:, c] = W[:, i0(c)] with perm[i0(c)] = c: the reference swaps the
//      identity's rows before the substitutions (inversion_native.cpp:
//      243-261); the substitutions act on each column independently, so the
//      same swaps become a gather of W's columns at the end.
// Work: n^3/3 + n^3 flops in the GEMM updates, the same count as LAPACK's
// getri (the reference's row-axpy loops do 2 n^3 on the zero-padded identity).
// The reference's loops accumulate every inverse entry in one sequential
// order whose backward pass is a dependent chain of about n^2/2 fused
// multiply-adds per column; no blocked order reproduces it, so the inverse
// agrees with the reference to rounding (a normwise bound), not bit for bit.
//
// Inversion, Cholesky modes, A^-1 = U^-1 L^-1 with U = L^T (A = L L^T):
//   1. CHOLESKY factors m with the bit-exact blocked Cholesky in its upper
//      form (U in the upper triangle, the lower cleared); CHOLESKY_UPFRONT
//      moves the caller's lower factor into the upper triangle (its upper
//      triangle is not read, as passes A and B of inversion_native.cpp:
//      341-375 read only the lower one);
//   2. W = I, then W = U^-1 W by the back substitution of the LU modes;
//   3. W = W^T = L^-1, in place;
//   4. W = U^-1 W, the same back substitution: W = A^-1;
//   5. m = W's upper triangle, mirrored into the lower one, so the inverse
//      is exactly symmetric as the reference's is (inversion_native.cpp:
//      393-409).
// A non-positive pivot stops at step 1 with m holding the partial lower
// factor (the upper form transposes only a complete factor), as the
// reference's lower factorization leaves it (:440-448); the status block
// gates steps 2-5.  Work: 2 n^3 flops, to rounding like the LU modes.
//
// Determinant: the product of U's diagonal in index order, one multiply at a
// time in the input type (determinant.cpp:18-27, so bit-identical to the
// reference for the same factors), the pivot parity (the number of i with
// pivot[i] != i+1) and, beyond the reference, log|det| for orders whose
// product over- or underflows.  LU mode returns 0 when the factorization met
// an exact zero pivot (determinant.cpp:66-75).  The Cholesky modes
// (determinant.cpp:28-37,80-90) take the product of the lower Cholesky
// factor's diagonal the same way (CHOLESKY factors m first with the
// bit-exact blocked Cholesky and returns 0 if m is not positive definite;
// CHOLESKY_UPFRONT reads the given factor); that product is sqrt(det A),
// so log|det| is twice the sum of log l_ii.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstdint>
#include <mutex>

#include "lu_driver.cuh"

namespace b200la
{
namespace inv
{

constexpr int kNB      = 512;  // rows per substitution block (GEMM depth)
constexpr int kTile    = 128;  // GEMM tile, rows and columns
constexpr int kThreads = 256;  // 8 warps: 2 (rows) x 4 (columns), warp tile 64 x 32
constexpr int kStages  = 3;    // cp.async pipeline depth

// Per-type GEMM geometry.  KC: depth per stage, one 128-byte segment of an A
// row.  LDA: the A tile's padded row (+16 bytes), so the eight rows a warp
// reads at one depth index (rows tr + 8i, tr < 8) start 16 bytes apart in
// the bank space and never conflict.
template <typename T> struct Geo
{
    static constexpr int    CE      = 16 / (int)sizeof(T);
    static constexpr int    KC      = 128 / (int)sizeof(T);
    static constexpr int    LDA     = KC + CE;
    static constexpr int    A_ELEMS = kTile * LDA;
    static constexpr int    B_ELEMS = KC * kTile;
    static constexpr int    STAGE   = A_ELEMS + B_ELEMS;
    static constexpr size_t SMEM    = sizeof(T) * (size_t)kStages * STAGE;
};

// One 16-byte piece global -> shared, `valid` (<= 0 .. CE) leading elements
// copied and the rest zero-filled.  Whole pieces go as one 16-byte cp.async
// when the caller's rows are 16-byte aligned; partial ones element by element.
template <typename T>
__device__ __forceinline__ void load_piece(T* s, const T* g, const T* safe, int valid, bool vec16)
{
    constexpr int CE = Geo<T>::CE;
    if (vec16 && (valid >= CE || valid <= 0))
    {
        cp_async16(s, valid > 0 ? g : safe, valid > 0);
        return;
    }
#pragma unroll
    for (int e = 0; e < CE; ++e)
    {
        const bool v = e < valid;
        if (sizeof(T) == 8)
            cp_async8(s + e, v ? g + e : safe, v);
        else
            cp_async4(s + e, v ? g + e : safe, v);
    }
}

// Stage the A tile (kTile x KC from depth k0; smem row stride LDA) and the
// B tile (KC x kTile; smem row stride LDB).
template <typename T, int KC, int LDA, int LDB>
__device__ __forceinline__ void load_stage(T* sa, T* sb, const T* A, int64_t lda, const T* B,
    int64_t ldb, int M, int N, int K, int m0, int n0, int k0, bool vec16)
{
    constexpr int CE  = Geo<T>::CE;
    constexpr int APR = KC / CE;     // pieces per A row
    constexpr int BPR = kTile / CE;  // pieces per B row
    for (int e = threadIdx.x; e < kTile * APR; e += kThreads)
    {
        const int r = e / APR, q = e - (e / APR) * APR;
        const int row = m0 + r, col = k0 + q * CE;
        const int valid = row < M ? min(CE, K - col) : 0;
        load_piece(sa + r * LDA + q * CE, valid > 0 ? A + (int64_t)row * lda + col : A, A, valid, vec16);
    }
    for (int e = threadIdx.x; e < KC * BPR; e += kThreads)
    {
        const int p = e / BPR, q = e - (e / BPR) * BPR;
        const int row = k0 + p, col = n0 + q * CE;
        const int valid = row < K ? min(CE, N - col) : 0;
        load_piece(sb + p * LDB + q * CE, valid > 0 ? B + (int64_t)row * ldb + col : B, B, valid, vec16);
    }
}

// C[M x N] -= A[M x K] B[K x N], row-major with row strides lda, ldb, ldc.
// CTA tile kTile x kTile, K streamed in KC-deep stages through a kStages
// cp.async ring.  Thread (warp w, tr = lane/4, tc = lane%4) owns rows
// (w/4)*64 + tr + 8i and columns (w%4)*32 + 2tc + 8j + e, i, j < 8, 4, e < 2:
// 64 accumulators, fed per depth index by 8 scalar A reads (broadcast to the
// warp's four tc lanes) and 4 paired B reads (broadcast to the eight tr
// lanes).  The product is accumulated from zero and subtracted once.
template <typename T>
__global__ void __launch_bounds__(kThreads, 1) k_inv_gemm(int M, int N, int K, const T* __restrict__ A,
    int64_t lda, const T* __restrict__ B, int64_t ldb, T* __restrict__ C, int64_t ldc, int vec16,
    const DeviceStatus* gate)
{
    extern __shared__ __align__(16) unsigned char inv_smem[];
    if (gated(gate))
    {
        return;
    }
    using G           = Geo<T>;
    T*        smem    = reinterpret_cast<T*>(inv_smem);
    const int m0      = blockIdx.y * kTile;
    const int n0      = blockIdx.x * kTile;
    const int warp    = threadIdx.x >> 5;
    const int lane    = threadIdx.x & 31;
    const int tr      = lane >> 2;
    const int tc      = lane & 3;
    const int wm      = (warp >> 2) * 64;
    const int wn      = (warp & 3) * 32;
    const int nchunks = (K + G::KC - 1) / G::KC;
    const bool v16    = vec16 != 0;

    T acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
    {
#pragma unroll
        for (int j = 0; j < 8; ++j)
        {
            acc[i][j] = T(0);
        }
    }

#pragma unroll
    for (int s = 0; s < kStages - 1; ++s)
    {
        if (s < nchunks)
        {
            T* sa = smem + s * G::STAGE;
            load_stage<T, G::KC, G::LDA, kTile>(sa, sa + G::A_ELEMS, A, lda, B, ldb, M, N, K, m0, n0, s * G::KC, v16);
        }
        cp_async_commit();
    }
    for (int c = 0; c < nchunks; ++c)
    {
        cp_async_wait<kStages - 2>();
        __syncthreads();  // stage c landed for every thread; stage c-1 is free
        const int pf = c + kStages - 1;
        if (pf < nchunks)
        {
            T* sa = smem + (pf % kStages) * G::STAGE;
            load_stage<T, G::KC, G::LDA, kTile>(sa, sa + G::A_ELEMS, A, lda, B, ldb, M, N, K, m0, n0, pf * G::KC, v16);
        }
        cp_async_commit();
        const T* sa   = smem + (c % kStages) * G::STAGE;
        const T* arow = sa + (wm + tr) * G::LDA;
        const T* bcol = sa + G::A_ELEMS + wn + 2 * tc;
#pragma unroll 8
        for (int kk = 0; kk < G::KC; ++kk)
        {
            T a[8], b[8];
#pragma unroll
            for (int i = 0; i < 8; ++i)
            {
                a[i] = arow[8 * i * G::LDA + kk];
            }
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                const auto v = *reinterpret_cast<const typename Vec2<T>::type*>(bcol + kk * kTile + 8 * j);
                b[2 * j]     = v.x;
                b[2 * j + 1] = v.y;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i)
            {
#pragma unroll
                for (int j = 0; j < 8; ++j)
                {
                    acc[i][j] = fma(a[i], b[j], acc[i][j]);
                }
            }
        }
    }
    cp_async_wait<0>();

#pragma unroll
    for (int i = 0; i < 8; ++i)
    {
        const int row = m0 + wm + tr + 8 * i;
        if (row >= M)
        {
            continue;
        }
        T* crow = C + (int64_t)row * ldc;
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const int col = n0 + wn + 2 * tc + 8 * j;
            if (v16 && col + 1 < N)
            {
                auto* p = reinterpret_cast<typename Vec2<T>::type*>(crow + col);
                auto  v = *p;
                v.x -= acc[i][2 * j];
                v.y -= acc[i][2 * j + 1];
                *p = v;
            }
            else
            {
                if (col < N)
                {
                    crow[col] -= acc[i][2 * j];
                }
                if (col + 1 < N)
                {
                    crow[col + 1] -= acc[i][2 * j + 1];
                }
            }
        }
    }
}

// Solve a sub-block of at most kTrsmBlock rows, X[r0:r0+sw, 0:ncols] =
// T[r0:r0+sw, r0:r0+sw]^-1 X (T unit lower when !upper, else upper), for a
// block row of the inverse.  Each column is spread over 8 lanes of a warp
// (lane = 4 r + c: column c of the warp's 4, rows r + 8k, k < 8); at step p
// the owner of row p finishes it (divides by the diagonal when upper) and
// broadcasts it with a shuffle, and every lane updates its rows still to
// be solved.  T's sub-block is staged in shared memory.  32 columns per CTA.
constexpr int kDiagThreads = 256;
constexpr int kDiagCols    = kDiagThreads / 8;

template <typename T, bool upper>
__global__ void __launch_bounds__(kDiagThreads) k_inv_diag(const T* __restrict__ a, int64_t lda, int r0,
    int sw, T* __restrict__ x, int64_t ldx, int ncols, const DeviceStatus* gate)
{
    __shared__ T tri[kTrsmBlock][kTrsmBlock + 1];
    if (gated(gate))
    {
        return;
    }
    for (int e = threadIdx.x; e < kTrsmBlock * kTrsmBlock; e += kDiagThreads)
    {
        const int i = e / kTrsmBlock, j = e - (e / kTrsmBlock) * kTrsmBlock;
        const bool in = i < sw && j < sw && (upper ? j >= i : j < i);
        tri[i][j]     = in ? a[(int64_t)(r0 + i) * lda + r0 + j] : T(0);
    }
    __syncthreads();
    const int  warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int  r = lane >> 2, c = lane & 3;
    const int  col  = blockIdx.x * kDiagCols + warp * 4 + c;
    const bool live = col < ncols;
    T          v[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
    {
        const int i = r + 8 * k;
        v[k]        = live && i < sw ? x[(int64_t)(r0 + i) * ldx + col] : T(0);
    }
#pragma unroll
    for (int q = 0; q < kTrsmBlock; ++q)
    {
        const int p = upper ? kTrsmBlock - 1 - q : q;
        if (p < sw)
        {
            T vp = v[p >> 3];
            if (upper)
            {
                vp = vp / tri[p][p];
                if (r == (p & 7))
                {
                    v[p >> 3] = vp;
                }
            }
            vp = __shfl_sync(0xffffffffu, vp, (p & 7) * 4 + c);
#pragma unroll
            for (int k = 0; k < 8; ++k)
            {
                const int i = r + 8 * k;
                if (upper ? i < p : (i > p && i < sw))
                {
                    v[k] = fma(-tri[i][p], vp, v[k]);
                }
            }
        }
    }
    if (live)
    {
#pragma unroll
        for (int k = 0; k < 8; ++k)
        {
            const int i = r + 8 * k;
            if (i < sw)
            {
                x[(int64_t)(r0 + i) * ldx + col] = v[k];
            }
        }
    }
}

// W = I (n x n, row-major); one CTA per row at a time.
template <typename T> __global__ void k_inv_identity(T* __restrict__ w, int n, const DeviceStatus* gate)
{
    if (gated(gate))
    {
        return;
    }
    for (int r = blockIdx.x; r < n; r += gridDim.x)
    {
        T* row = w + (int64_t)r * n;
        for (int c = threadIdx.x; c < n; c += blockDim.x)
        {
            row[c] = c == r ? T(1) : T(0);
        }
    }
}

// iperm[perm[i]] = i.
__global__ void k_inv_iperm(const int32_t* __restrict__ perm, int32_t* __restrict__ iperm, int n,
    const DeviceStatus* gate)
{
    if (gated(gate))
    {
        return;
    }
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        iperm[perm[i]] = i;
    }
}

// m[r][c] = w[r][iperm[c]]; one CTA per row at a time (the row's scattered
// reads stay in L1/L2, the writes are coalesced).
template <typename T>
__global__ void k_inv_gather(const T* __restrict__ w, const int32_t* __restrict__ iperm, T* __restrict__ m,
    int n, const DeviceStatus* gate)
{
    if (gated(gate))
    {
        return;
    }
    for (int r = blockIdx.x; r < n; r += gridDim.x)
    {
        const T* wr = w + (int64_t)r * n;
        T*       mr = m + (int64_t)r * n;
        for (int c = threadIdx.x; c < n; c += blockDim.x)
        {
            mr[c] = wr[iperm[c]];
        }
    }
}

// m[r][c] = w[min(r,c)][max(r,c)]: the upper triangle of w, mirrored.  One
// CTA per row at a time; the lower part reads w's column r (strided, once).
template <typename T>
__global__ void k_inv_sym_copy(const T* __restrict__ w, T* __restrict__ m, int n, const DeviceStatus* gate)
{
    if (gated(gate))
    {
        return;
    }
    for (int r = blockIdx.x; r < n; r += gridDim.x)
    {
        T* mr = m + (int64_t)r * n;
        for (int c = threadIdx.x; c < n; c += blockDim.x)
        {
            mr[c] = c >= r ? w[(int64_t)r * n + c] : w[(int64_t)c * n + r];
        }
    }
}

// Determinant result block in the workspace.
struct DetResult
{
    double  product;  // U's diagonal product in the input type, widened
    double  log_abs;  // sum of log|u_ii|
    int32_t swaps;    // number of i with pivot[i] != i + 1
    int32_t skipped;  // 1: LU mode met an exact zero pivot (product is 0)
};

constexpr int kDetThreads = 1024;
constexpr int kDetChunk   = 4096;

// One CTA.  The diagonal is staged in shared memory kDetChunk entries at a
// time and multiplied by thread 0 in index order; the swap count and the
// log sum are reduced in a fixed order (deterministic).
template <typename T>
__global__ void __launch_bounds__(kDetThreads) k_det(const T* __restrict__ m, int n,
    const int64_t* __restrict__ pivot, const DeviceStatus* gate, DetResult* out)
{
    __shared__ T      diag[kDetChunk];
    __shared__ double red_log[kDetThreads / 32];
    __shared__ int    red_swaps[kDetThreads / 32];
    const bool skip  = gated(gate);
    int        swaps = 0;
    double     lg    = 0.0;
    for (int i = threadIdx.x; i < n; i += kDetThreads)
    {
        swaps += pivot != nullptr && pivot[i] - 1 != i ? 1 : 0;
        lg += log(fabs((double)m[(int64_t)i * (n + 1)]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
        swaps += __shfl_xor_sync(0xffffffffu, swaps, o);
        lg += __shfl_xor_sync(0xffffffffu, lg, o);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
    {
        red_log[warp]   = lg;
        red_swaps[warp] = swaps;
    }
    T prod = T(1);
    for (int c0 = 0; c0 < n; c0 += kDetChunk)
    {
        const int cnt = min(kDetChunk, n - c0);
        __syncthreads();
        for (int i = threadIdx.x; i < cnt; i += kDetThreads)
        {
            diag[i] = m[(int64_t)(c0 + i) * (n + 1)];
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            for (int i = 0; i < cnt; ++i)
            {
                prod *= diag[i];
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double lsum = 0.0;
        int    ssum = 0;
        for (int w = 0; w < kDetThreads / 32; ++w)
        {
            lsum += red_log[w];
            ssum += red_swaps[w];
        }
        out->product = skip ? 0.0 : (double)prod;
        out->log_abs = skip ? -INFINITY : lsum;
        out->swaps   = ssum;
        out->skipped = skip ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <typename T> struct Plan
{
    GetrfPlan<T> gp;  // first: the device status block sits at the workspace start
    int32_t*     perm;
    int32_t*     iperm;
    int64_t*     piv;  // pivots when the caller passes none (LU mode)
    DetResult*   det;
    T*           w;  // n x n (inversion only)
};

template <typename T> Plan<T> plan(Arena& a, int64_t n, bool with_w)
{
    Plan<T> p;
    p.gp    = plan_getrf<T>(a);
    p.perm  = a.next<int32_t>((size_t)n);
    p.iperm = a.next<int32_t>((size_t)n);
    p.piv   = a.next<int64_t>((size_t)n);
    p.det   = a.next<DetResult>(1);
    p.w     = with_w ? a.next<T>((size_t)n * (size_t)n) : nullptr;
    return p;
}

bool lu_mode(int mode) { return mode == B200LA_LU_LINEAR_SOLVER || mode == B200LA_LU_UPFRONT_LINEAR_SOLVER; }
bool chol_mode(int mode)
{
    return mode == B200LA_CHOLESKY_LINEAR_SOLVER || mode == B200LA_CHOLESKY_UPFRONT_LINEAR_SOLVER;
}
// inversion and determinant: the LU and Cholesky modes
bool valid_mode(int mode, bool) { return lu_mode(mode) || chol_mode(mode); }

template <typename T> size_t ws_size(int64_t n, int mode, bool with_w)
{
    if (n <= 0 || n > INT_MAX / 2 || !valid_mode(mode, with_w))
    {
        return 0;
    }
    Arena a;
    plan<T>(a, n, with_w);
    return a.size();
}

// Argument checks shared by both operators; messages follow the reference's.
int check_args(const void* m, const int64_t* pivot, int64_t n, int mode, const char* op)
{
    if (m == nullptr)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "%s::apply: m must not be null", op);
    }
    if (n <= 0)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "%s::apply: lda must be positive", op);
    }
    const bool inversion = op[0] == 'i';
    if (!valid_mode(mode, inversion))
    {
        return set_error(B200LA_INVALID_ARGUMENT, "unsupported linear_solver_type (%d)", mode);
    }
    if (mode == B200LA_LU_UPFRONT_LINEAR_SOLVER && pivot == nullptr)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "%s: LU_UPFRONT needs the factors' pivot array", op);
    }
    if (n > INT_MAX / 2)
    {
        return set_error(B200LA_NOT_SUPPORTED, "%s: order too large", op);
    }
    return B200LA_SUCCESS;
}

template <typename T> int ensure_attributes()
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
    B200LA_CUDA(cudaFuncSetAttribute(k_inv_gemm<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Geo<T>::SMEM));
    if (dev >= 0 && dev < 64)
    {
        done[dev] = true;
    }
    return B200LA_SUCCESS;
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <typename T>
int launch_gemm(int M, int N, int K, const T* a, const T* b, T* c, int64_t ld, const DeviceStatus* gate,
    cudaStream_t s)
{
    const int  vec16 = aligned16(a) && aligned16(b) && aligned16(c) && ((size_t)ld * sizeof(T)) % 16 == 0;
    const dim3 grid((unsigned)((N + kTile - 1) / kTile), (unsigned)((M + kTile - 1) / kTile));
    prof_begin(KC_INV_GEMM, s);
    if constexpr (sizeof(T) == 8)
    {
        if (K <= kBandK)
        {
            // the 64-deep block-row updates: the band kernel (even work per
            // SM; C - A B from zero, rounding-equivalent)
            k_dmma_band<0><<<band_grid(M, N, device_sm_count()), kDmThreads, kBandSmem, s>>>(
                M, N, K, a, ld, b, ld, c, ld, vec16, gate);
        }
        else
        {
            const dim3 dgrid((unsigned)((N + kDmTile - 1) / kDmTile), (unsigned)((M + kDmTile - 1) / kDmTile));
            k_dmma_update<false><<<dgrid, kDmThreads, kDmSmem, s>>>(M, N, K, a, ld, b, ld, c, ld, vec16, gate);
        }
    }
    else
    {
        k_inv_gemm<T><<<grid, kThreads, Geo<T>::SMEM, s>>>(M, N, K, a, ld, b, ld, c, ld, vec16, gate);
    }
    prof_end(KC_INV_GEMM, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

// Solve one block row in place against its diagonal block: X[0:bw, 0:ncols]
// = T^-1 X with T = the bw x bw diagonal block at `a` (unit lower when
// !upper, else upper with its diagonal), in sub-blocks of kTrsmBlock rows
// taken in substitution order: k_inv_diag solves a sub-block (8 lanes
// per column group), the GEMM updates the block's remaining rows with it.
template <typename T>
int block_solve(bool upper, int bw, int ncols, const T* a, T* x, int64_t ld, const DeviceStatus* gate,
    cudaStream_t s)
{
    const int nsub = (bw + kTrsmBlock - 1) / kTrsmBlock;
    for (int step = 0; step < nsub; ++step)
    {
        int r0, sw, u0, um;
        if (!upper)
        {
            r0 = step * kTrsmBlock;
            sw = bw - r0 < kTrsmBlock ? bw - r0 : kTrsmBlock;
            u0 = r0 + sw;
            um = bw - u0;
        }
        else
        {
            const int hi = bw - step * kTrsmBlock;
            r0           = hi - kTrsmBlock > 0 ? hi - kTrsmBlock : 0;
            sw           = hi - r0;
            u0           = 0;
            um           = r0;
        }
        prof_begin(KC_SOLVE, s);
        const unsigned grid = (unsigned)((ncols + kDiagCols - 1) / kDiagCols);
        if (upper)
        {
            k_inv_diag<T, true><<<grid, kDiagThreads, 0, s>>>(a, ld, r0, sw, x, ld, ncols, gate);
        }
        else
        {
            k_inv_diag<T, false><<<grid, kDiagThreads, 0, s>>>(a, ld, r0, sw, x, ld, ncols, gate);
        }
        prof_end(KC_SOLVE, s);
        B200LA_LAUNCH_CHECK();
        if (um > 0)
        {
            const int rc = launch_gemm<T>(um, ncols, sw, a + (int64_t)u0 * ld + r0, x + (int64_t)r0 * ld,
                x + (int64_t)u0 * ld, ld, gate, s);
            if (rc != B200LA_SUCCESS)
            {
                return rc;
            }
        }
    }
    return B200LA_SUCCESS;
}

// Factor (LU, CHOLESKY) or reset the status (the UPFRONT modes); gate = the
// status block.  chol_upper: the Cholesky factor ends in the upper triangle
// (U = L^T, the inversion's form; the given lower one moved there for
// CHOLESKY_UPFRONT), else it stays lower (the determinant's form).
template <typename T>
int enqueue_factor(T* m, int n, int64_t* piv, int mode, const Plan<T>& p, cudaStream_t s, bool chol_upper = false)
{
    if (mode == B200LA_LU_LINEAR_SOLVER)
    {
        return enqueue_getrf<T>(m, n, piv, p.gp, s);
    }
    if (mode == B200LA_CHOLESKY_LINEAR_SOLVER)
    {
        return enqueue_potrf<T>(m, n, chol_upper, p.gp.st, s);
    }
    if (mode == B200LA_CHOLESKY_UPFRONT_LINEAR_SOLVER)
    {
        prof_begin(KC_INV_AUX, s);
        k_status_init<<<1, 32, 0, s>>>(p.gp.st, nullptr);
        prof_end(KC_INV_AUX, s);
        B200LA_LAUNCH_CHECK();
        if (chol_upper)
        {
            prof_begin(KC_INV_AUX, s);
            k_chol_to_upper<T><<<grid_1d((int64_t)n * n, 256), 256, 0, s>>>(m, n, p.gp.st);
            prof_end(KC_INV_AUX, s);
            B200LA_LAUNCH_CHECK();
        }
        return B200LA_SUCCESS;
    }
    prof_begin(KC_INV_AUX, s);
    k_status_init<<<1, 32, 0, s>>>(p.gp.st, p.gp.perm);
    prof_end(KC_INV_AUX, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

// W = U^-1 W with U the upper triangle of m (its diagonal included), all n
// columns: from the bottom block row, the block row solved against its
// diagonal block, then the rows above it updated by one GEMM.
template <typename T> int upper_solve(const T* m, T* w, int n, const DeviceStatus* gate, cudaStream_t s)
{
    const int64_t ld      = n;
    const int     nblocks = (n + kNB - 1) / kNB;
    for (int b = nblocks - 1; b >= 0; --b)
    {
        const int k0 = b * kNB, bw = n - k0 < kNB ? n - k0 : kNB;
        int rc = block_solve<T>(true, bw, n, m + (int64_t)k0 * ld + k0, w + (int64_t)k0 * ld, ld, gate, s);
        if (rc != B200LA_SUCCESS)
        {
            return rc;
        }
        if (k0 > 0)
        {
            rc = launch_gemm<T>(k0, n, bw, m + k0, w + (int64_t)k0 * ld, w, ld, gate, s);
            if (rc != B200LA_SUCCESS)
            {
                return rc;
            }
        }
    }
    return B200LA_SUCCESS;
}

template <typename T> int enqueue_inverse(T* m, int n, const int64_t* piv, const Plan<T>& p, cudaStream_t s)
{
    const DeviceStatus* gate = p.gp.st;
    const int           sms  = device_sm_count();
    const int           rows = n < 4 * sms ? n : 4 * sms;
    const size_t        psm  = perm_smem_bytes(n);
    prof_begin(KC_INV_AUX, s);
    k_perm_from_pivots<0><<<1, 256, psm, s>>>(piv, n, p.perm, psm > 0 ? 1 : 0, p.gp.st, gate);
    prof_end(KC_INV_AUX, s);
    B200LA_LAUNCH_CHECK();
    prof_begin(KC_INV_AUX, s);
    k_inv_iperm<<<grid_1d(n, 256), 256, 0, s>>>(p.perm, p.iperm, n, gate);
    prof_end(KC_INV_AUX, s);
    B200LA_LAUNCH_CHECK();
    prof_begin(KC_INV_AUX, s);
    k_inv_identity<T><<<rows, 256, 0, s>>>(p.w, n, gate);
    prof_end(KC_INV_AUX, s);
    B200LA_LAUNCH_CHECK();

    const int64_t ld      = n;
    const int     nblocks = (n + kNB - 1) / kNB;
    // W = L^-1 W: block row solve, then the rows below, columns [0, k1).
    for (int b = 0; b < nblocks; ++b)
    {
        const int k0 = b * kNB, bw = n - k0 < kNB ? n - k0 : kNB, k1 = k0 + bw;
        int rc = block_solve<T>(false, bw, k1, m + (int64_t)k0 * ld + k0, p.w + (int64_t)k0 * ld, ld, gate, s);
        if (rc != B200LA_SUCCESS)
        {
            return rc;
        }
        if (k1 < n)
        {
            rc = launch_gemm<T>(n - k1, k1, bw, m + (int64_t)k1 * ld + k0, p.w + (int64_t)k0 * ld,
                p.w + (int64_t)k1 * ld, ld, gate, s);
            if (rc != B200LA_SUCCESS)
            {
                return rc;
            }
        }
    }
    const int rc = upper_solve<T>(m, p.w, n, gate, s);
    if (rc != B200LA_SUCCESS)
    {
        return rc;
    }
    prof_begin(KC_INV_AUX, s);
    k_inv_gather<T><<<rows, 256, 0, s>>>(p.w, p.iperm, m, n, gate);
    prof_end(KC_INV_AUX, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

// The Cholesky modes after the factor is in m's upper triangle: W = I,
// W = U^-1 W, W = W^T, W = U^-1 W, m = W (upper triangle mirrored).
template <typename T> int enqueue_chol_inverse(T* m, int n, const Plan<T>& p, cudaStream_t s)
{
    const DeviceStatus* gate = p.gp.st;
    const int           sms  = device_sm_count();
    const int           rows = n < 4 * sms ? n : 4 * sms;
    prof_begin(KC_INV_AUX, s);
    k_inv_identity<T><<<rows, 256, 0, s>>>(p.w, n, gate);
    prof_end(KC_INV_AUX, s);
    B200LA_LAUNCH_CHECK();
    int rc = upper_solve<T>(m, p.w, n, gate, s);
    if (rc != B200LA_SUCCESS)
    {
        return rc;
    }
    // in place, square: no workspace (not gated: after a failed
    // factorization it only moves the unused scratch)
    if constexpr (sizeof(T) == 8)
    {
        rc = b200la_dtranspose(n, n, p.w, nullptr, 0, s);
    }
    else
    {
        rc = b200la_stranspose(n, n, p.w, nullptr, 0, s);
    }
    if (rc != B200LA_SUCCESS)
    {
        return rc;
    }
    rc = upper_solve<T>(m, p.w, n, gate, s);
    if (rc != B200LA_SUCCESS)
    {
        return rc;
    }
    prof_begin(KC_INV_AUX, s);
    k_inv_sym_copy<T><<<rows, 256, 0, s>>>(p.w, m, n, gate);
    prof_end(KC_INV_AUX, s);
    B200LA_LAUNCH_CHECK();
    return B200LA_SUCCESS;
}

template <typename T>
int inverse(T* m, int64_t* pivot, int64_t n, int mode, void* ws, size_t bytes, void* stream)
{
    int st = check_args(m, pivot, n, mode, "inversion");
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    const size_t need = ws_size<T>(n, mode, true);
    if (ws == nullptr || bytes < need)
    {
        return set_error(B200LA_WORKSPACE_TOO_SMALL,
            "inversion: workspace is null or too small (%zu < %zu bytes)", bytes, need);
    }
    st = prepare<T>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    st = ensure_attributes<T>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    Arena        a(ws, bytes);
    Plan<T>      p   = plan<T>(a, n, true);
    cudaStream_t s   = as_stream(stream);
    if (chol_mode(mode))
    {
        st = enqueue_factor<T>(m, (int)n, nullptr, mode, p, s, true);
        if (st != B200LA_SUCCESS)
        {
            return st;
        }
        return enqueue_chol_inverse<T>(m, (int)n, p, s);
    }
    int64_t* piv = pivot != nullptr ? pivot : p.piv;
    st           = enqueue_factor<T>(m, (int)n, piv, mode, p, s);
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    return enqueue_inverse<T>(m, (int)n, piv, p, s);
}

template <typename T>
int determinant(T* m, int64_t* pivot, int64_t n, int mode, T* product, int* sign, double* log_abs, void* ws,
    size_t bytes, void* stream)
{
    int st = check_args(m, pivot, n, mode, "determinant");
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    if (product == nullptr)
    {
        return set_error(B200LA_INVALID_ARGUMENT, "determinant: the result pointer must not be null");
    }
    const size_t need = ws_size<T>(n, mode, false);
    if (ws == nullptr || bytes < need)
    {
        return set_error(B200LA_WORKSPACE_TOO_SMALL,
            "determinant: workspace is null or too small (%zu < %zu bytes)", bytes, need);
    }
    st = prepare<T>();
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    Arena        a(ws, bytes);
    Plan<T>      p    = plan<T>(a, n, false);
    cudaStream_t s    = as_stream(stream);
    const bool   chol = chol_mode(mode);
    int64_t*     piv  = chol ? nullptr : pivot != nullptr ? pivot : p.piv;
    st                = enqueue_factor<T>(m, (int)n, piv, mode, p, s);
    if (st != B200LA_SUCCESS)
    {
        return st;
    }
    prof_begin(KC_INV_AUX, s);
    k_det<T><<<1, kDetThreads, 0, s>>>(m, (int)n, piv, p.gp.st, p.det);
    prof_end(KC_INV_AUX, s);
    B200LA_LAUNCH_CHECK();
    DetResult h{};
    B200LA_CUDA(cudaMemcpyAsync(&h, p.det, sizeof(h), cudaMemcpyDeviceToHost, s));
    int info = 0;
    st       = read_status(p.gp.st, &info, s);  // synchronizes s
    if (st < 0)
    {
        return st;
    }
    *product = (T)h.product;
    if (sign != nullptr)
    {
        *sign = (h.swaps & 1) ? -1 : 1;
    }
    if (log_abs != nullptr)
    {
        *log_abs = chol ? 2.0 * h.log_abs : h.log_abs;  // det(A) = (prod l_ii)^2
    }
    return h.skipped ? B200LA_SINGULAR : B200LA_SUCCESS;
}

}  // namespace inv
}  // namespace b200la

using namespace b200la;

extern "C" {

B200LA_API size_t b200la_dinverse_workspace_size(int64_t n, int mode) { return inv::ws_size<double>(n, mode, true); }
B200LA_API size_t b200la_sinverse_workspace_size(int64_t n, int mode) { return inv::ws_size<float>(n, mode, true); }
B200LA_API int    b200la_dinverse(double* m, int64_t* pivot, int64_t n, int mode, void* ws, size_t bytes, void* stream)
{
    return inv::inverse<double>(m, pivot, n, mode, ws, bytes, stream);
}
B200LA_API int b200la_sinverse(float* m, int64_t* pivot, int64_t n, int mode, void* ws, size_t bytes, void* stream)
{
    return inv::inverse<float>(m, pivot, n, mode, ws, bytes, stream);
}

B200LA_API size_t b200la_ddeterminant_workspace_size(int64_t n, int mode) { return inv::ws_size<double>(n, mode, false); }
B200LA_API size_t b200la_sdeterminant_workspace_size(int64_t n, int mode) { return inv::ws_size<float>(n, mode, false); }
B200LA_API int    b200la_ddeterminant(double* m, int64_t* pivot, int64_t n, int mode, double* product, int* sign,
       double* log_abs, void* ws, size_t bytes, void* stream)
{
    return inv::determinant<double>(m, pivot, n, mode, product, sign, log_abs, ws, bytes, stream);
}
B200LA_API int b200la_sdeterminant(float* m, int64_t* pivot, int64_t n, int mode, float* product, int* sign,
    double* log_abs, void* ws, size_t bytes, void* stream)
{
    return inv::determinant<float>(m, pivot, n, mode, product, sign, log_abs, ws, bytes, stream);
}

}  // extern "C"
