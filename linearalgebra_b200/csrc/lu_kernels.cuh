// Blocked right-looking LU with partial pivoting on a row-major n x n matrix
// (lda == n), one panel of width NB = 64 at a time:
//
//   k_panel        factor columns [k, k+w) of rows [k, n): per column a
//                  pivot search over every remaining row, the row swap
//                  inside the panel, the multipliers and the rank-1 update of
//                  the panel's remaining columns.  One cooperative grid; each
//                  CTA keeps its slice of panel rows in shared memory; the
//                  CTAs agree on each pivot through one exchange of
//                  per-CTA candidates (value, row index and the candidate's
//                  panel row) in global memory, with bounded waits.
//   k_laswp_trsm   apply the panel's row interchanges to the columns left and
//                  right of the panel (as one gather/scatter of the rows they
//                  touch) and, right of the panel, U12 = L11^-1 A12.
//   k_trailing     A22 -= L21 U12.
//
// Arithmetic follows the reference's NATIVE LU operation for operation
// (src/matrix_operation/cpu/native/lu_decomposition_native.cpp): the same
// panel width, the same reciprocal-or-divide multiplier rule, a fused
// multiply-add per update in the same per-element order, and the trailing
// update formed as delta = L21 U12 (accumulated from zero over the panel's
// columns in order) followed by a separate A22 - delta.  The factors and
// pivots are therefore the same numbers the reference computes.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cfloat>
#include <climits>

#include "common.cuh"

namespace b200la
{

constexpr int kNB           = 64;   // panel width (reference kLuBlockSize)
constexpr int kPanelThreads = 256;
constexpr int kMaxPanelCtas = 256;
constexpr int kSwapCols     = 64;   // columns per CTA in k_laswp_trsm

template <typename T> struct Vec2;
template <> struct Vec2<double>
{
    using type = double2;
};
template <> struct Vec2<float>
{
    using type = float2;
};

template <typename T> struct Limits;
template <> struct Limits<double>
{
    __device__ static constexpr double min_normal() { return DBL_MIN; }
};
template <> struct Limits<float>
{
    __device__ static constexpr float min_normal() { return FLT_MIN; }
};

// One per-CTA candidate of the pivot exchange.  `seq` = global column + 1
// marks the slot as filled for that column (the workspace is cleared at the
// start of every factorization).
struct alignas(16) SlotHeader
{
    double   key;
    int32_t  row;
    uint32_t seq;
};

// Row interchanges of one panel, as a permutation of the rows they touch:
// row dst[q] receives the pre-panel contents of row src[q], q < count.
// Slots q < w are the panel's own rows k+q.
struct PermList
{
    int32_t count;
    int32_t pad[63];
    int32_t dst[2 * kNB];
    int32_t src[2 * kNB];
};

template <typename T> struct PanelWs
{
    SlotHeader* hdr;      // [2][kMaxPanelCtas]
    T*          payload;  // [2][kMaxPanelCtas][kNB]
    T*          diag;     // [2][kNB]
    PermList*   perm;
};

// (key, row) ordering of the pivot search: larger key wins, equal keys go to
// the lower row, i.e. the first maximum in row order like the reference's
// sequential strict '>' scan.
__device__ __forceinline__ bool better(double ka, int ra, double kb, int rb)
{
    return ka > kb || (ka == kb && ra < rb);
}

// Pivot-search key of row `gr` for the column whose diagonal row is `c`.  The
// reference starts from |a_cc| and only lets a strictly larger |a_rc| replace
// it, so a NaN candidate below the diagonal never wins, and a NaN on the
// diagonal is never displaced.
template <typename T> __device__ __forceinline__ double pivot_key(T v, int gr, int c)
{
    const bool nan = v != v;
    if (gr == c)
    {
        return nan ? __longlong_as_double(0x7ff0000000000000ll) : (double)fabs(v);
    }
    return nan ? -1.0 : (double)fabs(v);
}

template <typename T>
__global__ void __launch_bounds__(kPanelThreads) k_panel(T* __restrict__ A, int n, int k, int w,
    int rows_per_cta, int in_smem, int64_t* __restrict__ pivot, PanelWs<T> ws,
    DeviceStatus* __restrict__ st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ T      urow[kNB];
    __shared__ int    piv_loc[kNB];
    __shared__ double red_key[kPanelThreads / 32];
    __shared__ int    red_row[kPanelThreads / 32];
    __shared__ int    s_p, s_g, s_abort;

    const int tid  = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int G    = gridDim.x;
    const int b    = blockIdx.x;
    const int r0   = k + b * rows_per_cta;
    const int nloc = max(0, min(n, r0 + rows_per_cta) - r0);

    T*           loc;
    const size_t ldl = in_smem ? (size_t)(kNB + 1) : (size_t)n;
    if (in_smem)
    {
        loc = reinterpret_cast<T*>(smem_raw);
        for (int e = tid; e < nloc * w; e += kPanelThreads)
        {
            const int r = e / w, c = e - (e / w) * w;
            loc[r * ldl + c] = A[(size_t)(r0 + r) * n + k + c];
        }
    }
    else
    {
        loc = A + (size_t)r0 * n + k;
    }
    if (tid == 0)
    {
        s_abort = 0;
    }
    __syncthreads();

    int64_t first_zero = -1;
    for (int jj = 0; jj < w; ++jj)
    {
        const int c   = k + jj;
        const int par = jj & 1;

        // ---- local candidate: best (key, row) over owned rows >= c
        double best    = -2.0;
        int    bestrow = INT_MAX;
        for (int r = max(0, c - r0) + tid; r < nloc; r += kPanelThreads)
        {
            const double key = pivot_key(loc[r * ldl + jj], r0 + r, c);
            if (better(key, r0 + r, best, bestrow))
            {
                best    = key;
                bestrow = r0 + r;
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
        {
            const double ok = __shfl_down_sync(0xffffffffu, best, off);
            const int    orow = __shfl_down_sync(0xffffffffu, bestrow, off);
            if (better(ok, orow, best, bestrow))
            {
                best    = ok;
                bestrow = orow;
            }
        }
        if (lane == 0)
        {
            red_key[warp] = best;
            red_row[warp] = bestrow;
        }
        __syncthreads();
        if (tid == 0)
        {
            for (int q = 1; q < kPanelThreads / 32; ++q)
            {
                if (better(red_key[q], red_row[q], best, bestrow))
                {
                    best    = red_key[q];
                    bestrow = red_row[q];
                }
            }
            red_key[0] = best;
            red_row[0] = bestrow;
        }
        __syncthreads();
        best    = red_key[0];
        bestrow = red_row[0];

        // ---- publish: candidate row, then (owner of row c) the diagonal row
        SlotHeader* H = ws.hdr + par * kMaxPanelCtas;
        if (bestrow != INT_MAX)
        {
            T* P = ws.payload + ((size_t)par * kMaxPanelCtas + b) * kNB;
            for (int cc = tid; cc < w; cc += kPanelThreads)
            {
                P[cc] = loc[(size_t)(bestrow - r0) * ldl + cc];
            }
        }
        if (c >= r0 && c < r0 + nloc)
        {
            T* D = ws.diag + par * kNB;
            for (int cc = tid; cc < w; cc += kPanelThreads)
            {
                D[cc] = loc[(size_t)(c - r0) * ldl + cc];
            }
        }
        __syncthreads();
        if (tid == 0)
        {
            H[b].key = best;
            H[b].row = bestrow;
            __threadfence();
            st_release_u32(&H[b].seq, (uint32_t)(c + 1));
        }

        // ---- gather every CTA's candidate (bounded wait), pick the pivot
        if (warp == 0)
        {
            double wk = -2.0;
            int    wr = INT_MAX, wg = -1;
            bool   timed_out = false;
            for (int g = lane; g < G; g += 32)
            {
                const uint64_t t0    = global_ns();
                uint32_t       polls = 0;
                while (ld_acquire_u32(&H[g].seq) != (uint32_t)(c + 1))
                {
                    if ((++polls & 255u) == 0 && global_ns() - t0 > kWaitLimitNs)
                    {
                        timed_out = true;
                        break;
                    }
                }
                if (timed_out)
                {
                    break;
                }
                const double kg = __ldcg(&H[g].key);
                const int    rg = __ldcg(&H[g].row);
                if (better(kg, rg, wk, wr))
                {
                    wk = kg;
                    wr = rg;
                    wg = g;
                }
            }
            if (__any_sync(0xffffffffu, timed_out))
            {
                if (lane == 0)
                {
                    raise_error(st, DEV_WAIT_TIMEOUT, 1);
                    s_abort = 1;
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
            {
                const double ok = __shfl_down_sync(0xffffffffu, wk, off);
                const int    orow = __shfl_down_sync(0xffffffffu, wr, off);
                const int    og = __shfl_down_sync(0xffffffffu, wg, off);
                if (better(ok, orow, wk, wr))
                {
                    wk = ok;
                    wr = orow;
                    wg = og;
                }
            }
            if (lane == 0)
            {
                s_p = wr;
                s_g = wg;
            }
        }
        __syncthreads();
        if (s_abort)
        {
            return;
        }
        const int p = s_p;
        const int g = s_g;
        if (tid == 0)
        {
            piv_loc[jj] = p;
            if (b == 0)
            {
                pivot[c] = (int64_t)p + 1;
            }
        }
        {
            const T* P = ws.payload + ((size_t)par * kMaxPanelCtas + g) * kNB;
            for (int cc = tid; cc < w; cc += kPanelThreads)
            {
                urow[cc] = __ldcg(P + cc);
            }
        }
        __syncthreads();

        // ---- swap rows c and p inside the panel
        if (p != c)
        {
            if (c >= r0 && c < r0 + nloc)
            {
                for (int cc = tid; cc < w; cc += kPanelThreads)
                {
                    loc[(size_t)(c - r0) * ldl + cc] = urow[cc];
                }
            }
            if (p >= r0 && p < r0 + nloc)
            {
                const T* D = ws.diag + par * kNB;
                for (int cc = tid; cc < w; cc += kPanelThreads)
                {
                    loc[(size_t)(p - r0) * ldl + cc] = __ldcg(D + cc);
                }
            }
        }
        __syncthreads();

        // ---- multipliers and rank-1 update of rows > c
        const T d = urow[jj];
        if (d == T(0))
        {
            if (first_zero < 0)
            {
                first_zero = c;
            }
            continue;
        }
        const bool use_recip = fabs(d) >= Limits<T>::min_normal();
        const T    recip     = use_recip ? (T)(T(1) / d) : T(1);
        const int  rbeg      = max(0, c + 1 - r0);
        for (int r = rbeg + tid; r < nloc; r += kPanelThreads)
        {
            T& l = loc[(size_t)r * ldl + jj];
            l    = use_recip ? l * recip : l / d;
        }
        __syncthreads();
        const int wrem = w - jj - 1;
        if (wrem > 0)
        {
            // 4 row lanes x 64 column lanes
            const int cl = tid & 63;
            const int rl = tid >> 6;
            if (cl < wrem)
            {
                const int cc = jj + 1 + cl;
                const T   u  = urow[cc];
                for (int r = rbeg + rl; r < nloc; r += kPanelThreads / 64)
                {
                    T* row = loc + (size_t)r * ldl;
                    row[cc] = fma(-row[jj], u, row[cc]);
                }
            }
        }
        __syncthreads();
    }

    // ---- write the factored slice back
    if (in_smem)
    {
        for (int e = tid; e < nloc * w; e += kPanelThreads)
        {
            const int r = e / w, c = e - (e / w) * w;
            A[(size_t)(r0 + r) * n + k + c] = loc[r * ldl + c];
        }
    }

    if (b == 0)
    {
        if (tid == 0 && first_zero >= 0)
        {
            if (st->first_zero < 0)
            {
                st->first_zero = first_zero;
            }
        }
        // The panel's interchanges as one permutation of the rows they touch.
        if (warp == 0)
        {
            __shared__ int pos_s[2 * kNB];
            __shared__ int cont_s[2 * kNB];
            __shared__ int cnt_s;
            for (int q = lane; q < w; q += 32)
            {
                pos_s[q]  = k + q;
                cont_s[q] = k + q;
            }
            if (lane == 0)
            {
                cnt_s = w;
            }
            __syncwarp();
            for (int jj = 0; jj < w; ++jj)
            {
                const int i = k + jj;
                const int p = piv_loc[jj];
                if (p == i)
                {
                    continue;
                }
                int slot_p;
                if (p < k + w)
                {
                    slot_p = p - k;
                }
                else
                {
                    const int cnt = cnt_s;
                    slot_p        = -1;
                    for (int q0 = w; q0 < cnt; q0 += 32)
                    {
                        const int      q   = q0 + lane;
                        const unsigned hit = __ballot_sync(0xffffffffu, q < cnt && pos_s[q] == p);
                        if (hit)
                        {
                            slot_p = q0 + __ffs(hit) - 1;
                            break;
                        }
                    }
                    if (slot_p < 0)
                    {
                        slot_p = cnt;
                        __syncwarp();
                        if (lane == 0)
                        {
                            pos_s[slot_p]  = p;
                            cont_s[slot_p] = p;
                            cnt_s          = cnt + 1;
                        }
                    }
                }
                __syncwarp();
                if (lane == 0)
                {
                    const int t     = cont_s[jj];
                    cont_s[jj]      = cont_s[slot_p];
                    cont_s[slot_p]  = t;
                }
                __syncwarp();
            }
            const int cnt = cnt_s;
            for (int q = lane; q < cnt; q += 32)
            {
                ws.perm->dst[q] = pos_s[q];
                ws.perm->src[q] = cont_s[q];
            }
            if (lane == 0)
            {
                ws.perm->count = cnt;
            }
        }
    }
}

// Row interchanges outside the panel and, right of it, U12 = L11^-1 A12.
// CTA b < n_left: columns [b*kSwapCols, ...) of [0, k); otherwise columns of
// [k+w, n).  One thread per column.
template <typename T>
__global__ void __launch_bounds__(kSwapCols) k_laswp_trsm(T* __restrict__ A, int n, int k, int w,
    const PermList* __restrict__ perm, int n_left)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T(*staged)[kSwapCols] = reinterpret_cast<T(*)[kSwapCols]>(smem_raw);           // [2*kNB]
    T(*L11)[kNB + 1]      = reinterpret_cast<T(*)[kNB + 1]>(smem_raw + sizeof(T) * 2 * kNB * kSwapCols);

    const int  tid   = threadIdx.x;
    const bool left  = (int)blockIdx.x < n_left;
    const int  c0    = left ? blockIdx.x * kSwapCols : k + w + (blockIdx.x - n_left) * kSwapCols;
    const int  cend  = left ? k : n;
    const int  col   = c0 + tid;
    const bool valid = col < cend;
    const int  cnt   = perm->count;

    for (int q = 0; q < cnt; ++q)
    {
        staged[q][tid] = valid ? A[(size_t)perm->src[q] * n + col] : T(0);
    }
    if (left)
    {
        if (valid)
        {
            for (int q = 0; q < cnt; ++q)
            {
                if (perm->dst[q] != perm->src[q])
                {
                    A[(size_t)perm->dst[q] * n + col] = staged[q][tid];
                }
            }
        }
        return;
    }
    // rows displaced below the panel
    if (valid)
    {
        for (int q = w; q < cnt; ++q)
        {
            A[(size_t)perm->dst[q] * n + col] = staged[q][tid];
        }
    }
    // L11 (unit lower, strictly below the diagonal)
    for (int e = tid; e < w * w; e += kSwapCols)
    {
        const int i = e / w, p = e - (e / w) * w;
        L11[i][p]   = p < i ? A[(size_t)(k + i) * n + k + p] : T(0);
    }
    __syncthreads();
    if (!valid)
    {
        return;
    }
    T x[kNB];
#pragma unroll
    for (int i = 0; i < kNB; ++i)
    {
        x[i] = i < w ? staged[i][tid] : T(0);
    }
    // column-oriented forward substitution: row i receives the updates of
    // rows 0..i-1 in that order, as in the reference's row-axpy loop
#pragma unroll
    for (int p = 0; p < kNB; ++p)
    {
        if (p < w)
        {
#pragma unroll
            for (int i = p + 1; i < kNB; ++i)
            {
                if (i < w)
                {
                    x[i] = fma(-L11[i][p], x[p], x[i]);
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < kNB; ++i)
    {
        if (i < w)
        {
            A[(size_t)(k + i) * n + col] = x[i];
        }
    }
}

// Trailing update A22 -= L21 U12 for one 128 x 64 tile of A22 per CTA.
// delta is accumulated per element from zero over the panel's w columns in
// order with fused multiply-adds, then subtracted from A22 once.
// Thread (warp, tr = lane/8, tc = lane%8) owns rows warp*32 + tr + 4i
// (i < 8) and columns 2*tc + 16*j + e (j < 4, e < 2) of the tile.
constexpr int kTileM = 128;
constexpr int kTileN = 64;

template <typename T>
__global__ void __launch_bounds__(128, 2) k_trailing(T* __restrict__ A, int n, int k, int w)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* As = reinterpret_cast<T*>(smem_raw);   // [kTileM][kNB + 1]
    T* Bs = As + kTileM * (kNB + 1);           // [kNB][kTileN]

    const int rest = n - k - w;
    const int m0   = blockIdx.y * kTileM;
    const int n0   = blockIdx.x * kTileN;
    const int tid  = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int tr   = lane >> 3;
    const int tc   = lane & 7;

    const T* L21 = A + (size_t)(k + w) * n + k;
    const T* U12 = A + (size_t)k * n + k + w;
    T*       C   = A + (size_t)(k + w) * n + k + w;

    for (int e = tid; e < kTileM * kNB; e += 128)
    {
        const int r = e / kNB, p = e % kNB;
        As[r * (kNB + 1) + p] = (m0 + r < rest && p < w) ? L21[(size_t)(m0 + r) * n + p] : T(0);
    }
    for (int e = tid; e < kNB * kTileN; e += 128)
    {
        const int p = e / kTileN, cc = e % kTileN;
        Bs[p * kTileN + cc] = (p < w && n0 + cc < rest) ? U12[(size_t)p * n + n0 + cc] : T(0);
    }
    __syncthreads();

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
    const T* arow = As + (warp * 32 + tr) * (kNB + 1);
    for (int p = 0; p < w; ++p)
    {
        T a[8], bv[8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
        {
            a[i] = arow[4 * i * (kNB + 1) + p];
        }
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const auto v2 = *reinterpret_cast<const typename Vec2<T>::type*>(
                Bs + p * kTileN + 2 * tc + 16 * j);
            bv[2 * j]     = v2.x;
            bv[2 * j + 1] = v2.y;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i)
        {
#pragma unroll
            for (int j = 0; j < 8; ++j)
            {
                acc[i][j] = fma(a[i], bv[j], acc[i][j]);
            }
        }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
    {
        const int r = m0 + warp * 32 + tr + 4 * i;
        if (r < rest)
        {
            T* crow = C + (size_t)r * n;
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
#pragma unroll
                for (int e = 0; e < 2; ++e)
                {
                    const int cc = n0 + 2 * tc + 16 * j + e;
                    if (cc < rest)
                    {
                        crow[cc] = crow[cc] - acc[i][2 * j + e];
                    }
                }
            }
        }
    }
}

__global__ void k_status_init(DeviceStatus* st, PermList* perm)
{
    if (threadIdx.x == 0)
    {
        st->error      = 0;
        st->error_site = 0;
        st->first_zero = -1;
        st->info       = 0;
        perm->count    = 0;
    }
}

__global__ void k_status_finish(DeviceStatus* st)
{
    if (threadIdx.x == 0)
    {
        st->info = st->first_zero + 1;
    }
}

}  // namespace b200la
