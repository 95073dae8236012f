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

#include <cooperative_groups.h>

#include <cfloat>
#include <climits>

#include "common.cuh"

namespace b200la
{

constexpr int kNB           = 64;   // panel width (reference kLuBlockSize)
constexpr int kPanelThreads = 256;
constexpr int kMaxPanelCtas = 160;  // >= the SM count of a B200 (148)
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

template <typename T> struct Vec16;
template <> struct Vec16<double>
{
    using type = double2;
};
template <> struct Vec16<float>
{
    using type = float4;
};

// Row stride of a panel slice held in shared memory: 64 values plus 16 bytes
// of padding, so rows stay 16-byte aligned for vector access while
// consecutive rows start in different banks.
template <typename T> constexpr int panel_ldl() { return kNB + 16 / (int)sizeof(T); }

template <typename T> struct Limits;
template <> struct Limits<double>
{
    __device__ static constexpr double min_normal() { return DBL_MIN; }
};
template <> struct Limits<float>
{
    __device__ static constexpr float min_normal() { return FLT_MIN; }
};

// The pivot exchange of k_panel uses self-validating 8-byte words: the low
// half carries 4 data bytes, the high half the flag of the column being
// exchanged (global column + 1).  An aligned 8-byte access is single-copy
// atomic, so a reader that sees the expected flag in every word it needs has
// the data of that column without any release/acquire fence.  The exchange
// buffers are cleared at the start of every factorization.
__device__ __forceinline__ uint64_t ll_word(uint32_t data, uint32_t flag)
{
    return ((uint64_t)flag << 32) | data;
}
__device__ __forceinline__ void st_u64x2(uint64_t* p, uint64_t a, uint64_t b)
{
    asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b) : "memory");
}
__device__ __forceinline__ void st_u64(uint64_t* p, uint64_t a)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(a) : "memory");
}
__device__ __forceinline__ void ld_u64x2(const uint64_t* p, uint64_t& a, uint64_t& b)
{
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p) : "memory");
}
__device__ __forceinline__ uint64_t ld_u64(const uint64_t* p)
{
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

template <typename T> struct LLWords;
template <> struct LLWords<double>
{
    static constexpr int kWords = 2;
};
template <> struct LLWords<float>
{
    static constexpr int kWords = 1;
};

__device__ __forceinline__ void ll_store(uint64_t* base, int idx, double v, uint32_t flag)
{
    const uint64_t bits = (uint64_t)__double_as_longlong(v);
    st_u64x2(base + 2 * idx, ll_word((uint32_t)bits, flag), ll_word((uint32_t)(bits >> 32), flag));
}
__device__ __forceinline__ void ll_store(uint64_t* base, int idx, float v, uint32_t flag)
{
    st_u64(base + idx, ll_word(__float_as_uint(v), flag));
}
__device__ __forceinline__ bool ll_load(const uint64_t* base, int idx, uint32_t flag, double& v)
{
    uint64_t a, b;
    ld_u64x2(base + 2 * idx, a, b);
    if ((uint32_t)(a >> 32) != flag || (uint32_t)(b >> 32) != flag)
    {
        return false;
    }
    v = __longlong_as_double((long long)(((b & 0xffffffffull) << 32) | (a & 0xffffffffull)));
    return true;
}
__device__ __forceinline__ bool ll_load(const uint64_t* base, int idx, uint32_t flag, float& v)
{
    const uint64_t a = ld_u64(base + idx);
    if ((uint32_t)(a >> 32) != flag)
    {
        return false;
    }
    v = __uint_as_float((uint32_t)a);
    return true;
}

// Header of one CTA's candidate: 4 words = key (2), row, unused.
constexpr int kHdrWords = 4;

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
    uint64_t* hdr;      // [2][kMaxPanelCtas][kHdrWords]
    uint64_t* payload;  // [2][kMaxPanelCtas][kNB * LLWords<T>::kWords]
    uint64_t* diag;     // [2][kNB * LLWords<T>::kWords]
    PermList* perm;
};

template <typename T> constexpr size_t panel_hdr_words() { return (size_t)2 * kMaxPanelCtas * kHdrWords; }
template <typename T> constexpr size_t panel_payload_words()
{
    return (size_t)2 * kMaxPanelCtas * kNB * LLWords<T>::kWords;
}
template <typename T> constexpr size_t panel_diag_words() { return (size_t)2 * kNB * LLWords<T>::kWords; }

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

// The interchanges of one panel (pivot rows piv_loc[0..w), 0-based) as one
// permutation of the rows they touch (PermList).  Run by one warp.
static __device__ __noinline__ void build_perm_list(const int* piv_loc, int k, int w, PermList* perm, int lane)
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
            const int t    = cont_s[jj];
            cont_s[jj]     = cont_s[slot_p];
            cont_s[slot_p] = t;
        }
        __syncwarp();
    }
    const int cnt = cnt_s;
    for (int q = lane; q < cnt; q += 32)
    {
        perm->dst[q] = pos_s[q];
        perm->src[q] = cont_s[q];
    }
    if (lane == 0)
    {
        perm->count = cnt;
    }
}

__device__ __forceinline__ void warp_best(double& key, int& row)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        const double ok   = __shfl_down_sync(0xffffffffu, key, off);
        const int    orow = __shfl_down_sync(0xffffffffu, row, off);
        if (better(ok, orow, key, row))
        {
            key = ok;
            row = orow;
        }
    }
}

// Block-wide best (key, row): every thread passes its own candidate; all
// threads get the result.  Two barriers.
__device__ __forceinline__ void block_best(double& key, int& row, double* red_key, int* red_row)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    warp_best(key, row);
    if (lane == 0)
    {
        red_key[warp] = key;
        red_row[warp] = row;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        for (int q = 1; q < kPanelThreads / 32; ++q)
        {
            if (better(red_key[q], red_row[q], key, row))
            {
                key = red_key[q];
                row = red_row[q];
            }
        }
        red_key[kPanelThreads / 32] = key;
        red_row[kPanelThreads / 32] = row;
    }
    __syncthreads();
    key = red_key[kPanelThreads / 32];
    row = red_row[kPanelThreads / 32];
}

// Multipliers and rank-1 update of the panel rows below the diagonal row c
// for column jj, one thread per row, plus that thread's best candidate for
// the next column.  Per element the operations are the reference's:
// l = a_rj * (1/d) (or a_rj / d), then a_rc = fma(-l, u_c, a_rc) for c > j.
template <typename T>
__device__ __forceinline__ void panel_update_rows(T* loc, size_t ldl, int rbeg, int nloc, int r0,
    int jj, int w, int c, const T* urow, T d, double& nk, int& nr)
{
    using VT             = typename Vec16<T>::type;
    constexpr int V      = 16 / (int)sizeof(T);
    const bool zero      = d == T(0);
    const bool use_recip = fabs(d) >= Limits<T>::min_normal();
    const T    recip     = use_recip ? (T)(T(1) / d) : T(1);
    const bool has_next  = jj + 1 < w;
    const bool vec_ok    = ((ldl * sizeof(T)) % 16 == 0) && ((reinterpret_cast<uintptr_t>(loc) & 15) == 0);
    for (int r = rbeg + (int)threadIdx.x; r < nloc; r += kPanelThreads)
    {
        T* row = loc + (size_t)r * ldl;
        if (!zero)
        {
            const T x = row[jj];
            const T l = use_recip ? x * recip : x / d;
            row[jj]   = l;
            int cc    = jj + 1;
            if (vec_ok)
            {
                for (; cc < w && (cc % V) != 0; ++cc)
                {
                    row[cc] = fma(-l, urow[cc], row[cc]);
                }
                for (; cc + V <= w; cc += V)
                {
                    VT       rv = *reinterpret_cast<VT*>(row + cc);
                    const VT uv = *reinterpret_cast<const VT*>(urow + cc);
                    if constexpr (V == 2)
                    {
                        rv.x = fma(-l, uv.x, rv.x);
                        rv.y = fma(-l, uv.y, rv.y);
                    }
                    else
                    {
                        rv.x = fma(-l, uv.x, rv.x);
                        rv.y = fma(-l, uv.y, rv.y);
                        rv.z = fma(-l, uv.z, rv.z);
                        rv.w = fma(-l, uv.w, rv.w);
                    }
                    *reinterpret_cast<VT*>(row + cc) = rv;
                }
            }
            for (; cc < w; ++cc)
            {
                row[cc] = fma(-l, urow[cc], row[cc]);
            }
        }
        if (has_next)
        {
            const double key = pivot_key(row[jj + 1], r0 + r, c + 1);
            if (better(key, r0 + r, nk, nr))
            {
                nk = key;
                nr = r0 + r;
            }
        }
    }
}


// Copy a panel slice (nloc rows of w values at A[r0.., k..], row stride n)
// into shared memory (row stride ldl) or back.  16-byte vectors when the
// rows allow it, and every thread issues 8 loads before it stores any, so a
// thread's loads overlap instead of each waiting for the previous one.
template <typename T, bool TO_SMEM>
__device__ __forceinline__ void panel_slice_copy(T* loc, int ldl, T* A, int n, int r0, int k, int nloc, int w)
{
    using VT         = typename Vec16<T>::type;
    constexpr int V  = 16 / (int)sizeof(T);
    constexpr int B  = 8;
    const bool    vec = (w % V) == 0 && (n % V) == 0 && (k % V) == 0 &&
                     (reinterpret_cast<uintptr_t>(A) & 15) == 0 && ((ldl * sizeof(T)) % 16) == 0 &&
                     (reinterpret_cast<uintptr_t>(loc) & 15) == 0;
    if (vec)
    {
        const int CPR   = w / V;  // chunks per row
        const int total = nloc * CPR;
        for (int e0 = threadIdx.x; e0 < total; e0 += kPanelThreads * B)
        {
            VT v[B];
#pragma unroll
            for (int t = 0; t < B; ++t)
            {
                const int e = e0 + t * kPanelThreads;
                if (e < total)
                {
                    const int r = e / CPR, c = (e - (e / CPR) * CPR) * V;
                    v[t]        = TO_SMEM ? *reinterpret_cast<const VT*>(A + (size_t)(r0 + r) * n + k + c)
                                          : *reinterpret_cast<const VT*>(loc + (size_t)r * ldl + c);
                }
            }
#pragma unroll
            for (int t = 0; t < B; ++t)
            {
                const int e = e0 + t * kPanelThreads;
                if (e < total)
                {
                    const int r = e / CPR, c = (e - (e / CPR) * CPR) * V;
                    if (TO_SMEM)
                        *reinterpret_cast<VT*>(loc + (size_t)r * ldl + c) = v[t];
                    else
                        *reinterpret_cast<VT*>(A + (size_t)(r0 + r) * n + k + c) = v[t];
                }
            }
        }
        return;
    }
    const int total = nloc * w;
    for (int e0 = threadIdx.x; e0 < total; e0 += kPanelThreads * B)
    {
        T v[B];
#pragma unroll
        for (int t = 0; t < B; ++t)
        {
            const int e = e0 + t * kPanelThreads;
            if (e < total)
            {
                const int r = e / w, c = e - (e / w) * w;
                v[t]        = TO_SMEM ? A[(size_t)(r0 + r) * n + k + c] : loc[(size_t)r * ldl + c];
            }
        }
#pragma unroll
        for (int t = 0; t < B; ++t)
        {
            const int e = e0 + t * kPanelThreads;
            if (e < total)
            {
                const int r = e / w, c = e - (e / w) * w;
                if (TO_SMEM)
                    loc[(size_t)r * ldl + c] = v[t];
                else
                    A[(size_t)(r0 + r) * n + k + c] = v[t];
            }
        }
    }
}

constexpr int kMaxSlotsPerLane = (kMaxPanelCtas + 31) / 32;

template <typename T>
__global__ void __launch_bounds__(kPanelThreads) k_panel(T* __restrict__ A, int n, int k, int w,
    int rows_per_cta, int in_smem, int64_t* __restrict__ pivot, PanelWs<T> ws,
    DeviceStatus* __restrict__ st)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) T urow[kNB];
    __shared__ __align__(16) T drow[kNB];
    __shared__ int    piv_loc[kNB];
    __shared__ double red_key[kPanelThreads / 32 + 1];
    __shared__ int    red_row[kPanelThreads / 32 + 1];
    __shared__ int    s_p, s_g, s_abort;

    const int tid  = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int G    = gridDim.x;
    const int b    = blockIdx.x;
    const int r0   = k + b * rows_per_cta;
    const int nloc = max(0, min(n, r0 + rows_per_cta) - r0);

    T*           loc;
    const size_t ldl = in_smem ? (size_t)panel_ldl<T>() : (size_t)n;
    if (in_smem)
    {
        loc = reinterpret_cast<T*>(smem_raw);
        panel_slice_copy<T, true>(loc, (int)ldl, A, n, r0, k, nloc, w);
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

    // candidate for the first column
    double cand_key = -2.0;
    int    cand_row = INT_MAX;
    for (int r = max(0, k - r0) + tid; r < nloc; r += kPanelThreads)
    {
        const double key = pivot_key(loc[r * ldl], r0 + r, k);
        if (better(key, r0 + r, cand_key, cand_row))
        {
            cand_key = key;
            cand_row = r0 + r;
        }
    }
    block_best(cand_key, cand_row, red_key, red_row);

    int64_t first_zero = -1;
    for (int jj = 0; jj < w; ++jj)
    {
        const int c   = k + jj;
        const int par = jj & 1;

        // ---- publish this CTA's candidate row, its header and (owner of row
        // c) the diagonal row as flagged words; no fence is needed
        const uint32_t flag = (uint32_t)(c + 1);
        uint64_t*      H    = ws.hdr + (size_t)par * kMaxPanelCtas * kHdrWords;
        constexpr int  PW   = kNB * LLWords<T>::kWords;
        if (cand_row != INT_MAX && tid < w)
        {
            ll_store(ws.payload + ((size_t)par * kMaxPanelCtas + b) * PW, tid,
                loc[(size_t)(cand_row - r0) * ldl + tid], flag);
        }
        if (c >= r0 && c < r0 + nloc && tid >= 64 && tid < 64 + w)
        {
            ll_store(ws.diag + (size_t)par * PW, tid - 64, loc[(size_t)(c - r0) * ldl + (tid - 64)], flag);
        }
        if (tid == kPanelThreads - 1)
        {
            ll_store(H + (size_t)b * kHdrWords, 0, cand_key, flag);
            st_u64x2(H + (size_t)b * kHdrWords + 2, ll_word((uint32_t)cand_row, flag), ll_word(0u, flag));
        }

        // ---- wait for every CTA's header (all of a lane's slots polled
        // together, bounded) and pick the pivot
        if (warp == 0)
        {
            double         hk[kMaxSlotsPerLane];
            int            hr[kMaxSlotsPerLane];
            bool           done[kMaxSlotsPerLane];
            const uint64_t t0        = global_ns();
            bool           timed_out = false;
#pragma unroll
            for (int t = 0; t < kMaxSlotsPerLane; ++t)
            {
                done[t] = lane + 32 * t >= G;
                hk[t]   = -2.0;
                hr[t]   = INT_MAX;
            }
            for (uint32_t polls = 0;; ++polls)
            {
                bool all = true;
#pragma unroll
                for (int t = 0; t < kMaxSlotsPerLane; ++t)
                {
                    if (!done[t])
                    {
                        const uint64_t* h = H + (size_t)(lane + 32 * t) * kHdrWords;
                        double          kv;
                        uint64_t        w0, w1;
                        const bool      kok = ll_load(h, 0, flag, kv);
                        ld_u64x2(h + 2, w0, w1);
                        if (kok && (uint32_t)(w0 >> 32) == flag)
                        {
                            hk[t]   = kv;
                            hr[t]   = (int)(uint32_t)w0;
                            done[t] = true;
                        }
                        all = all && done[t];
                    }
                }
                if (all)
                {
                    break;
                }
                if ((polls & 63u) == 63u && global_ns() - t0 > kWaitLimitNs)
                {
                    timed_out = true;
                    break;
                }
            }
            double wk = -2.0;
            int    wr = INT_MAX, wg = -1;
#pragma unroll
            for (int t = 0; t < kMaxSlotsPerLane; ++t)
            {
                if (lane + 32 * t < G && better(hk[t], hr[t], wk, wr))
                {
                    wk = hk[t];
                    wr = hr[t];
                    wg = lane + 32 * t;
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
                const double ok   = __shfl_down_sync(0xffffffffu, wk, off);
                const int    orow = __shfl_down_sync(0xffffffffu, wr, off);
                const int    og   = __shfl_down_sync(0xffffffffu, wg, off);
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
        // ---- the pivot row (and, for the owner of row p, the old row c) in
        // one round trip
        const bool own_c = c >= r0 && c < r0 + nloc;
        const bool own_p = p != c && p >= r0 && p < r0 + nloc;
        {
            const uint64_t* src = nullptr;
            int             cc  = -1;
            T*              dst = nullptr;
            if (tid < w)
            {
                src = ws.payload + ((size_t)par * kMaxPanelCtas + g) * PW;
                cc  = tid;
                dst = urow;
            }
            else if (own_p && tid >= 64 && tid < 64 + w)
            {
                src = ws.diag + (size_t)par * PW;
                cc  = tid - 64;
                dst = drow;
            }
            if (src != nullptr)
            {
                const uint64_t t0 = global_ns();
                T              v;
                uint32_t       polls = 0;
                while (!ll_load(src, cc, flag, v))
                {
                    if ((++polls & 63u) == 0 && global_ns() - t0 > kWaitLimitNs)
                    {
                        raise_error(st, DEV_WAIT_TIMEOUT, 2);
                        s_abort = 1;
                        break;
                    }
                }
                dst[cc] = v;
            }
        }
        __syncthreads();
        if (s_abort)
        {
            return;
        }

        // ---- swap rows c and p inside the panel
        if (p != c)
        {
            if (own_c)
            {
                for (int cc = tid; cc < w; cc += kPanelThreads)
                {
                    loc[(size_t)(c - r0) * ldl + cc] = urow[cc];
                }
            }
            if (own_p)
            {
                for (int cc = tid; cc < w; cc += kPanelThreads)
                {
                    loc[(size_t)(p - r0) * ldl + cc] = drow[cc];
                }
            }
            __syncthreads();
        }

        // ---- multipliers, rank-1 update and the next column's candidate
        const T d = urow[jj];
        if (d == T(0) && first_zero < 0)
        {
            first_zero = c;
        }
        double nk = -2.0;
        int    nr = INT_MAX;
        panel_update_rows(loc, ldl, max(0, c + 1 - r0), nloc, r0, jj, w, c, urow, d, nk, nr);
        cand_key = nk;
        cand_row = nr;
        block_best(cand_key, cand_row, red_key, red_row);
    }

    // ---- write the factored slice back
    if (in_smem)
    {
        panel_slice_copy<T, false>(loc, (int)ldl, A, n, r0, k, nloc, w);
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
        if (warp == 0)
        {
            build_perm_list(piv_loc, k, w, ws.perm, lane);
        }
    }
}

// ---------------------------------------------------------------------------
// Panel factorization inside one thread-block cluster.
//
// Used when the panel's rows fit in the shared memory of one cluster of CL
// CTAs (16 where the device allows that cluster size, else 8); W is the
// panel width the slice is laid out for (64, or 32 for the mixed-precision
// factorization's tallest panels, whose 64-column slices would not fit).
// Same arithmetic as k_panel.  Per column, one cluster barrier and two
// block barriers:
//   * warp 0 posts this CTA's candidate (the warps' best, reduced with
//     redux.sync over integer keys that order like the reference's
//     comparisons) with the candidate row's values, and warp 1 of the CTA
//     that holds the diagonal row c posts row c, in shared memory
//     double-buffered by column parity;
//   * after the cluster barrier, warp 0 reads the CL posted keys through
//     distributed shared memory, reduces them, reads the pivot row (and, in
//     the CTA that holds row p, row c) and hands them over through shared
//     memory; block barrier;
//   * row c takes the pivot row, every row below is updated (the thread of
//     row p takes row c's values as it updates it) and the warps reduce
//     their next-column candidates; block barrier.
// A post of parity q is rewritten two columns later, after the next cluster
// barrier, which no CTA passes before every CTA has finished reading it.
// Cluster and block barriers are hardware barriers over co-scheduled CTAs:
// there is no spin-wait in this kernel.
// ---------------------------------------------------------------------------

template <typename T> struct PivKey;
template <> struct PivKey<float>
{
    using type = uint32_t;
};
template <> struct PivKey<double>
{
    using type = unsigned long long;
};

// Integer pivot-search key of value v (larger wins, ties go to the lower
// row): |v|'s bits + 2, 1 for a NaN below the diagonal (never wins over a
// number), the maximum for a NaN on the diagonal (never displaced), and 0
// for "no candidate".  Orders exactly like pivot_key.
template <typename T> __device__ __forceinline__ typename PivKey<T>::type piv_key_bits(T v, bool diag)
{
    using K = typename PivKey<T>::type;
    if (v != v)
    {
        return diag ? ~K(0) : K(1);
    }
    if constexpr (sizeof(T) == 4)
    {
        return (K)__float_as_uint(fabsf(v)) + K(2);
    }
    else
    {
        return (K)__double_as_longlong(fabs(v)) + K(2);
    }
}

// Warp-wide best (key, row) with redux.sync: largest key, then lowest row.
template <typename K> __device__ __forceinline__ void warp_best_bits(K& key, int& row)
{
    if constexpr (sizeof(K) == 4)
    {
        const uint32_t m = __reduce_max_sync(0xffffffffu, key);
        row              = __reduce_min_sync(0xffffffffu, key == m ? row : INT_MAX);
        key              = m;
    }
    else
    {
        const uint32_t hi = __reduce_max_sync(0xffffffffu, (uint32_t)(key >> 32));
        const uint32_t lo = __reduce_max_sync(0xffffffffu, (uint32_t)(key >> 32) == hi ? (uint32_t)key : 0u);
        const K        m  = ((K)hi << 32) | lo;
        row               = __reduce_min_sync(0xffffffffu, key == m ? row : INT_MAX);
        key               = m;
    }
}

__device__ __forceinline__ uint32_t cluster_rank()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cluster_size()
{
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ void cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t map_to_rank(uint32_t local_addr, uint32_t rank)
{
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local_addr), "r"(rank));
    return r;
}
__device__ __forceinline__ float ld_dsmem(const float* local_equiv, uint32_t rank)
{
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(map_to_rank(smem_u32(local_equiv), rank)) : "memory");
    return v;
}
__device__ __forceinline__ double ld_dsmem(const double* local_equiv, uint32_t rank)
{
    double v;
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(map_to_rank(smem_u32(local_equiv), rank)) : "memory");
    return v;
}
__device__ __forceinline__ void ld_dsmem_u64x2(const void* local_equiv, uint32_t rank, unsigned long long& a,
    unsigned long long& b)
{
    asm volatile("ld.shared::cluster.v2.u64 {%0, %1}, [%2];"
                 : "=l"(a), "=l"(b)
                 : "r"(map_to_rank(smem_u32(local_equiv), rank))
                 : "memory");
}

// What one CTA posts for a column: its candidate and the candidate row.
template <typename T, int W> struct alignas(16) ClusterPost
{
    unsigned long long key;  // PivKey<T>::type, widened
    int32_t            row;  // global row, INT_MAX if none
    int32_t            pad;
    T                  data[W];
};

template <typename T, int W> constexpr int cluster_ldl() { return W + 16 / (int)sizeof(T); }
template <typename T, int W> constexpr size_t cluster_row_bytes() { return (size_t)cluster_ldl<T, W>() * sizeof(T); }
// The FP32 32-column kernel (the mixed factorization's) can start with the
// previous panel's interchanges, U12 and update of its own columns; it holds
// that panel's L11 and U12 in 8.3 KB more static shared memory.
template <typename T, int W> constexpr bool cluster_fuses() { return W == 32 && sizeof(T) == 4; }
// Dynamic shared memory of k_panel_cluster<T, W>: 227 KB less its static
// arrays (6 KB; 14 KB for the fusing kernel).
template <typename T, int W> constexpr size_t cluster_dyn_max()
{
    return cluster_fuses<T, W>() ? 227 * 1024 - 14 * 1024 : 227 * 1024 - 6 * 1024;
}

template <typename T, int W>
__global__ void __launch_bounds__(kPanelThreads, 1) k_panel_cluster(T* __restrict__ A, int n, int k, int w,
    int rows_per_cta, int64_t* __restrict__ pivot, PermList* __restrict__ perm, DeviceStatus* __restrict__ st,
    const PermList* __restrict__ pperm, int pk)
{
    using K             = typename PivKey<T>::type;
    using VT            = typename Vec16<T>::type;
    constexpr int V     = 16 / (int)sizeof(T);
    constexpr int LDL   = cluster_ldl<T, W>();
    constexpr int WARPS = kPanelThreads / 32;
    static_assert(W % 32 == 0 && W <= kNB, "panel width");

    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ ClusterPost<T, W> post[2];
    __shared__ __align__(16) T   post_crow[2][W];  // row c, posted by its owner
    __shared__ __align__(16) T   urow[W];          // the pivot row
    __shared__ __align__(16) T   drow[W];          // row c, in the CTA that holds row p
    __shared__ K                 red_key[WARPS];
    __shared__ int               red_row[WARPS];
    __shared__ int               piv_loc[W];
    __shared__ int               s_p;
    constexpr int                FZ = cluster_fuses<T, W>() ? 32 : 1;
    __shared__ __align__(16) T   fz_l[FZ][FZ + 1];  // the previous panel's L11
    __shared__ __align__(16) T   fz_u[FZ][FZ];      // its U12 for this panel's columns

    const int      tid  = threadIdx.x;
    const int      lane = tid & 31;
    const int      warp = tid >> 5;
    const uint32_t CL   = cluster_size();
    const uint32_t b    = cluster_rank();
    const int      r0   = k + (int)b * rows_per_cta;
    const int      nloc = max(0, min(n, r0 + rows_per_cta) - r0);

    // threads per row (a power of two, 1..W/CW_MIN) so that the CTA's rows
    // keep every thread busy; each thread of a row owns CW contiguous columns
    constexpr int CW_MIN = 16 / (int)sizeof(T) > 4 ? 16 / (int)sizeof(T) : 4;  // 4 columns (a vector or two)
    int           TPR    = 1;
    while (TPR * 2 <= W / CW_MIN && rows_per_cta * TPR * 2 <= kPanelThreads)
    {
        TPR *= 2;
    }
    const int CW    = W / TPR;
    const int slots = kPanelThreads / TPR;  // rows updated at once
    const int slot  = tid / TPR;
    const int chunk = tid % TPR;

    T* loc = reinterpret_cast<T*>(smem_raw);
    panel_slice_copy<T, true>(loc, LDL, A, n, r0, k, nloc, w);
    __syncthreads();

    // With pperm: this panel's columns have not yet received the previous
    // panel's (columns [pk, k)) interchanges, U12 and update; apply them here
    // with the arithmetic of k_laswp_trsm and k_trailing (U12 row i takes rows
    // 0..i-1 in order; each element's products summed from zero in order,
    // then subtracted), so the factors are bit-identical to the unfused path.
    if constexpr (FZ == 32)
    {
        if (pperm != nullptr && (k - pk < 1 || k - pk > 32))
        {
            if (tid == 0)
            {
                raise_error(st, DEV_BAD_INPUT, 30);  // the host only fuses panels up to 32 wide
            }
        }
        else if (pperm != nullptr)
        {
            const int pw  = k - pk;
            const int cnt = pperm->count;
            // rows of this CTA that the interchanges replace: their sources'
            // values, from global memory (not yet interchanged there)
            for (int q = pw + warp; q < cnt; q += WARPS)
            {
                const int dst = pperm->dst[q], src = pperm->src[q];
                if (dst != src && dst >= r0 && dst < r0 + nloc)
                {
                    for (int j = lane; j < w; j += 32)
                    {
                        loc[(size_t)(dst - r0) * LDL + j] = A[(size_t)src * n + k + j];
                    }
                }
            }
            // L11 of the previous panel, and its rows' new contents here
            for (int e = tid; e < pw * pw; e += kPanelThreads)
            {
                const int i = e / pw, m = e - i * pw;
                fz_l[i][m]  = A[(size_t)(pk + i) * n + pk + m];
            }
            for (int e = tid; e < 32 * 32; e += kPanelThreads)
            {
                const int i = e >> 5, c = e & 31;
                fz_u[i][c]  = (i < pw && c < w) ? A[(size_t)pperm->src[i] * n + k + c] : T(0);
            }
            __syncthreads();
            // U12 = L11^-1 (those rows), one thread per column
            if (tid < 32)
            {
                T u[32];
#pragma unroll
                for (int i = 0; i < 32; ++i)
                {
                    u[i] = fz_u[i][tid];
                }
#pragma unroll
                for (int pp = 0; pp < 31; ++pp)
                {
#pragma unroll
                    for (int i = pp + 1; i < 32; ++i)
                    {
                        if (i < pw)
                        {
                            u[i] = fma(-fz_l[i][pp], u[pp], u[i]);
                        }
                    }
                }
#pragma unroll
                for (int i = 0; i < 32; ++i)
                {
                    fz_u[i][tid] = u[i];
                }
            }
            __syncthreads();
            if (b == 0)
            {
                for (int e = tid; e < pw * w; e += kPanelThreads)
                {
                    const int i = e / w, c = e - i * w;
                    A[(size_t)(pk + i) * n + k + c] = fz_u[i][c];
                }
            }
            // this CTA's rows -= L21 U12 (L21: the previous panel's final
            // rows, in global memory); a thread per row, all 32 columns
            const bool lvec = (n % 4) == 0 && (pk % 4) == 0 && (reinterpret_cast<uintptr_t>(A) & 15) == 0;
            for (int r = tid; r < nloc; r += kPanelThreads)
            {
                const T* lr = A + (size_t)(r0 + r) * n + pk;
                T        lv[32];
                if (lvec && pw == 32)
                {
#pragma unroll
                    for (int m = 0; m < 32; m += 4)
                    {
                        const float4 q = *reinterpret_cast<const float4*>(lr + m);
                        lv[m] = q.x, lv[m + 1] = q.y, lv[m + 2] = q.z, lv[m + 3] = q.w;
                    }
                }
                else
                {
#pragma unroll
                    for (int m = 0; m < 32; ++m)
                    {
                        lv[m] = m < pw ? lr[m] : T(0);
                    }
                }
                T acc[32];
#pragma unroll
                for (int c = 0; c < 32; ++c)
                {
                    acc[c] = T(0);
                }
#pragma unroll
                for (int m = 0; m < 32; ++m)
                {
                    if (m < pw)
                    {
#pragma unroll
                        for (int c = 0; c < 32; c += 4)
                        {
                            const float4 uq = *reinterpret_cast<const float4*>(&fz_u[m][c]);
                            acc[c]          = fma(lv[m], uq.x, acc[c]);
                            acc[c + 1]      = fma(lv[m], uq.y, acc[c + 1]);
                            acc[c + 2]      = fma(lv[m], uq.z, acc[c + 2]);
                            acc[c + 3]      = fma(lv[m], uq.w, acc[c + 3]);
                        }
                    }
                }
                T* row = loc + (size_t)r * LDL;
#pragma unroll
                for (int c = 0; c < 32; ++c)
                {
                    if (c < w)
                    {
                        row[c] = row[c] - acc[c];
                    }
                }
            }
            __syncthreads();
        }
    }

    {
        K   ck = 0;
        int cr = INT_MAX;
        for (int r = max(0, k - r0) + tid; r < nloc; r += kPanelThreads)
        {
            const K key = piv_key_bits(loc[(size_t)r * LDL], r0 + r == k);
            if (key > ck)
            {
                ck = key;
                cr = r0 + r;
            }
        }
        warp_best_bits(ck, cr);
        if (lane == 0)
        {
            red_key[warp] = ck;
            red_row[warp] = cr;
        }
    }
    __syncthreads();

    int64_t first_zero = -1;
    for (int jj = 0; jj < w; ++jj)
    {
        const int      c      = k + jj;
        const int      par    = jj & 1;
        const uint32_t rank_c = (uint32_t)((c - k) / rows_per_cta);
        // ---- post: warp 0 the CTA's candidate, warp 1 of row c's CTA row c
        if (warp == 0)
        {
            K   key = lane < WARPS ? red_key[lane] : K(0);
            int row = lane < WARPS ? red_row[lane] : INT_MAX;
            warp_best_bits(key, row);
            if (lane == 0)
            {
                post[par].key = (unsigned long long)key;
                post[par].row = row;
            }
            if (row != INT_MAX)
            {
                const T* src = loc + (size_t)(row - r0) * LDL;
                for (int j = lane; j < w; j += 32)
                {
                    post[par].data[j] = src[j];
                }
            }
        }
        else if (warp == 1 && b == rank_c)
        {
            const T* src = loc + (size_t)(c - r0) * LDL;
            for (int j = lane; j < w; j += 32)
            {
                post_crow[par][j] = src[j];
            }
        }
        cluster_barrier();
        // ---- the pivot (warp 0): keys, then the pivot row (and row c)
        if (warp == 0)
        {
            unsigned long long hk = 0, hr = INT_MAX;
            if (lane < (int)CL)
            {
                ld_dsmem_u64x2(&post[par], (uint32_t)lane, hk, hr);
            }
            K   pk = (K)hk;
            int p  = (int)(uint32_t)hr;
            warp_best_bits(pk, p);
            const uint32_t rank_p = (uint32_t)((p - k) / rows_per_cta);
            for (int j = lane; j < w; j += 32)
            {
                urow[j] = ld_dsmem(&post[par].data[j], rank_p);
            }
            if (p != c && rank_p == b)
            {
                for (int j = lane; j < w; j += 32)
                {
                    drow[j] = ld_dsmem(&post_crow[par][j], rank_c);
                }
            }
            if (lane == 0)
            {
                s_p         = p;
                piv_loc[jj] = p;  // pivot[] is written after the last column: a global store
                                  // here would hold up the next release barrier
            }
        }
        __syncthreads();
        const int  p     = s_p;
        const bool own_p = p != c && p >= r0 && p < r0 + nloc;
        const T    d     = urow[jj];
        if (d == T(0) && first_zero < 0)
        {
            first_zero = c;
        }
        // row c takes the pivot row (no other thread reads row c this column)
        if (p != c && b == rank_c)
        {
            for (int j = tid; j < w; j += kPanelThreads)
            {
                loc[(size_t)(c - r0) * LDL + j] = urow[j];
            }
        }
        // multipliers, rank-1 update and the next column's candidates: TPR
        // threads per row, each on a chunk of CW columns (the multiplier is
        // computed by each of them, identically)
        const bool zero      = d == T(0);
        const bool use_recip = fabs(d) >= Limits<T>::min_normal();
        const T    recip     = use_recip ? (T)(T(1) / d) : T(1);
        const bool has_next  = jj + 1 < w;
        const int  cc0       = chunk * CW;  // this thread's columns [cc0, cc0 + CW)
        K          ck        = 0;
        int        cr        = INT_MAX;
        const int rb = max(0, c + 1 - r0);
        // the same trip count in every thread, so that the warp-wide sync
        // below is reached by all lanes
        const int trips = nloc > rb ? (nloc - rb + slots - 1) / slots : 0;
        for (int t = 0; t < trips; ++t)
        {
            const int r = rb + slot + t * slots;
            if (r >= nloc)
            {
                if (TPR > 1 && !zero)
                {
                    __syncwarp();
                }
                continue;
            }
            T*         row     = loc + (size_t)r * LDL;
            const bool swapped = own_p && r0 + r == p;
            const T*   src     = swapped ? drow : row;
            if (swapped)
            {
                // row c's multipliers move with it (vectors, cc0 is aligned)
                const int je = min(cc0 + CW, jj);
                int       j  = cc0;
                for (; j + V <= je; j += V)
                {
                    *reinterpret_cast<VT*>(row + j) = *reinterpret_cast<const VT*>(drow + j);
                }
                for (; j < je; ++j)
                {
                    row[j] = drow[j];
                }
            }
            if (!zero)
            {
                const T x = src[jj];
                const T l = use_recip ? x * recip : x / d;
                if (TPR > 1)
                {
                    __syncwarp();  // every thread of the row has read a_rj before it is overwritten
                }
                if (jj >= cc0 && jj < cc0 + CW)
                {
                    row[jj] = l;
                }
                const int ce = min(cc0 + CW, w);
                int       cc = max(cc0, jj + 1);
                for (; cc < ce && (cc % V) != 0; ++cc)
                {
                    row[cc] = fma(-l, urow[cc], src[cc]);
                }
                for (; cc + V <= ce; cc += V)
                {
                    const VT sv = *reinterpret_cast<const VT*>(src + cc);
                    const VT uv = *reinterpret_cast<const VT*>(urow + cc);
                    VT       rv;
                    if constexpr (V == 2)
                    {
                        rv.x = fma(-l, uv.x, sv.x);
                        rv.y = fma(-l, uv.y, sv.y);
                    }
                    else
                    {
                        rv.x = fma(-l, uv.x, sv.x);
                        rv.y = fma(-l, uv.y, sv.y);
                        rv.z = fma(-l, uv.z, sv.z);
                        rv.w = fma(-l, uv.w, sv.w);
                    }
                    *reinterpret_cast<VT*>(row + cc) = rv;
                }
                for (; cc < ce; ++cc)
                {
                    row[cc] = fma(-l, urow[cc], src[cc]);
                }
            }
            else if (swapped)
            {
                for (int j = max(cc0, jj); j < cc0 + CW && j < w; ++j)
                {
                    row[j] = drow[j];
                }
            }
            if (has_next && jj + 1 >= cc0 && jj + 1 < cc0 + CW)
            {
                const K key = piv_key_bits(row[jj + 1], r0 + r == c + 1);
                if (key > ck)
                {
                    ck = key;
                    cr = r0 + r;
                }
            }
        }
        warp_best_bits(ck, cr);
        if (lane == 0)
        {
            red_key[warp] = ck;
            red_row[warp] = cr;
        }
        __syncthreads();
    }
    cluster_barrier();  // no CTA exits while its shared memory may still be read

    panel_slice_copy<T, false>(loc, LDL, A, n, r0, k, nloc, w);
    if (b == 0)
    {
        if (tid == 0 && first_zero >= 0 && st->first_zero < 0)
        {
            st->first_zero = first_zero;
        }
        if (warp == 0)
        {
            build_perm_list(piv_loc, k, w, perm, lane);
        }
        else if (warp == 1)
        {
            for (int j = lane; j < w; j += 32)
            {
                pivot[k + j] = (int64_t)piv_loc[j] + 1;
            }
        }
    }
}

// The floor of k_panel_cluster's per-column exchange: the same cluster and
// threads, warp 0's post of a key, the cluster barrier, warp 0's reads of
// the CL keys and of W pivot-row values through distributed shared memory,
// and the two block barriers; no slice, no update, no candidate search.
// Thread 0 of rank 0 writes the elapsed %globaltimer nanoseconds of
// `columns` columns to *ns.
template <typename T, int W>
__global__ void __launch_bounds__(kPanelThreads, 1) k_panel_exchange_floor(int columns,
    unsigned long long* __restrict__ ns)
{
    using K             = typename PivKey<T>::type;
    constexpr int WARPS = kPanelThreads / 32;
    __shared__ ClusterPost<T, W> post[2];
    __shared__ __align__(16) T   urow[W];
    __shared__ K                 red_key[WARPS];
    __shared__ int               red_row[WARPS];
    __shared__ int               s_p;
    const int      tid  = threadIdx.x;
    const int      lane = tid & 31;
    const int      warp = tid >> 5;
    const uint32_t CL   = cluster_size();
    const uint32_t b    = cluster_rank();
    for (int j = tid; j < W; j += kPanelThreads)
    {
        post[0].data[j] = T(j);
        post[1].data[j] = T(j);
    }
    if (lane == 0)
    {
        red_key[warp] = (K)(warp * 7 % 5 + 2);
        red_row[warp] = warp + (int)b * 100;
    }
    cluster_barrier();
    const uint64_t t0  = global_ns();
    T              acc = T(0);
    for (int jj = 0; jj < columns; ++jj)
    {
        const int par = jj & 1;
        if (warp == 0)
        {
            K   key = lane < WARPS ? red_key[lane] : K(0);
            int row = lane < WARPS ? red_row[lane] : INT_MAX;
            warp_best_bits(key, row);
            if (lane == 0)
            {
                post[par].key = (unsigned long long)key;
                post[par].row = row;
            }
        }
        cluster_barrier();
        if (warp == 0)
        {
            unsigned long long hk = 0, hr = INT_MAX;
            if (lane < (int)CL)
            {
                ld_dsmem_u64x2(&post[par], (uint32_t)lane, hk, hr);
            }
            K   pk = (K)hk;
            int p  = (int)(uint32_t)hr;
            warp_best_bits(pk, p);
            const uint32_t rank_p = (uint32_t)(p % 100) % CL;
            for (int j = lane; j < W; j += 32)
            {
                urow[j] = ld_dsmem(&post[par].data[j], rank_p);
            }
            if (lane == 0)
            {
                s_p = p;
            }
        }
        __syncthreads();
        acc += urow[jj % W];
        if (lane == 0)
        {
            red_key[warp] = (K)(s_p & 1023) + K(2);
            red_row[warp] = s_p + warp;
        }
        __syncthreads();
    }
    const uint64_t t1 = global_ns();
    cluster_barrier();
    if (b == 0 && tid == 0)
    {
        *ns = (t1 - t0) + (acc == T(-1) ? 1ull : 0ull);
    }
}

// Row interchanges outside the panel and, right of it, U12 = L11^-1 A12.
// CTA b < n_left: columns [left_begin + b*kSwapCols, ...) of
// [left_begin, left_end), interchanges only; otherwise columns of
// [right_begin, right_end) (right_begin >= k+w), with U12 solved for those
// below u12_end.  (The plain LU passes left [0, k) and right [k+w, n); the
// mixed LU's look-ahead applies an outer block's interchanges right of the
// block in a later launch with only a left range, and inside a block first
// the next panel's columns, then the rest of the block.)  256 threads: 4 row groups x 64 columns for the gather/scatter
// (each thread loads its up to 32 rows before storing, so the loads overlap),
// then one thread per column for the substitution.
constexpr int kSwapThreads = 256;
constexpr int kSwapGroups  = kSwapThreads / kSwapCols;
constexpr int kSwapPerThr  = (2 * kNB + kSwapGroups - 1) / kSwapGroups;

template <typename T> constexpr size_t laswp_smem_bytes()
{
    return sizeof(T) * (2 * kNB * kSwapCols + kNB * (kNB + 1));
}

template <typename T>
__global__ void __launch_bounds__(kSwapThreads) k_laswp_trsm(T* __restrict__ A, int n, int k, int w,
    const PermList* __restrict__ perm, int n_left, int u12_end, int left_begin, int left_end, int right_end,
    int right_begin)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T(*staged)[kSwapCols] = reinterpret_cast<T(*)[kSwapCols]>(smem_raw);  // [2*kNB]
    T(*L11)[kNB + 1] = reinterpret_cast<T(*)[kNB + 1]>(smem_raw + sizeof(T) * 2 * kNB * kSwapCols);

    const int  tid   = threadIdx.x;
    const int  cl    = tid % kSwapCols;
    const int  rg    = tid / kSwapCols;
    const int  c0    = (int)blockIdx.x < n_left ? left_begin + (int)blockIdx.x * kSwapCols
                                                : right_begin + ((int)blockIdx.x - n_left) * kSwapCols;
    // `left`: only the interchanges (the left range, or right of the panel
    // at or beyond u12_end, whose U12 rows are solved later)
    const bool left  = (int)blockIdx.x < n_left || c0 >= u12_end;
    const int  cend  = (int)blockIdx.x < n_left ? left_end : right_end;
    const int  col   = c0 + cl;
    const bool valid = col < cend;
    const int  cnt   = perm->count;

    {
        T v[kSwapPerThr];
#pragma unroll
        for (int t = 0; t < kSwapPerThr; ++t)
        {
            const int q = rg + kSwapGroups * t;
            v[t]        = (valid && q < cnt) ? A[(size_t)perm->src[q] * n + col] : T(0);
        }
#pragma unroll
        for (int t = 0; t < kSwapPerThr; ++t)
        {
            const int q = rg + kSwapGroups * t;
            if (q < cnt)
            {
                staged[q][cl] = v[t];
            }
        }
    }
    if (!left)
    {
        // L11, 16 loads per thread in flight before the stores
        constexpr int PT = kNB * kNB / kSwapThreads;
        T             lv[PT];
#pragma unroll
        for (int t = 0; t < PT; ++t)
        {
            const int e = tid + t * kSwapThreads;
            const int i = e / kNB, p = e - (e / kNB) * kNB;
            lv[t]       = (i < w && p < i) ? A[(size_t)(k + i) * n + k + p] : T(0);
        }
#pragma unroll
        for (int t = 0; t < PT; ++t)
        {
            const int e = tid + t * kSwapThreads;
            L11[e / kNB][e - (e / kNB) * kNB] = lv[t];
        }
    }
    __syncthreads();
    // scatter: every touched row (left), or the rows displaced below the
    // panel (right; the panel rows receive U12 below)
    if (valid)
    {
        for (int q = (left ? 0 : w) + rg; q < cnt; q += kSwapGroups)
        {
            const int dst = perm->dst[q];
            if (!left || dst != perm->src[q])
            {
                A[(size_t)dst * n + col] = staged[q][cl];
            }
        }
    }
    if (left)
    {
        return;
    }
    // U12 = L11^-1 A12 on the staged panel rows, column-oriented: step p
    // applies row p (final) to rows p+1..w-1, so row i receives the updates
    // of rows 0..i-1 in that order, as in the reference's row-axpy loop.
    for (int p = 0; p + 1 < w; ++p)
    {
        __syncthreads();
        const T xp = staged[p][cl];
        for (int i = p + 1 + rg; i < w; i += kSwapGroups)
        {
            staged[i][cl] = fma(-L11[i][p], xp, staged[i][cl]);
        }
    }
    __syncthreads();
    if (valid)
    {
        for (int i = rg; i < w; i += kSwapGroups)
        {
            A[(size_t)(k + i) * n + col] = staged[i][cl];
        }
    }
}

// ---------------------------------------------------------------------------
// cp.async helpers (Ampere-style asynchronous global->shared copies).
// `bytes` is 16 or the element size; src_bytes = 0 zero-fills.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(gmem),
        "r"(valid ? 16 : 0)
        : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(s), "l"(gmem),
        "r"(valid ? 8 : 0)
        : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem, bool valid)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(s), "l"(gmem),
        "r"(valid ? 4 : 0)
        : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Copy `count` contiguous elements (count * sizeof(T) a multiple of 16 when
// vec16) from gmem to smem, zero-filling when !valid; chunks are distributed
// by the caller.
template <typename T>
__device__ __forceinline__ void cp_async_chunk(T* smem, const T* gmem, bool valid, bool vec16)
{
    if (vec16)
    {
        cp_async16(smem, gmem, valid);
    }
    else
    {
#pragma unroll
        for (int e = 0; e < (int)(16 / sizeof(T)); ++e)
        {
            if (sizeof(T) == 8)
                cp_async8(smem + e, gmem + e, valid);
            else
                cp_async4(smem + e, gmem + e, valid);
        }
    }
}

// ---------------------------------------------------------------------------
// Trailing update A22 -= L21 U12.
//
// A CTA owns a band of kBandM = 128 rows of A22 and a chunk of kChunkN = 256
// of its columns.  The band's L21 rows (128 x w) are staged once in shared
// memory; the chunk is streamed as 8 tiles of 128 x 32 with a two-stage
// cp.async pipeline carrying the tile's U12 slice (w x 32) and its A22 tile.
// For every element, delta is accumulated from zero over the panel's w
// columns in order with fused multiply-adds and then subtracted from A22 once
// (the reference computes delta with its GEMM and subtracts it in a second
// pass).  Thread (warp, tr = lane/8, tc = lane%8) owns tile rows
// warp*32 + tr + 4i (i < 8) and columns 2*tc + 16*j + e (j, e < 2).
// L21 is stored with the 16-byte chunk index XORed by (row % 4) so the four
// rows a warp reads at one depth index hit different banks.
// ---------------------------------------------------------------------------
constexpr int kBandM  = 128;
constexpr int kTileNc = 32;
constexpr int kChunkN = 256;

template <typename T> constexpr int chunk_elems() { return 16 / (int)sizeof(T); }

template <typename T> constexpr size_t trailing_smem_bytes()
{
    return sizeof(T) * ((size_t)kBandM * kNB + 2 * ((size_t)kNB * kTileNc + (size_t)kBandM * kTileNc));
}

template <typename T>
__device__ __forceinline__ void trailing_issue_tile(T* Bs, T* Cs, const T* U12, const T* C, int n,
    int w, int rest, int ncols, int m0, int nt0, bool vec16)
{
    constexpr int CE = chunk_elems<T>();
    constexpr int BC = kTileNc / CE;  // chunks per tile row
    // U12 slice: w x 32
    for (int e = threadIdx.x; e < kNB * BC; e += 128)
    {
        const int  p = e / BC, q = e - (e / BC) * BC;
        const int  col = nt0 + q * CE;
        const bool v   = p < w && col < ncols;
        cp_async_chunk(Bs + p * kTileNc + q * CE, v ? U12 + (size_t)p * n + col : U12, v, vec16);
    }
    // A22 tile: 128 x 32
    for (int e = threadIdx.x; e < kBandM * BC; e += 128)
    {
        const int  r = e / BC, q = e - (e / BC) * BC;
        const int  col = nt0 + q * CE;
        const bool v   = m0 + r < rest && col < ncols;
        cp_async_chunk(Cs + r * kTileNc + q * CE, v ? C + (size_t)(m0 + r) * n + col : C, v, vec16);
    }
}

template <typename T>
__global__ void __launch_bounds__(128, 1) k_trailing(T* __restrict__ A, int n, int k, int w, int ncols,
    int c_off)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int CE = chunk_elems<T>();
    T*            As = reinterpret_cast<T*>(smem_raw);           // [kBandM][kNB], swizzled
    T*            Bs = As + kBandM * kNB;                          // [2][kNB][kTileNc]
    T*            Cs = Bs + 2 * kNB * kTileNc;                     // [2][kBandM][kTileNc]

    const int rest = n - k - w;  // rows of A22; its columns are [c_off, c_off + ncols) from k + w
    const int m0   = blockIdx.y * kBandM;
    const int n0   = blockIdx.x * kChunkN;
    const int tid  = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int tr   = lane >> 3;
    const int tc   = lane & 7;
    const bool vec16 = (((size_t)n * sizeof(T)) % 16 == 0) && ((reinterpret_cast<uintptr_t>(A) & 15) == 0);

    const T* L21 = A + (size_t)(k + w) * n + k;
    const T* U12 = A + (size_t)k * n + k + w + c_off;
    T*       C   = A + (size_t)(k + w) * n + k + w + c_off;

    // stage the band's L21 rows (chunk index XOR (row % 4))
    {
        constexpr int AC = kNB / CE;  // chunks per row
        for (int e = tid; e < kBandM * AC; e += 128)
        {
            const int  r = e / AC, q = e - (e / AC) * AC;
            const bool v = m0 + r < rest && q * CE < w;
            cp_async_chunk(As + r * kNB + (q ^ (r & 3)) * CE,
                v ? L21 + (size_t)(m0 + r) * n + q * CE : L21, v, vec16);
        }
    }
    const int ntiles = min(kChunkN, ncols - n0) > 0 ? (min(kChunkN, ncols - n0) + kTileNc - 1) / kTileNc : 0;
    trailing_issue_tile(Bs, Cs, U12, C, n, w, rest, ncols, m0, n0, vec16);
    cp_async_commit();
    if (ntiles > 1)
    {
        trailing_issue_tile(Bs + kNB * kTileNc, Cs + kBandM * kTileNc, U12, C, n, w, rest, ncols, m0,
            n0 + kTileNc, vec16);
    }
    cp_async_commit();

    // element p of row r lives at As[r][((p / CE) ^ (r % 4)) * CE + p % CE]
    const T* arow = As + (warp * 32 + tr) * kNB;
    const int sw  = tr & 3;  // rows warp*32 + tr + 4i all have row % 4 == tr % 4

    for (int t = 0; t < ntiles; ++t)
    {
        cp_async_wait<1>();
        __syncthreads();
        const T* B  = Bs + (t & 1) * kNB * kTileNc;
        T*       Ct = Cs + (t & 1) * kBandM * kTileNc;

        T acc[8][4];
#pragma unroll
        for (int i = 0; i < 8; ++i)
        {
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                acc[i][j] = T(0);
            }
        }
        for (int p = 0; p < w; ++p)
        {
            const int pa = ((p / CE) ^ sw) * CE + (p % CE);
            T         a[8], bv[4];
#pragma unroll
            for (int i = 0; i < 8; ++i)
            {
                a[i] = arow[4 * i * kNB + pa];
            }
#pragma unroll
            for (int j = 0; j < 2; ++j)
            {
                const auto v2 = *reinterpret_cast<const typename Vec2<T>::type*>(B + p * kTileNc + 2 * tc + 16 * j);
                bv[2 * j]     = v2.x;
                bv[2 * j + 1] = v2.y;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i)
            {
#pragma unroll
                for (int j = 0; j < 4; ++j)
                {
                    acc[i][j] = fma(a[i], bv[j], acc[i][j]);
                }
            }
        }
        const int nt0 = n0 + t * kTileNc;
#pragma unroll
        for (int i = 0; i < 8; ++i)
        {
            const int rl = warp * 32 + tr + 4 * i;
            const int r  = m0 + rl;
            if (r < rest)
            {
                T* crow = C + (size_t)r * n;
#pragma unroll
                for (int j = 0; j < 2; ++j)
                {
                    const int cl = 2 * tc + 16 * j;
                    const auto v2 = *reinterpret_cast<const typename Vec2<T>::type*>(Ct + rl * kTileNc + cl);
                    if (nt0 + cl < ncols)
                    {
                        crow[nt0 + cl] = v2.x - acc[i][2 * j];
                    }
                    if (nt0 + cl + 1 < ncols)
                    {
                        crow[nt0 + cl + 1] = v2.y - acc[i][2 * j + 1];
                    }
                }
            }
        }
        __syncthreads();  // buffer (t & 1) is free again
        if (t + 2 < ntiles)
        {
            trailing_issue_tile(Bs + (t & 1) * kNB * kTileNc, Cs + (t & 1) * kBandM * kTileNc, U12, C,
                n, w, rest, ncols, m0, n0 + (t + 2) * kTileNc, vec16);
        }
        cp_async_commit();
    }
    cp_async_wait<0>();
}

static __global__ void k_status_init(DeviceStatus* st, PermList* perm)
{
    if (threadIdx.x == 0)
    {
        st->error      = 0;
        st->error_site = 0;
        st->first_zero = -1;
        st->info       = 0;
        if (perm != nullptr)
        {
            perm->count = 0;
        }
    }
}

static __global__ void k_status_finish(DeviceStatus* st)
{
    if (threadIdx.x == 0)
    {
        st->info = st->first_zero + 1;
    }
}

}  // namespace b200la
